/*
 * Test infrastructure (oracle harness), not product code.
 *
 * Implementation of the minimal MPI interface in mpi.h.  With the environment
 * variable CGFDM_SHIM_NPROC unset or 1 the program is one rank and every
 * neighbour is MPI_PROC_NULL, which reproduces the reference's single-rank
 * semantics (zero halos, init_MPI.cpp:40-55).  With CGFDM_SHIM_NPROC=N the
 * first rank forks N-1 more ranks inside MPI_Init; the ranks then exchange
 * halos (MPI_Sendrecv) through one POSIX shared-memory mailbox per ordered
 * rank pair and synchronise through a sense-reversing barrier in a shared
 * anonymous mapping.  Every wait is bounded (CGFDM_SHIM_TIMEOUT seconds,
 * default 900): on expiry all ranks are killed and the run exits non-zero.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <fcntl.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define SHIM_MAX_RANKS 1024
#define SHIM_MAX_REDUCE 16

typedef struct {
  volatile int64_t count;      /* ranks arrived in the current episode */
  volatile int64_t sense;      /* flips when an episode completes */
  volatile int64_t abort_code; /* nonzero once any rank aborts */
  volatile pid_t pids[SHIM_MAX_RANKS];
  double reduce[SHIM_MAX_RANKS][SHIM_MAX_REDUCE];
} shim_ctl;

typedef struct {
  volatile int64_t seq_written;
  volatile int64_t seq_read;
  volatile int64_t size;
  int64_t pad[5];
} mbox_hdr;

static int g_rank = 0, g_size = 1;
static int g_dims[3] = {1, 1, 1};
static shim_ctl *g_ctl = NULL;
static pid_t g_leader = 0;
static int64_t g_local_sense = 0;
static double g_timeout = 900.0;

typedef struct {
  mbox_hdr *hdr;
  size_t mapped; /* bytes mapped, header included */
  int fd;
} mbox_map;
static mbox_map *g_send = NULL, *g_recv = NULL; /* indexed by peer rank */

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void shim_die(int code, const char *why) {
  fprintf(stderr, "[mpi-shim rank %d] abort(%d): %s\n", g_rank, code, why);
  fflush(stderr);
  if (g_ctl) {
    __atomic_store_n(&g_ctl->abort_code, code ? code : 1, __ATOMIC_SEQ_CST);
    for (int r = 0; r < g_size; ++r)
      if (r != g_rank && g_ctl->pids[r] > 0) kill(g_ctl->pids[r], SIGKILL);
  }
  _exit(code ? code : 1);
}

static void backoff(double t0, long *spins) {
  if (g_ctl && __atomic_load_n(&g_ctl->abort_code, __ATOMIC_ACQUIRE))
    _exit((int)g_ctl->abort_code);
  if (++*spins < 2000) return;
  if ((*spins & 255) == 0 && now_s() - t0 > g_timeout) shim_die(97, "timeout waiting on a peer");
  struct timespec ts = {0, 20000};
  nanosleep(&ts, NULL);
}

int MPI_Init(int *argc, char ***argv) {
  (void)argc; (void)argv;
  const char *e = getenv("CGFDM_SHIM_NPROC");
  const char *t = getenv("CGFDM_SHIM_TIMEOUT");
  if (t) g_timeout = atof(t);
  g_size = e ? atoi(e) : 1;
  if (g_size < 1) g_size = 1;
  if (g_size > SHIM_MAX_RANKS) shim_die(98, "too many ranks");
  g_rank = 0;
  g_leader = getpid();
  g_send = (mbox_map *)calloc(g_size, sizeof(mbox_map));
  g_recv = (mbox_map *)calloc(g_size, sizeof(mbox_map));
  if (g_size == 1) return MPI_SUCCESS;
  g_ctl = (shim_ctl *)mmap(NULL, sizeof(shim_ctl), PROT_READ | PROT_WRITE,
                           MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (g_ctl == MAP_FAILED) shim_die(99, "mmap control block");
  memset((void *)g_ctl, 0, sizeof(shim_ctl));
  g_ctl->pids[0] = getpid();
  fflush(NULL);
  for (int r = 1; r < g_size; ++r) {
    pid_t p = fork();
    if (p < 0) shim_die(99, "fork");
    if (p == 0) {
      g_rank = r;
      g_ctl->pids[r] = getpid();
      break;
    }
    g_ctl->pids[r] = p;
  }
  MPI_Barrier(MPI_COMM_WORLD);
  return MPI_SUCCESS;
}

static void mbox_name(char *buf, int src, int dst) {
  snprintf(buf, 128, "/cgfdmshim.%d.%d.%d", (int)g_leader, src, dst);
}

static void mbox_unlink_all(void) {
  char name[128];
  for (int s = 0; s < g_size; ++s)
    for (int d = 0; d < g_size; ++d) {
      mbox_name(name, s, d);
      shm_unlink(name);
    }
}

int MPI_Finalize(void) {
  if (g_size > 1) {
    MPI_Barrier(MPI_COMM_WORLD);
    if (g_rank == 0) {
      for (int r = 1; r < g_size; ++r) {
        int st = 0;
        waitpid(g_ctl->pids[r], &st, 0);
      }
      mbox_unlink_all();
    } else {
      fflush(NULL);
      _exit(0);
    }
  }
  return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int code) {
  (void)comm;
  if (g_size > 1 && g_rank == 0) mbox_unlink_all();
  shim_die(code, "MPI_Abort called by the program");
  return code;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = g_rank; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = g_size; return 0; }
int MPI_Comm_free(MPI_Comm *comm) { (void)comm; return 0; }

int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  if (g_size == 1) return 0;
  g_local_sense = !g_local_sense;
  int64_t arrived = __atomic_add_fetch(&g_ctl->count, 1, __ATOMIC_ACQ_REL);
  if (arrived == g_size) {
    __atomic_store_n(&g_ctl->count, 0, __ATOMIC_RELAXED);
    __atomic_store_n(&g_ctl->sense, g_local_sense, __ATOMIC_RELEASE);
  } else {
    double t0 = now_s();
    long spins = 0;
    while (__atomic_load_n(&g_ctl->sense, __ATOMIC_ACQUIRE) != g_local_sense) backoff(t0, &spins);
  }
  return 0;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart) {
  (void)old; (void)periods; (void)reorder;
  int prod = 1;
  for (int d = 0; d < 3; ++d) {
    g_dims[d] = d < ndims ? dims[d] : 1;
    prod *= g_dims[d];
  }
  if (prod != g_size) {
    char msg[160];
    snprintf(msg, sizeof msg, "PX*PY*PZ=%d but CGFDM_SHIM_NPROC=%d", prod, g_size);
    shim_die(1002, msg);
  }
  *cart = 1;
  return 0;
}

/* Row-major rank order (last dimension fastest), as in the MPI standard. */
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords) {
  (void)comm;
  int c[3];
  c[2] = rank % g_dims[2];
  c[1] = (rank / g_dims[2]) % g_dims[1];
  c[0] = rank / (g_dims[2] * g_dims[1]);
  for (int d = 0; d < maxdims && d < 3; ++d) coords[d] = c[d];
  return 0;
}

static int cart_rank(const int *c) {
  for (int d = 0; d < 3; ++d)
    if (c[d] < 0 || c[d] >= g_dims[d]) return MPI_PROC_NULL;
  return (c[0] * g_dims[1] + c[1]) * g_dims[2] + c[2];
}

int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *src, int *dst) {
  int c[3];
  MPI_Cart_coords(comm, g_rank, 3, c);
  int cs[3] = {c[0], c[1], c[2]}, cd[3] = {c[0], c[1], c[2]};
  cs[dir] -= disp;
  cd[dir] += disp;
  *src = cart_rank(cs);
  *dst = cart_rank(cd);
  return 0;
}

static size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_FLOAT: return 4;
    case MPI_INT: return 4;
    case MPI_DOUBLE: return 8;
    default: return 1;
  }
}

static void map_mbox(mbox_map *m, int src, int dst, size_t need, int create) {
  char name[128];
  mbox_name(name, src, dst);
  if (m->fd <= 0) {
    double t0 = now_s();
    long spins = 0;
    for (;;) {
      m->fd = shm_open(name, O_RDWR | (create ? O_CREAT : 0), 0600);
      if (m->fd >= 0) break;
      if (errno != ENOENT) shim_die(96, "shm_open");
      backoff(t0, &spins);
    }
  }
  struct stat st;
  size_t want = sizeof(mbox_hdr) + need;
  double t1 = now_s();
  long spins1 = 0;
  for (;;) {
    fstat(m->fd, &st);
    if ((size_t)st.st_size >= want) break;
    if (create) {
      if (ftruncate(m->fd, (off_t)want) != 0) shim_die(96, "ftruncate");
    } else {
      backoff(t1, &spins1);
    }
  }
  if (m->hdr && m->mapped >= (size_t)st.st_size) return;
  if (m->hdr) munmap((void *)m->hdr, m->mapped);
  m->mapped = (size_t)st.st_size;
  m->hdr = (mbox_hdr *)mmap(NULL, m->mapped, PROT_READ | PROT_WRITE, MAP_SHARED, m->fd, 0);
  if (m->hdr == MAP_FAILED) shim_die(96, "mmap mailbox");
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                 int sendtag, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status *status) {
  (void)sendtag; (void)recvtag; (void)comm;
  if (status) { status->MPI_SOURCE = source; status->MPI_TAG = recvtag; status->MPI_ERROR = 0; }
  if (g_size == 1) return 0;
  if (dest >= 0) {
    size_t bytes = (size_t)sendcount * type_size(sendtype);
    mbox_map *m = &g_send[dest];
    if (!m->hdr) map_mbox(m, g_rank, dest, bytes, 1);
    double t0 = now_s();
    long spins = 0;
    while (__atomic_load_n(&m->hdr->seq_written, __ATOMIC_ACQUIRE) !=
           __atomic_load_n(&m->hdr->seq_read, __ATOMIC_ACQUIRE))
      backoff(t0, &spins);
    if (m->mapped < sizeof(mbox_hdr) + bytes) map_mbox(m, g_rank, dest, bytes, 1);
    memcpy((char *)m->hdr + sizeof(mbox_hdr), sendbuf, bytes);
    m->hdr->size = (int64_t)bytes;
    __atomic_add_fetch(&m->hdr->seq_written, 1, __ATOMIC_RELEASE);
  }
  if (source >= 0) {
    size_t bytes = (size_t)recvcount * type_size(recvtype);
    mbox_map *m = &g_recv[source];
    if (!m->hdr) map_mbox(m, source, g_rank, 0, 0);
    double t0 = now_s();
    long spins = 0;
    while (__atomic_load_n(&m->hdr->seq_written, __ATOMIC_ACQUIRE) ==
           __atomic_load_n(&m->hdr->seq_read, __ATOMIC_ACQUIRE))
      backoff(t0, &spins);
    size_t got = (size_t)m->hdr->size;
    if (got > bytes) got = bytes;
    if (m->mapped < sizeof(mbox_hdr) + got) map_mbox(m, source, g_rank, got, 0);
    memcpy(recvbuf, (char *)m->hdr + sizeof(mbox_hdr), got);
    __atomic_add_fetch(&m->hdr->seq_read, 1, __ATOMIC_RELEASE);
  }
  return 0;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm) {
  (void)comm;
  if (count > SHIM_MAX_REDUCE) shim_die(95, "allreduce count too large");
  double v[SHIM_MAX_REDUCE];
  for (int i = 0; i < count; ++i)
    v[i] = type == MPI_FLOAT ? ((const float *)sendbuf)[i]
         : type == MPI_INT   ? ((const int *)sendbuf)[i]
                             : ((const double *)sendbuf)[i];
  if (g_size > 1) {
    MPI_Barrier(comm);
    for (int i = 0; i < count; ++i) g_ctl->reduce[g_rank][i] = v[i];
    MPI_Barrier(comm);
    for (int i = 0; i < count; ++i) {
      double acc = g_ctl->reduce[0][i];
      for (int r = 1; r < g_size; ++r) {
        double x = g_ctl->reduce[r][i];
        acc = op == MPI_MIN ? (x < acc ? x : acc) : op == MPI_MAX ? (x > acc ? x : acc) : acc + x;
      }
      v[i] = acc;
    }
    MPI_Barrier(comm);
  }
  for (int i = 0; i < count; ++i) {
    if (type == MPI_FLOAT) ((float *)recvbuf)[i] = (float)v[i];
    else if (type == MPI_INT) ((int *)recvbuf)[i] = (int)v[i];
    else ((double *)recvbuf)[i] = v[i];
  }
  return 0;
}

int MPI_Get_processor_name(char *name, int *len) {
  gethostname(name, MPI_MAX_PROCESSOR_NAME);
  *len = (int)strlen(name);
  return 0;
}
