/*
 * Test infrastructure (oracle harness), not product code.
 *
 * A minimal MPI interface sufficient to compile the reference CGFDM sources
 * (src-new-FP32-SVE/*.cpp) without an MPI installation.  It covers exactly
 * the calls the reference makes (init_MPI.cpp:21-64, MPI_send_recv*.cpp,
 * calc_CFL.cpp:317-327, propagate.cpp:135-211, addMoment.cpp:229).
 *
 * The implementation (mpi_shim.c) runs either one rank, or N ranks as forked
 * processes that exchange halos through POSIX shared memory, so that the
 * reference's own domain decomposition can be timed on all host cores.
 */
#ifndef CGFDM_ORACLE_MPI_SHIM_H
#define CGFDM_ORACLE_MPI_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-1)
#define MPI_CHAR 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_INT 4
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart);
int MPI_Cart_shift(MPI_Comm comm, int dir, int disp, int *src, int *dst);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                 int sendtag, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Get_processor_name(char *name, int *len);

#ifdef __cplusplus
}
#endif
#endif
