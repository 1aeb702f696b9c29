/*
 * cgfdm_b200 -- B200-native (sm_100a) time-stepping hot path of CGFDM.
 *
 * C ABI: plain C types, host pointers and sizes only; every function returns a
 * status code (CGFDM_OK = 0) instead of aborting.  A handle owns all device
 * memory of one simulation; distinct handles may be driven from distinct host
 * threads.  All array arguments are HOST memory unless stated otherwise.
 *
 * The reference entry point this library replaces is
 *   void propagate(MPI_Comm, MPI_COORD, MPI_NEIGHBOR, GRID, PARAMS, WAVE,
 *                  Mat_rDZ, FLOAT *CJM, SOURCE_FILE_INPUT, long long *srcIndex,
 *                  float *momentRate, float *momentRateSlice, SLICE,
 *                  SLICE_DATA, SLICE_DATA)
 *   (src-new-FP32-SVE/functions.h:133-138, propagate.cpp:24-228), called once
 *   from run() (run.cpp:100-104) on every MPI rank.  This library is the
 *   single-rank drop-in: no halo exchange, the whole grid on one GPU.
 *
 * Array layouts are the reference's (XFAST, HALO = 3, padded dims
 * _nx_ = nx + 6, _ny_ = ny + 6, _nz_ = nz + 6, num = _nx_*_ny_*_nz_):
 *   cjm        13 x num float, fields xi_x xi_y xi_z et_x et_y et_z zt_x zt_y
 *              zt_z J mu lambda buoyancy (CJM.cpp:117-131), mu/lambda/b already
 *              converted (CJM.cpp:47-73)
 *   rdz        2 x (_nx_*_ny_) x 9 float, _rDZ_DX then _rDZ_DY
 *              (contravariant.cpp:179-198, 329-351)
 *   wavefield  9 x num float: Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz
 *   stations   int32 [nsta][3] padded-grid indices (station.cpp:288-290);
 *              output float [nsta][nt][9] (station.cpp:333-343)
 *   pgv        float [ny][nx][2]: PGVh, PGV (PGV.cpp:80-99)
 */
#ifndef CGFDM_B200_H
#define CGFDM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference's MPI_Abort codes where one exists) ---- */
#define CGFDM_OK 0
#define CGFDM_ERR_ARG 1            /* invalid argument / size */
#define CGFDM_ERR_PARAMS 100       /* params.json missing/unparsable (getParams.cpp:23,46) */
#define CGFDM_ERR_CFL 110          /* DT above the CFL limit (calc_CFL.cpp:341-344) */
#define CGFDM_ERR_PML 130          /* nPML larger than the grid (pml_deriv.cpp:53-59) */
#define CGFDM_ERR_NO_SOURCE 180    /* no source configured (modelChecking.cpp:37) */
#define CGFDM_ERR_SOURCE 181       /* source outside the grid / unreadable source file */
#define CGFDM_ERR_IO 200           /* file could not be read or written */
#define CGFDM_ERR_CUDA 300         /* a CUDA runtime call failed */
#define CGFDM_ERR_NOMEM 301        /* device memory budget exceeded at admission */
#define CGFDM_ERR_NO_KERNEL 302    /* CUDA extension unusable (no device / wrong arch) */
#define CGFDM_ERR_TIMEOUT 303      /* a bounded device-side wait expired */
#define CGFDM_ERR_STATE 304        /* call not valid in the handle's current state */
#define CGFDM_ERR_CANCELLED 305    /* the server request was cancelled */

/* ---- storage precision of wavefield and coefficients ---- */
#define CGFDM_FP32 0   /* float everywhere: the reference's FP32 build */
#define CGFDM_FP16 1   /* scaled half storage, FP32 arithmetic (macro.h:65-73) */
#define CGFDM_BF16 2   /* scaled bfloat16 storage, FP32 arithmetic */
#define CGFDM_FP64 3   /* double everywhere: the accuracy oracle run */

/* ---- kernel selection ---- */
#define CGFDM_KERNEL_AUTO 0      /* fastest kernel for the precision */
#define CGFDM_KERNEL_EXACT 1     /* reference operation order, no FMA contraction:
                                    bit-identical to the reference's FP32 CPU path */
#define CGFDM_KERNEL_STREAM 2    /* TMA-staged z-streaming fused stage kernel (grids
                                    whose opposite PML slabs overlap, nPML above half
                                    of nx or ny, run the exact-order kernel) */

typedef struct {
  int32_t nx, ny, nz;     /* interior points (params NX, NY, NZ) */
  int32_t npml;           /* PML thickness (params nPML); 0 disables the PML */
  float dh;               /* grid spacing DH (m) */
  float dt;               /* time step DT (s) */
  int32_t nt;             /* number of steps NT = (int)(TMAX/DT) */
  int32_t precision;      /* CGFDM_FP32 ... */
  int32_t kernel;         /* CGFDM_KERNEL_* */
  int32_t device;         /* CUDA device ordinal */
} cgfdm_desc;

typedef struct cgfdm_handle cgfdm_handle;

/* Version / build identification; returns a static string. */
const char *cgfdm_version(void);

/* Text of the last error raised on the calling host thread. */
const char *cgfdm_last_error(void);

/* Device bytes a handle with this descriptor will hold (wavefield, RK
 * buffers, coefficients, PML slabs), used for admission control. */
int cgfdm_device_bytes(const cgfdm_desc *desc, int64_t *bytes);

/* Creates a handle and allocates its device memory; the wavefield starts at
 * rest (allocWave/allocPML zero-fill, wave_deriv.cpp:42, pml_deriv.cpp:26).
 * Replaces the allocation half of propagate.cpp:65-92. */
int cgfdm_create(const cgfdm_desc *desc, cgfdm_handle **out);
int cgfdm_destroy(cgfdm_handle *h);

/* Uploads the medium/metric coefficients and free-surface matrices in the
 * reference layout (the CJM and mat_rDZ arguments of propagate()).  Waits for
 * the handle's outstanding work first and returns once the upload is done;
 * the RK accumulator is cleared (a stage 0 rewrites it before any read). */
int cgfdm_set_model(cgfdm_handle *h, const float *cjm, const float *rdz);

/* The smoothed explosive point source of singleSource.cpp:78-177 at padded
 * indices (sx, sy, sz) with Ricker centre frequency rickerfc. */
int cgfdm_set_point_source(cgfdm_handle *h, int32_t sx, int32_t sy, int32_t sz,
                           float rickerfc);

/* The finite-fault source of addMoment.cpp:222-339: npts cell indices
 * (padded linear, the srcIndex argument of propagate()) and the moment-rate
 * table momentRate [nt][npts][6] sampled at dt.  If `scaled` is 0 the
 * table is scaled here by mu*Cv/(J*DH^3) (calculate_MomentRate,
 * addMoment.cpp:12-65); pass 1 if it already is. */
int cgfdm_set_fault_source(cgfdm_handle *h, const int64_t *src_index, const float *moment_rate,
                           int64_t npts, int32_t nt, float dt, int32_t scaled);

/* Station list (padded indices); seismograms are recorded every step. */
int cgfdm_set_stations(cgfdm_handle *h, const int32_t *xyz, int32_t nsta);

/* Advances nsteps time steps (sources, 4 RK stages, stations, PGV) on the
 * CUDA stream `stream` (a cudaStream_t, NULL = the handle's own stream).
 * Asynchronous: returns once the work is enqueued. */
int cgfdm_run(cgfdm_handle *h, int32_t nsteps, void *stream);

/* One RK stage irk (0..3) with MacCormack signs fb1..fb3 and no source,
 * station or PGV work: the unit of the stage-level parity tests.  Stages 1-3
 * read the RK accumulator that stage 0 (or cgfdm_set_state) left; a
 * cgfdm_set_model call in between clears it (see cgfdm_set_state). */
int cgfdm_stage(cgfdm_handle *h, int32_t irk, int32_t fb1, int32_t fb2, int32_t fb3,
                void *stream);

/* Waits for all work of the handle. */
int cgfdm_synchronize(cgfdm_handle *h);

/* Completed steps so far. */
int cgfdm_steps_done(cgfdm_handle *h, int32_t *it);

/* Host copies of results (blocking). */
int cgfdm_get_stations(cgfdm_handle *h, float *wave);          /* [nsta][nt][9] */
int cgfdm_get_pgv(cgfdm_handle *h, float *pgv);                /* [ny][nx][2]   */
int cgfdm_get_wavefield(cgfdm_handle *h, float *w);            /* 9 x num       */
/* Free-surface velocity snapshot (Vx, Vy, Vz on the top interior layer,
 * data_io.cpp:481-491): float [3][ny][nx]. */
int cgfdm_get_free_surface(cgfdm_handle *h, float *v3);

/* Stage-test state access: the input W of stage irk, the RK accumulator t
 * and (for irk 1..3) the step-start state m, each 9 x num; PML auxiliaries as
 * 5 slabs (x1 y1 z1 x2 y2) x {Aux, t, m}, each [npos][9]
 * (pml_deriv.cpp:12-32).  get_state returns the last stage's output W, t and
 * m (m is the stage input for irk 0, as the reference's m_W copy).
 * Ordering: cgfdm_set_model stages its upload through the RK accumulator and
 * clears it afterwards, so call it before cgfdm_set_state -- a t set for a
 * stage irk > 0 and followed by cgfdm_set_model is lost. */
int cgfdm_set_state(cgfdm_handle *h, int32_t irk, const float *W, const float *t,
                    const float *m, const float *aux);
int cgfdm_get_state(cgfdm_handle *h, float *W, float *t, float *m, float *aux);
int cgfdm_aux_floats(cgfdm_handle *h, int64_t *n);   /* floats of one aux set */

/* Device timing of the last cgfdm_run, from CUDA events on its stream (only
 * when enabled with cgfdm_set_timing): [0] the whole run in ms, [1] the sum
 * of the fused-stage kernel durations in ms, [2] the number of those stage
 * launches. */
int cgfdm_set_timing(cgfdm_handle *h, int32_t on);
int cgfdm_get_timing(cgfdm_handle *h, float *ms3);

/* Per-kernel view of the last cgfdm_run (device events, timing enabled):
 * [0] streaming-kernel time in ms, [1] its launches, [2] the algorithmic
 * bytes those launches move (fields read and written once per point and
 * stage; the PML auxiliaries, handled inside the same kernel, are not
 * counted), [3] kernels launched by the run (counted whether or not timing is
 * on), [4] time between the streaming kernel and the exact-order kernel in
 * ms (no kernel runs there), [5] exact-order (free-surface) kernel time in
 * ms, [6] stages timed, [7] the streaming kernel's tile height (0: not used). */
int cgfdm_get_kernel_stats(cgfdm_handle *h, double *out8);

/* Tile form of the streaming kernel: 16 (32 x 16 tiles, one CTA per SM),
 * 8 (32 x 8 tiles, two CTAs per SM), 64 (FP16 / BF16 storage only: 64 x 8
 * interior tiles with two x-adjacent points per thread, the 32 x 8 form
 * elsewhere), or 0 (the default): autotune -- the first cgfdm_run times one
 * stage with each form on this handle's buffers (blocking that call for a
 * few stage times) and keeps the fastest; the choice is cached per
 * (precision, grid) for the process.  If the environment variable
 * CGFDM_TUNE_CACHE names a file, choices are also kept there across
 * processes: a grid with an entry for this GPU is not timed again, and new
 * choices are written back (a JSON object of [form, depth, tiled surface]
 * triples; a malformed file is ignored and rewritten).  The forms split the grid differently
 * between the interior launch and the PML launch, whose variants round the
 * elastic combination differently, so they agree to rounding. */
int cgfdm_set_tile_rows(cgfdm_handle *h, int32_t rows);

/* Depth of the streaming kernel's work items: the planes above the bottom
 * PML slab are cut into chunks of `planes` z planes per work item (0, the
 * default: about 40 items per CTA slot, at least 16 planes each).  Shorter
 * chunks keep neighbouring tiles closer in time (their halo rows meet in
 * L2) but re-read four planes per chunk. */
int cgfdm_set_chunk(cgfdm_handle *h, int32_t planes);

/* The fast path's configuration in use (after the autotuner, if it ran),
 * three values: form_chunk[0] = the streaming kernel's tile form 16, 8 or
 * 64; form_chunk[1] = planes per work item (0: automatic); form_chunk[2] = 1
 * if the free-surface layers run on the tiled kernel (the exact-order kernel
 * on the PML-slab columns), 0 if on the exact-order kernel alone.  All 0 when
 * the handle runs the exact-order kernel only. */
int cgfdm_get_tuning(cgfdm_handle *h, int32_t *form_chunk);

/* Checkpoint / resume at a step boundary (no counterpart in the reference):
 * the handle's raw device state -- step wavefield, the two other stage
 * buffers (their halo cells hold point-source values), step-start PML
 * auxiliaries, PGV map, seismograms so far and the step counter -- into a
 * host buffer of cgfdm_checkpoint_bytes bytes.  Loading it into a handle
 * created with the same descriptor, sources and stations continues the run
 * bit for bit.  The layout is this library's own (header "CGFDMCK1"). */
int cgfdm_checkpoint_bytes(cgfdm_handle *h, int64_t *bytes);
int cgfdm_checkpoint_save(cgfdm_handle *h, void *buf, int64_t bytes);
int cgfdm_checkpoint_load(cgfdm_handle *h, const void *buf, int64_t bytes);

/* Failure-detection testing (no counterpart in the reference): kind 1 makes
 * the next streaming-kernel launch of the handle leave one tile-plane load
 * unissued, so that one CTA's bounded wait expires (about 2^31 clock cycles,
 * a second); the CTA waits for its other copies, sets the error flag and
 * returns, and the next synchronizing call reports CGFDM_ERR_TIMEOUT once.
 * No memory is touched and the context stays usable; that stage's outputs
 * are not valid.  kind 0 clears a pending injection. */
#define CGFDM_FAULT_NONE 0
#define CGFDM_FAULT_DROP_LOAD 1
int cgfdm_inject_fault(cgfdm_handle *h, int32_t kind);

/* Replays each time step of cgfdm_run as a CUDA graph (on = 1) instead of
 * launching its kernels one by one; one graph per phase of the step counter
 * mod 8 (the MacCormack signs repeat with period 8), captured on the second
 * step of that phase and kept until the sources, stations, model or tile
 * height change.  Results are identical either way.  While timing is
 * enabled (cgfdm_set_timing) steps run without graphs.  The stream passed to
 * cgfdm_run must be capturable (not the legacy NULL stream: pass NULL to use
 * the handle's own stream). */
int cgfdm_set_graph(cgfdm_handle *h, int32_t on);

/* ---- batches: many independent scenarios advanced together ------------
 * No counterpart in the reference (one run per process there).  A batch
 * holds n handles of one precision on one device (uneven grid sizes, own
 * sources, stations, and step counters).  cgfdm_batch_run advances every
 * member by nsteps: per stage, the streaming part of all members runs in
 * persistent launches whose work queue spans the members (16 members per
 * launch pair; members at different phases of the MacCormack schedule are
 * grouped), and each member's free-surface layers, sources and stations run
 * as its own small kernels.  Results equal running each member alone.  With
 * cgfdm_batch_set_graph(b, 1) each batch step is replayed as a CUDA graph.
 * Members keep their own state: read their results with the handle getters
 * after cgfdm_batch_synchronize.  Destroy the batch before its members. */
typedef struct cgfdm_batch cgfdm_batch;
int cgfdm_batch_create(cgfdm_handle *const *handles, int32_t n, cgfdm_batch **out);
int cgfdm_batch_run(cgfdm_batch *b, int32_t nsteps, void *stream);
int cgfdm_batch_set_graph(cgfdm_batch *b, int32_t on);
int cgfdm_batch_synchronize(cgfdm_batch *b);
int cgfdm_batch_destroy(cgfdm_batch *b);

/* ---- serving: a request loop with continuous batching -------------------
 * No counterpart in the reference.  A server owns one device and a worker
 * thread.  cgfdm_server_submit queues a simulation (the cgfdm_propagate
 * inputs, copied) from any thread and returns at once.  The worker admits
 * queued requests in arrival order while their device footprint
 * (cgfdm_device_bytes) fits the HBM budget, keeps their wavefields resident,
 * and advances all admitted requests of one precision together as one batch
 * (cgfdm_batch) by chunk_steps steps per round -- the batches of different
 * precisions on their own streams, overlapping on the device.  A newly
 * admitted request first runs chunk_steps / 10 steps (at least one) in a
 * short round of the newcomers alone, so that its first seismogram rows come
 * back without waiting for a full round of every running request.  After each
 * round the new seismogram rows of every request are copied back
 * (cgfdm_server_read_rows reads them while the request runs), finished
 * requests release their memory, and requests that arrived meanwhile join
 * the next round.  Each request's results equal a lone run bit for bit.
 * cgfdm_server_stats: [0] p50 and [1] p99 time from submission to the first
 * streamed seismogram chunk (ms), [2] p50 and [3] p99 time to completion
 * (ms), [4] aggregate grid-point updates per second (Gpt/s) from the first
 * submission to the last completion, [5] completed requests, [6] seconds
 * the worker spent in rounds, [7] peak admitted device bytes. */
#define CGFDM_REQ_QUEUED 0
#define CGFDM_REQ_RUNNING 1
#define CGFDM_REQ_DONE 2
#define CGFDM_REQ_FAILED 3
#define CGFDM_REQ_CANCELLED 4

typedef struct {
  int64_t hbm_budget_bytes; /* admission budget; 0 = free device memory minus 4 GiB */
  int32_t chunk_steps;      /* steps per round (seismograms stream back per round); 0 = 100 */
  int32_t device;
  int32_t use_graph;        /* 1: each batch step is replayed as a CUDA graph */
} cgfdm_server_opts;

typedef struct cgfdm_server cgfdm_server;
int cgfdm_server_create(const cgfdm_server_opts *opts, cgfdm_server **out);
int cgfdm_server_submit(cgfdm_server *s, const cgfdm_desc *desc, const float *cjm,
                        const float *rdz, int32_t point_src, const int32_t *point_xyz,
                        float rickerfc, const int64_t *src_index, const float *moment_rate,
                        int64_t npts, int32_t src_nt, float src_dt, const int32_t *sta_xyz,
                        int32_t nsta, int64_t *id);
/* state (CGFDM_REQ_*) and the number of steps streamed back so far */
int cgfdm_server_poll(cgfdm_server *s, int64_t id, int32_t *state, int32_t *steps);
/* copies rows [from, upto) of every station into wave [nsta][nt][9] */
int cgfdm_server_read_rows(cgfdm_server *s, int64_t id, int32_t from, float *wave,
                           int32_t *upto);
/* blocks until the request ends; copies its seismograms [nsta][nt][9] and PGV
 * map [ny][nx][2] (either may be NULL) and latencies (ms: to the first
 * chunk, to completion), then forgets the request */
int cgfdm_server_wait(cgfdm_server *s, int64_t id, float *wave, float *pgv, double *lat_ms2);
/* cancels a request: a queued one leaves the queue at once; an admitted one
 * stops after the round it is in, and its device memory is released; wait()
 * then returns CGFDM_ERR_CANCELLED */
int cgfdm_server_cancel(cgfdm_server *s, int64_t id);
int cgfdm_server_stats(cgfdm_server *s, double *out8);
int cgfdm_server_destroy(cgfdm_server *s);

/* ---- one RK stage without any device allocation ------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * while they run -- a serving process that splits all of HBM into fixed pools
 * at start-up, or a framework whose allocator owns every byte of device
 * memory -- this runs the same stage as cgfdm_stage on a handle (streaming
 * kernel below the three free-surface layers, exact-order kernel for them)
 * on buffers the caller already owns, and allocates nothing.  Its only
 * scratch (error flag, work-queue counter, PML profile table) is a fixed
 * 64 KiB device array per device, held by every GPU that loads the library.
 *
 * Every pointer is DEVICE memory, 256-byte aligned (as cudaMalloc returns).
 * Wavefields (9 fields: Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz) and cjm (13 fields,
 * as CJM.cpp) are in the storage type, scaled as a handle of that precision
 * expects, in the library's device layout for elem_bytes = 4 (FP32) or 2
 * (FP16 / BF16): _nx_ = nx + 6, _ny_ = ny + 6, _nz_ = nz + 6,
 * xoff = 128 / elem_bytes - 3, px = roundup(_nx_ + xoff, 32),
 * plane = px * _ny_, fs = roundup(plane * _nz_, 32); field f of padded point
 * (i, j, k) at element f * fs + xoff + i + j * px + k * plane.  rdz is
 * 2 x (_nx_*_ny_) x 9 float.  The four auxiliary buffers are float, each the
 * slabs x1 y1 z1 x2 y2 concatenated, every slab field-major [9][np] (value v
 * of slab point pos at v * np + pos, pos x-fastest, np the slab's points;
 * the reference's own order is [pos][9]), as many floats as cgfdm_aux_floats
 * reports for a handle of the same grid.  Stage irk reads
 * w_in, cjm, rdz, w_m (stages 1-2), t (stages 1-3), aux_in, aux_m (stages
 * 1-2), aux_t (stages 1-3), and writes w_out, t (stages 0-2), aux_out and
 * aux_t (stages 0-2).
 *
 * Limits and rules: precision FP32, FP16 or BF16; the PML profile table must
 * fit the scratch (nx + ny + nz + 18 <= 5440, else CGFDM_ERR_ARG).  All calls
 * on one device share the scratch and see what the last call left there:
 * each call zeroes the work-queue counter itself, so calls whose work
 * overlaps on the GPU race.  The error flag starts at zero, is set by an
 * expired bounded wait, and is read and cleared only when `wait` is
 * non-zero: then the call synchronizes `stream` and returns CGFDM_ERR_TIMEOUT
 * if it was set.  With wait = 0 the call only enqueues work on `stream`
 * (current device): the profile table reaches the scratch through the
 * parameters of small fill kernels, not through a host-to-device copy.  The
 * first call on a device resolves the scratch address; make it before any
 * stream capture.  Each streaming-kernel variant has its shared-memory
 * attribute set on its first launch in the process.  A pointer that is not
 * 256-byte aligned is rejected with CGFDM_ERR_ARG.
 */
typedef struct {
  int32_t nx, ny, nz, npml;
  float dh, dt;
  int32_t precision;
  int32_t irk, fb1, fb2, fb3;
  const void *w_in;
  void *w_out;
  const void *w_m;
  void *t;
  const void *cjm;
  const float *rdz;
  const float *aux_in;
  float *aux_out;
  const float *aux_m;
  float *aux_t;
} cgfdm_stage_buffers;

int cgfdm_stage_noalloc(const cgfdm_stage_buffers *b, void *stream, int32_t wait);

/* Drop-in for propagate() with host buffers: uploads the model and sources,
 * runs all nt steps, returns station seismograms, the PGV map and the final
 * free-surface snapshot.  Any output pointer may be NULL. */
int cgfdm_propagate(const cgfdm_desc *desc, const float *cjm, const float *rdz,
                    int32_t point_src, const int32_t *point_xyz, float rickerfc,
                    const int64_t *src_index, const float *moment_rate, int64_t npts,
                    int32_t src_nt, float src_dt, const int32_t *sta_xyz, int32_t nsta,
                    float *sta_out, float *pgv_out, float *freesurf_out);

/* The reference program end to end (main.cpp -> run.cpp -> propagate.cpp) on
 * one GPU: reads params.json / station.json / model files from run_dir,
 * performs the setup on the host, runs the hot path here, and writes the
 * reference's output files under params "out" (station_mpi_0_0_0.bin,
 * PGV_Z_mpi_0_0_0.bin, V*_/FreeSurfV*_ slices, coord/medium slices). */
int cgfdm_run_directory(const char *run_dir, int32_t precision, int32_t kernel,
                        int32_t device);

/* Host setup only (run.cpp:56-131 + propagate.cpp:65-128): builds the arrays
 * the hot path consumes from the files in run_dir.  Buffers are allocated by
 * the library and released with cgfdm_free_setup. */
typedef struct {
  cgfdm_desc desc;
  float *cjm;             /* 13 x num */
  float *rdz;             /* 2 x nsurf x 9 */
  float *coord;           /* num x 3 (AoS, coord.cpp:137-139) */
  float *medium;          /* num x 3 Vs Vp rho, before conversion */
  float *pml;             /* alpha/beta/d x/y/z block (init_pml_para.cpp:21-51) */
  int32_t point_src;      /* 1 if the single smoothed source is active */
  int32_t point_xyz[3];
  float rickerfc;
  int64_t npts;           /* finite-fault cells after merging duplicates */
  int32_t src_nt;
  float src_dt;
  int64_t *src_index;     /* [npts] */
  float *moment_rate;     /* [src_nt][npts][6], scaled */
  int32_t nsta;
  int32_t *sta_xyz;       /* [nsta][3] padded */
  void *owner;            /* library-owned storage behind the arrays */
  float *terrain;         /* [_ny_][_nx_] surface height before the stretch (m) */
} cgfdm_setup;

/* FP32 storage constants (cgfdm_setup_from_directory_ex with CGFDM_FP32). */
int cgfdm_setup_from_directory(const char *run_dir, cgfdm_setup *out);
/* precision selects the storage scaling of cjm and the moment rates: for
 * CGFDM_FP16 / CGFDM_BF16 the reference's FP16 constants Cv, Cs, Crho
 * (macro.h:65-73), the form a handle of that precision expects. */
int cgfdm_setup_from_directory_ex(const char *run_dir, int32_t precision, cgfdm_setup *out);
int cgfdm_free_setup(cgfdm_setup *s);

#ifdef __cplusplus
}
#endif
#endif
