// cgfdm_stage_noalloc: one fused RK stage on caller-owned device buffers
// that allocates no device memory.
//
// The handle API allocates its buffers, the streaming kernel's error flag and
// work-queue counter, and the PML profile table with cudaMalloc.  Some hosts
// cannot do that while they run: a serving process that carves all of HBM
// into fixed pools at start-up, or a runtime whose own allocator owns every
// byte of device memory and forbids outside cudaMalloc/cudaFree calls.  They
// pass their own wavefield, coefficient and auxiliary buffers here instead;
// the few bytes of scratch the kernels need live in one file-scope device
// array of fixed size, which every GPU that loads the library holds until the
// process exits.
//
// Scratch (kScratchBytes = 64 KiB per device, shared by every call on it and
// keeping the last call's contents):
//   [0, 4)     error flag.  Zero when the module loads; a kernel sets it when a
//              bounded wait expires; only a call with wait != 0 reads it back
//              and clears it.
//   [4, 8)     work-queue counter of the streaming kernel.  It must be zero
//              when the kernel starts; every call zeroes it (cudaMemsetAsync on
//              the caller's stream) before every launch.
//   [256, ...) PML profiles alpha, beta, d for x, y, z (3 x (_nx_+_ny_+_nz_)
//              floats), rewritten by every call before its launches.  The
//              values travel in the parameters of small fill kernels on the
//              caller's stream (no host-to-device copy from pageable memory,
//              which could block the host), so a call only enqueues work.
// A grid whose profile table does not fit (nx + ny + nz + 18 > 5440) is
// rejected with CGFDM_ERR_ARG.  Because all calls on a device share the
// scratch, calls whose work overlaps on the GPU (different streams or host
// threads) race.  The first call on a device resolves the scratch address
// with cudaGetSymbolAddress (the array's name in host code is only a host
// stand-in, never a device address); make that first call before any stream
// capture.  Each streaming-kernel variant has its shared-memory attribute set
// on its first launch in the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cgfdm_b200.h"
#include "engine.h"
#include "kernels.h"

namespace cgfdm {
namespace {

constexpr int kScratchBytes = 64 * 1024;
constexpr int kProfileOffset = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
unsigned char *g_addr[kMaxDevices] = {};

// Device address of the scratch on device `dev`, which must be current;
// resolved once per device.
cudaError_t scratch_of(int dev, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    unsigned char *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

// Fill kernel for the profile table: its values arrive in the kernel's
// parameter space (at most 32 KB), copied by the launch itself.
constexpr int kFillChunk = 7936;
struct FillChunk {
  int n;
  float v[kFillChunk];
};
__global__ void fill_profile_kernel(float *dst, const __grid_constant__ FillChunk c) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < c.n; q += gridDim.x * blockDim.x)
    dst[q] = c.v[q];
}

cudaError_t upload_profiles(float *dst, const std::vector<float> &prof, cudaStream_t st) {
  static thread_local FillChunk c;
  for (size_t q0 = 0; q0 < prof.size(); q0 += kFillChunk) {
    c.n = (int)std::min<size_t>(kFillChunk, prof.size() - q0);
    std::memcpy(c.v, prof.data() + q0, sizeof(float) * c.n);
    fill_profile_kernel<<<(c.n + 255) / 256, 256, 0, st>>>(dst + q0, c);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

#define NA_TRY(x)                                                                 \
  do {                                                                            \
    cudaError_t e_ = (x);                                                         \
    if (e_ != cudaSuccess) return fail(CGFDM_ERR_CUDA, std::string(#x) + ": " +   \
                                       cudaGetErrorString(e_));                   \
  } while (0)

template <typename S>
int stage_noalloc(const cgfdm_stage_buffers &b, cudaStream_t st, unsigned char *scratch) {
  const Layout L = make_layout(b.nx, b.ny, b.nz, (int)sizeof(S));
  StageArgs<S> a{};
  a.win = (const S *)b.w_in;
  a.wout = (S *)b.w_out;
  a.wm = (const S *)b.w_m;
  a.t = (S *)b.t;
  a.cjm = (const S *)b.cjm;
  a.rdz = b.rdz;
  a.pml = (const float *)(scratch + kProfileOffset);
  a.L = L;
  a.npml = b.npml;
  a.rDH = (float)(1.0 / b.dh);
  a.DT = b.dt;
  a.fb1 = b.fb1; a.fb2 = b.fb2; a.fb3 = b.fb3;
  a.irk = b.irk;
  // PML slabs x1 y1 z1 x2 y2 (no top z slab), each field-major [9][pos] with
  // pos x-fastest inside the slab, concatenated in that order
  a.nslab = b.npml > 0 ? 5 : 0;
  long long off = 0, big = 0;  // big: the largest slab's 9 x points
  for (int s = 0; s < a.nslab; ++s) {
    const int ax = s % 3, far = s >= 3;
    int n[3] = {b.nx, b.ny, b.nz}, o[3] = {HALO, HALO, HALO};
    o[ax] = HALO + far * (n[ax] - b.npml);
    n[ax] = b.npml;
    SlabDev<float> &sl = a.slab[s];
    sl.n0 = n[0]; sl.n1 = n[1]; sl.n2 = n[2];
    sl.off0 = o[0]; sl.off1 = o[1]; sl.off2 = o[2];
    sl.np = (long long)n[0] * n[1] * n[2];
    sl.axis = ax;
    sl.ain = b.aux_in + off;
    sl.aout = b.aux_out + off;
    sl.am = b.aux_m + off;
    sl.at = b.aux_t + off;
    off += 9LL * n[0] * n[1] * n[2];
    big = std::max(big, 9LL * n[0] * n[1] * n[2]);
  }
  // the profile table is rewritten by every call, through kernel parameters
  NA_TRY(upload_profiles((float *)(scratch + kProfileOffset),
                         pml_profiles(b.nx, b.ny, b.nz, b.npml, b.dh), st));
  int *err = (int *)scratch, *counter = (int *)(scratch + 4);
  // as a handle does: the exact-order kernel alone when opposite PML slabs
  // overlap (nPML above half the grid) or a slab is too large for the
  // streaming kernel's 32-bit auxiliary offsets
  const bool overlap = b.npml > 0 && (2 * b.npml > b.nx || 2 * b.npml > b.ny || big >= (1LL << 32));
  const int ksurf = overlap ? HALO : L.nz_ - HALO - 3;
  if (ksurf > HALO) {  // the streaming launch has planes: it needs the tensor maps
    alignas(64) unsigned char maps[kStreamMapsBytes];
    int rc = encode_stream_maps<S>(a.win, a.cjm, a.wm, a.t, L, maps);
    if (rc) return rc;
    StageArgs<S> lower = a;
    lower.kbeg = HALO;
    lower.kend = ksurf;
    NA_TRY(launch_stage_stream<S>(lower, maps, err, counter, st));
  }
  a.kbeg = ksurf;
  a.kend = L.nz_ - HALO;
  if (overlap)
    NA_TRY(launch_stage_exact<S>(a, st));
  else  // the free-surface layers as a handle runs them
    NA_TRY(launch_stage_top<S>(a, st));
  return CGFDM_OK;
}

}  // namespace
}  // namespace cgfdm

extern "C" int cgfdm_stage_noalloc(const cgfdm_stage_buffers *b, void *stream, int32_t wait) {
  using namespace cgfdm;
  if (!b) return fail(CGFDM_ERR_ARG, "null buffer descriptor");
  if (b->nx <= 0 || b->ny <= 0 || b->nz < 4 || !(b->dh > 0) || !(b->dt > 0))
    return fail(CGFDM_ERR_ARG, "invalid grid: nx, ny >= 1, nz >= 4, dh and dt > 0");
  if (b->npml < 0 || b->npml == 1 || b->npml > b->nx || b->npml > b->ny || b->npml > b->nz)
    return fail(CGFDM_ERR_PML, "nPML must be 0 or 2..min(nx, ny, nz)");
  if (b->irk < 0 || b->irk > 3 || (b->fb1 != 1 && b->fb1 != -1) ||
      (b->fb2 != 1 && b->fb2 != -1) || (b->fb3 != 1 && b->fb3 != -1))
    return fail(CGFDM_ERR_ARG, "irk must be 0..3 and fb1..fb3 must be +1 or -1");
  if (b->precision != CGFDM_FP32 && b->precision != CGFDM_FP16 && b->precision != CGFDM_BF16)
    return fail(CGFDM_ERR_ARG, "the no-allocation stage supports FP32, FP16 and BF16");
  if (!b->w_in || !b->w_out || !b->w_m || !b->t || !b->cjm || !b->rdz)
    return fail(CGFDM_ERR_ARG, "a wavefield, coefficient or rDZ pointer is null");
  if (b->npml > 0 && (!b->aux_in || !b->aux_out || !b->aux_m || !b->aux_t))
    return fail(CGFDM_ERR_ARG, "nPML > 0 needs the four auxiliary buffers");
  {
    const void *ptrs[] = {b->w_in, b->w_out, b->w_m, b->t, b->cjm, b->rdz,
                          b->aux_in, b->aux_out, b->aux_m, b->aux_t};
    const char *names[] = {"w_in", "w_out", "w_m", "t", "cjm", "rdz",
                           "aux_in", "aux_out", "aux_m", "aux_t"};
    for (int q = 0; q < 10; ++q)
      if (ptrs[q] && ((uintptr_t)ptrs[q] & 255u))
        return fail(CGFDM_ERR_ARG, std::string(names[q]) +
                                       " is not 256-byte aligned (the streaming kernel's tensor "
                                       "maps and aligned rows need cudaMalloc alignment)");
  }
  const long long need =
      kProfileOffset + 3LL * sizeof(float) * ((b->nx + 6LL) + (b->ny + 6LL) + (b->nz + 6LL));
  if (need > kScratchBytes)
    return fail(CGFDM_ERR_ARG, "grid too large for the no-allocation scratch: the PML profile "
                               "table needs " + std::to_string(need) + " bytes, the scratch holds " +
                               std::to_string(kScratchBytes) + " (nx + ny + nz + 18 <= 5440)");
  int dev = 0;
  NA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(CGFDM_ERR_ARG, "device index out of range");
  unsigned char *scratch = nullptr;
  NA_TRY(scratch_of(dev, &scratch));
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  switch (b->precision) {
    case CGFDM_FP32: rc = stage_noalloc<float>(*b, st, scratch); break;
    case CGFDM_FP16: rc = stage_noalloc<__half>(*b, st, scratch); break;
    default: rc = stage_noalloc<__nv_bfloat16>(*b, st, scratch); break;
  }
  if (rc || !wait) return rc;
  int flag = 0;
  NA_TRY(cudaStreamSynchronize(st));
  NA_TRY(cudaMemcpy(&flag, scratch, sizeof flag, cudaMemcpyDeviceToHost));
  if (flag) {
    NA_TRY(cudaMemset(scratch, 0, sizeof flag));
    return fail(CGFDM_ERR_TIMEOUT, "a bounded device-side wait of the streaming kernel expired");
  }
  return CGFDM_OK;
}
