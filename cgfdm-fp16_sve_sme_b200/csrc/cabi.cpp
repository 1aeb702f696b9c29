// extern "C" boundary (include/cgfdm_b200.h).
#include <sys/stat.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/cgfdm_b200.h"
#include "engine.h"
#include "setup.h"

struct cgfdm_handle {
  std::unique_ptr<cgfdm::Engine> eng;
};

struct cgfdm_batch {
  std::unique_ptr<cgfdm::BatchBase> b;
};

using cgfdm::set_error;

namespace {

int check(cgfdm_handle *h) {
  if (!h || !h->eng) {
    set_error("null handle");
    return CGFDM_ERR_ARG;
  }
  return CGFDM_OK;
}

template <class F> int guarded(F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    set_error("host memory exhausted");
    return CGFDM_ERR_NOMEM;
  } catch (const std::exception &e) {
    set_error(e.what());
    return CGFDM_ERR_ARG;
  }
}

#define H_OR_FAIL(h)          \
  do {                        \
    int rc_ = check(h);       \
    if (rc_) return rc_;      \
  } while (0)

}  // namespace

extern "C" {

const char *cgfdm_version(void) { return "cgfdm_b200 0.1 (sm_100a)"; }

const char *cgfdm_last_error(void) { return cgfdm::last_error(); }

int cgfdm_device_bytes(const cgfdm_desc *d, int64_t *bytes) {
  if (!d || !bytes) return CGFDM_ERR_ARG;
  *bytes = cgfdm::engine_device_bytes(*d);
  return CGFDM_OK;
}

int cgfdm_create(const cgfdm_desc *desc, cgfdm_handle **out) {
  if (!desc || !out) return CGFDM_ERR_ARG;
  return guarded([&] {
    auto *h = new cgfdm_handle();
    int rc = cgfdm::make_engine(*desc, h->eng);
    if (rc) {
      delete h;
      *out = nullptr;
      return rc;
    }
    *out = h;
    return CGFDM_OK;
  });
}

int cgfdm_destroy(cgfdm_handle *h) {
  delete h;
  return CGFDM_OK;
}

int cgfdm_set_model(cgfdm_handle *h, const float *cjm, const float *rdz) {
  H_OR_FAIL(h);
  if (!cjm || !rdz) return CGFDM_ERR_ARG;
  return guarded([&] { return h->eng->set_model(cjm, rdz); });
}

int cgfdm_set_point_source(cgfdm_handle *h, int32_t sx, int32_t sy, int32_t sz, float rickerfc) {
  H_OR_FAIL(h);
  return h->eng->set_point_source(sx, sy, sz, rickerfc);
}

int cgfdm_set_fault_source(cgfdm_handle *h, const int64_t *idx, const float *rate, int64_t npts,
                           int32_t nt, float dt, int32_t scaled) {
  H_OR_FAIL(h);
  if (npts > 0 && (!idx || !rate || nt < 2 || !(dt > 0))) return CGFDM_ERR_ARG;
  return guarded([&] { return h->eng->set_fault_source(idx, rate, npts, nt, dt, scaled != 0); });
}

int cgfdm_set_stations(cgfdm_handle *h, const int32_t *xyz, int32_t nsta) {
  H_OR_FAIL(h);
  if (nsta > 0 && !xyz) return CGFDM_ERR_ARG;
  return guarded([&] { return h->eng->set_stations(xyz, nsta); });
}

int cgfdm_run(cgfdm_handle *h, int32_t nsteps, void *stream) {
  H_OR_FAIL(h);
  if (nsteps < 0) return CGFDM_ERR_ARG;
  return h->eng->run(nsteps, stream);
}

int cgfdm_stage(cgfdm_handle *h, int32_t irk, int32_t fb1, int32_t fb2, int32_t fb3, void *stream) {
  H_OR_FAIL(h);
  auto okfb = [](int f) { return f == 1 || f == -1; };
  if (irk < 0 || irk > 3 || !okfb(fb1) || !okfb(fb2) || !okfb(fb3)) return CGFDM_ERR_ARG;
  return h->eng->stage(irk, fb1, fb2, fb3, stream);
}

int cgfdm_synchronize(cgfdm_handle *h) {
  H_OR_FAIL(h);
  return h->eng->synchronize();
}

int cgfdm_steps_done(cgfdm_handle *h, int32_t *it) {
  H_OR_FAIL(h);
  if (!it) return CGFDM_ERR_ARG;
  *it = h->eng->steps_done();
  return CGFDM_OK;
}

int cgfdm_get_stations(cgfdm_handle *h, float *wave) {
  H_OR_FAIL(h);
  if (!wave) return CGFDM_ERR_ARG;
  return h->eng->get_stations(wave);
}

int cgfdm_get_pgv(cgfdm_handle *h, float *pgv) {
  H_OR_FAIL(h);
  if (!pgv) return CGFDM_ERR_ARG;
  return h->eng->get_pgv(pgv);
}

int cgfdm_get_wavefield(cgfdm_handle *h, float *w) {
  H_OR_FAIL(h);
  if (!w) return CGFDM_ERR_ARG;
  return guarded([&] { return h->eng->get_wavefield(w); });
}

int cgfdm_get_free_surface(cgfdm_handle *h, float *v3) {
  H_OR_FAIL(h);
  if (!v3) return CGFDM_ERR_ARG;
  return h->eng->get_free_surface(v3);
}

int cgfdm_set_state(cgfdm_handle *h, int32_t irk, const float *W, const float *t, const float *m,
                    const float *aux) {
  H_OR_FAIL(h);
  return guarded([&] { return h->eng->set_state(irk, W, t, m, aux); });
}

int cgfdm_get_state(cgfdm_handle *h, float *W, float *t, float *m, float *aux) {
  H_OR_FAIL(h);
  return guarded([&] { return h->eng->get_state(W, t, m, aux); });
}

int cgfdm_aux_floats(cgfdm_handle *h, int64_t *n) {
  H_OR_FAIL(h);
  if (!n) return CGFDM_ERR_ARG;
  *n = h->eng->aux_floats();
  return CGFDM_OK;
}

int cgfdm_set_timing(cgfdm_handle *h, int32_t on) {
  H_OR_FAIL(h);
  return h->eng->set_timing(on != 0);
}

int cgfdm_get_timing(cgfdm_handle *h, float *ms3) {
  H_OR_FAIL(h);
  if (!ms3) return CGFDM_ERR_ARG;
  return h->eng->get_timing(ms3);
}

int cgfdm_checkpoint_bytes(cgfdm_handle *h, int64_t *bytes) {
  H_OR_FAIL(h);
  if (!bytes) return CGFDM_ERR_ARG;
  *bytes = h->eng->checkpoint_bytes();
  return CGFDM_OK;
}

int cgfdm_checkpoint_save(cgfdm_handle *h, void *buf, int64_t bytes) {
  H_OR_FAIL(h);
  if (!buf) return CGFDM_ERR_ARG;
  return h->eng->checkpoint_save(buf, bytes);
}

int cgfdm_checkpoint_load(cgfdm_handle *h, const void *buf, int64_t bytes) {
  H_OR_FAIL(h);
  if (!buf) return CGFDM_ERR_ARG;
  return h->eng->checkpoint_load(buf, bytes);
}

int cgfdm_inject_fault(cgfdm_handle *h, int32_t kind) {
  H_OR_FAIL(h);
  return h->eng->inject_fault(kind);
}

int cgfdm_set_graph(cgfdm_handle *h, int32_t on) {
  H_OR_FAIL(h);
  return h->eng->set_graph(on != 0);
}

int cgfdm_batch_create(cgfdm_handle *const *hs, int32_t n, cgfdm_batch **out) {
  if (!hs || n <= 0 || !out) return CGFDM_ERR_ARG;
  *out = nullptr;
  return guarded([&] {
    std::vector<cgfdm::Engine *> e;
    for (int q = 0; q < n; ++q) {
      int rc = check(hs[q]);
      if (rc) return rc;
      e.push_back(hs[q]->eng.get());
    }
    auto *b = new cgfdm_batch();
    int rc = cgfdm::make_batch(e.data(), n, b->b);
    if (rc) {
      delete b;
      return rc;
    }
    *out = b;
    return CGFDM_OK;
  });
}

int cgfdm_batch_run(cgfdm_batch *b, int32_t nsteps, void *stream) {
  if (!b || !b->b || nsteps < 0) return CGFDM_ERR_ARG;
  return b->b->run(nsteps, stream);
}

int cgfdm_batch_set_graph(cgfdm_batch *b, int32_t on) {
  if (!b || !b->b) return CGFDM_ERR_ARG;
  return b->b->set_graph(on != 0);
}

int cgfdm_batch_synchronize(cgfdm_batch *b) {
  if (!b || !b->b) return CGFDM_ERR_ARG;
  return b->b->synchronize();
}

int cgfdm_batch_destroy(cgfdm_batch *b) {
  delete b;
  return CGFDM_OK;
}

int cgfdm_set_chunk(cgfdm_handle *h, int32_t planes) {
  H_OR_FAIL(h);
  return h->eng->set_chunk(planes);
}

int cgfdm_set_tile_rows(cgfdm_handle *h, int32_t rows) {
  H_OR_FAIL(h);
  return h->eng->set_tile_rows(rows);
}

int cgfdm_get_tuning(cgfdm_handle *h, int32_t *form_chunk) {
  H_OR_FAIL(h);
  if (!form_chunk) {
    set_error("null output");
    return CGFDM_ERR_ARG;
  }
  return h->eng->get_tuning(form_chunk);
}

int cgfdm_get_kernel_stats(cgfdm_handle *h, double *out8) {
  H_OR_FAIL(h);
  if (!out8) return CGFDM_ERR_ARG;
  return h->eng->get_kernel_stats(out8);
}

int cgfdm_propagate(const cgfdm_desc *desc, const float *cjm, const float *rdz, int32_t point_src,
                    const int32_t *point_xyz, float rickerfc, const int64_t *src_index,
                    const float *moment_rate, int64_t npts, int32_t src_nt, float src_dt,
                    const int32_t *sta_xyz, int32_t nsta, float *sta_out, float *pgv_out,
                    float *freesurf_out) {
  if (!desc || !cjm || !rdz) return CGFDM_ERR_ARG;
  cgfdm_handle *h = nullptr;
  int rc = cgfdm_create(desc, &h);
  if (rc) return rc;
  std::unique_ptr<cgfdm_handle> guard(h);
  if ((rc = cgfdm_set_model(h, cjm, rdz))) return rc;
  if (point_src && point_xyz &&
      (rc = cgfdm_set_point_source(h, point_xyz[0], point_xyz[1], point_xyz[2], rickerfc)))
    return rc;
  if (npts > 0 && (rc = cgfdm_set_fault_source(h, src_index, moment_rate, npts, src_nt, src_dt, 1)))
    return rc;
  if (nsta > 0 && (rc = cgfdm_set_stations(h, sta_xyz, nsta))) return rc;
  if ((rc = cgfdm_run(h, desc->nt, nullptr))) return rc;
  if ((rc = cgfdm_synchronize(h))) return rc;
  if (sta_out && nsta > 0 && (rc = cgfdm_get_stations(h, sta_out))) return rc;
  if (pgv_out && (rc = cgfdm_get_pgv(h, pgv_out))) return rc;
  if (freesurf_out && (rc = cgfdm_get_free_surface(h, freesurf_out))) return rc;
  return CGFDM_OK;
}

int cgfdm_setup_from_directory_ex(const char *run_dir, int32_t precision, cgfdm_setup *out) {
  if (!run_dir || !out) return CGFDM_ERR_ARG;
  if (precision < CGFDM_FP32 || precision > CGFDM_FP64) return CGFDM_ERR_ARG;
  return guarded([&] {
    std::memset(out, 0, sizeof *out);
    // the arrays stay in the setup's own vectors; `owner` keeps them alive
    std::unique_ptr<cgfdm::Setup> s(new cgfdm::Setup);
    int rc = cgfdm::build_setup(run_dir, precision, *s);
    if (rc) return rc;
    out->desc = s->desc;
    out->cjm = s->cjm.data();
    out->rdz = s->rdz.data();
    out->coord = s->coord.data();
    out->medium = s->medium.data();
    out->pml = s->pml.data();
    out->point_src = s->point_src;
    std::memcpy(out->point_xyz, s->point_xyz, sizeof s->point_xyz);
    out->rickerfc = s->p.rickerfc;
    out->npts = (int64_t)s->src_index.size();
    out->src_nt = s->src_nt;
    out->src_dt = s->src_dt;
    out->src_index = s->src_index.data();
    out->moment_rate = s->moment_rate.data();
    out->nsta = (int32_t)s->sta_xyz.size() / 3;
    out->sta_xyz = s->sta_xyz.data();
    out->terrain = s->terrain.data();
    out->owner = s.release();
    return CGFDM_OK;
  });
}

int cgfdm_setup_from_directory(const char *run_dir, cgfdm_setup *out) {
  return cgfdm_setup_from_directory_ex(run_dir, CGFDM_FP32, out);
}

int cgfdm_free_setup(cgfdm_setup *s) {
  if (!s) return CGFDM_ERR_ARG;
  delete (cgfdm::Setup *)s->owner;
  std::memset(s, 0, sizeof *s);
  return CGFDM_OK;
}

namespace {

// Slice and free-surface snapshots of run_directory, written without
// stalling the time loop (data_io.cpp:323-495 file layout): each snapshot is
// packed on the work stream into a device staging slot, copied into a
// pinned host slot on a copy stream, and written to its files only when the
// slot comes round again (three slots), so the GPU keeps stepping meanwhile.
class SnapshotPipe {
 public:
  struct File {
    std::string name;
    char axis;
    size_t off, n;
  };
  ~SnapshotPipe() {
    for (auto &s : slots_) {
      if (s.dev) cudaFree(s.dev);
      if (s.host) cudaFreeHost(s.host);
      if (s.packed) cudaEventDestroy(s.packed);
      if (s.copied) cudaEventDestroy(s.copied);
    }
    if (copy_) cudaStreamDestroy(copy_);
  }
  int init(size_t floats) {
    floats_ = floats;
    if (cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking) != cudaSuccess) return fail();
    for (auto &s : slots_) {
      if (cudaMalloc(&s.dev, sizeof(float) * floats) != cudaSuccess ||
          cudaMallocHost(&s.host, sizeof(float) * floats) != cudaSuccess ||
          cudaEventCreateWithFlags(&s.packed, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming) != cudaSuccess)
        return fail();
    }
    return CGFDM_OK;
  }
  // The next slot's device buffer (after writing out what it held).
  int begin(float **dev) {
    Slot &s = slots_[next_];
    int rc = drain(s);
    if (rc) return rc;
    *dev = s.dev;
    return CGFDM_OK;
  }
  // The slot begun last is packed (on `work`): copy it out, remember files.
  int commit(cudaStream_t work, std::vector<File> files) {
    Slot &s = slots_[next_];
    if (cudaEventRecord(s.packed, work) != cudaSuccess ||
        cudaStreamWaitEvent(copy_, s.packed, 0) != cudaSuccess ||
        cudaMemcpyAsync(s.host, s.dev, sizeof(float) * floats_, cudaMemcpyDeviceToHost, copy_) !=
            cudaSuccess ||
        cudaEventRecord(s.copied, copy_) != cudaSuccess)
      return fail();
    s.files = std::move(files);
    s.pending = true;
    next_ = (next_ + 1) % kSlots;
    return CGFDM_OK;
  }
  int finish() {
    for (int q = 0; q < kSlots; ++q) {
      int rc = drain(slots_[(next_ + q) % kSlots]);
      if (rc) return rc;
    }
    return CGFDM_OK;
  }

 private:
  static constexpr int kSlots = 3;
  struct Slot {
    float *dev = nullptr, *host = nullptr;
    cudaEvent_t packed = nullptr, copied = nullptr;
    std::vector<File> files;
    bool pending = false;
  };
  int drain(Slot &s) {
    if (!s.pending) return CGFDM_OK;
    if (cudaEventSynchronize(s.copied) != cudaSuccess) return fail();
    s.pending = false;
    for (const File &f : s.files) {
      int rc = cgfdm::write_slice_file(f.name, f.axis, s.host + f.off, f.n);
      if (rc) return rc;
    }
    return CGFDM_OK;
  }
  int fail() {
    set_error(std::string("snapshot pipeline: ") + cudaGetErrorString(cudaGetLastError()));
    return CGFDM_ERR_CUDA;
  }
  Slot slots_[kSlots];
  size_t floats_ = 0;
  int next_ = 0;
  cudaStream_t copy_ = nullptr;
};

}  // namespace

int cgfdm_run_directory(const char *run_dir, int32_t precision, int32_t kernel, int32_t device) {
  if (!run_dir) return CGFDM_ERR_ARG;
  return guarded([&] {
    cgfdm::Setup s;
    int rc = cgfdm::build_setup(run_dir, precision, s);
    if (rc) return rc;
    s.desc.kernel = kernel;
    s.desc.device = device;
    std::string out = s.p.OUT;
    if (!out.empty() && out[0] != '/') out = std::string(run_dir) + "/" + out;
    mkdir(out.c_str(), 0777);  // createDir (create_dir.cpp)
    if ((rc = cgfdm::write_model_slices(s, out))) return rc;
    std::unique_ptr<cgfdm::Engine> eng;
    if ((rc = cgfdm::make_engine(s.desc, eng))) return rc;
    if ((rc = eng->set_model(s.cjm.data(), s.rdz.data()))) return rc;
    if (s.point_src &&
        (rc = eng->set_point_source(s.point_xyz[0], s.point_xyz[1], s.point_xyz[2], s.p.rickerfc)))
      return rc;
    if (!s.src_index.empty() &&
        (rc = eng->set_fault_source(s.src_index.data(), s.moment_rate.data(),
                                    (int64_t)s.src_index.size(), s.src_nt, s.src_dt, true)))
      return rc;
    const int nsta = (int)s.sta_xyz.size() / 3;
    if (nsta > 0 && (rc = eng->set_stations(s.sta_xyz.data(), nsta))) return rc;
    // propagate.cpp:142-198 with the slice output every IT_SKIP steps
    const int NT = s.desc.nt, skip = s.p.IT_SKIP > 0 ? s.p.IT_SKIP : NT + 1;
    const double cv_inv = (precision == CGFDM_FP16 || precision == CGFDM_BF16) ? 1.0 / 5.0e3 : 1.0;
    const int at[3] = {s.p.sliceX + 3, s.p.sliceY + 3, s.p.sliceZ + 3};
    const int lim[3] = {s.nx_ - 3, s.ny_ - 3, s.nz_ - 3};
    // what one snapshot holds: V slices through sliceX/Y/Z, free-surface V
    std::vector<std::pair<int, size_t>> slice_axes;  // (axis, points)
    size_t floats = 0;
    for (int ax = 0; ax < 3; ++ax) {
      if (at[ax] < 3 || at[ax] >= lim[ax]) continue;
      const size_t n = ax == 0 ? (size_t)s.p.NY * s.p.NZ : ax == 1 ? (size_t)s.p.NX * s.p.NZ
                                                                    : (size_t)s.p.NX * s.p.NY;
      slice_axes.push_back({ax, n});
      floats += 3 * n;
    }
    const size_t nsurf = (size_t)s.p.NX * s.p.NY;
    if (s.p.sliceFreeSurf) floats += 3 * nsurf;
    SnapshotPipe pipe;
    if (floats > 0 && (rc = pipe.init(floats))) return rc;
    const char *vn[3] = {"Vx", "Vy", "Vz"};
    for (int it = 0; it < NT; ++it) {
      if ((rc = eng->run(1, nullptr))) return rc;
      if (floats == 0 || it % skip != 0) continue;
      float *dev = nullptr;
      if ((rc = pipe.begin(&dev))) return rc;
      std::vector<SnapshotPipe::File> files;
      size_t off = 0;
      char name[512];
      for (const auto &sa : slice_axes) {
        const int ax = sa.first;
        for (int v = 0; v < 3; ++v) {
          if ((rc = eng->enqueue_slice(v, ax, at[ax], cv_inv, dev + off))) return rc;
          std::snprintf(name, sizeof name, "%s/%s_%d", out.c_str(), vn[v], it);
          files.push_back({name, "XYZ"[ax], off, sa.second});
          off += sa.second;
        }
      }
      if (s.p.sliceFreeSurf) {
        for (int v = 0; v < 3; ++v) {  // the top interior layer (data_io.cpp:481-491)
          if ((rc = eng->enqueue_slice(v, 2, s.nz_ - 3 - 1, cv_inv, dev + off))) return rc;
          std::snprintf(name, sizeof name, "%s/FreeSurf%s_%d", out.c_str(), vn[v], it);
          files.push_back({name, 'Z', off, nsurf});
          off += nsurf;
        }
      }
      if ((rc = pipe.commit(eng->work_stream(), std::move(files)))) return rc;
    }
    if (floats > 0 && (rc = pipe.finish())) return rc;
    if ((rc = eng->synchronize())) return rc;
    if (nsta > 0) {
      std::vector<float> wave((size_t)nsta * NT * 9);
      if ((rc = eng->get_stations(wave.data()))) return rc;
      if ((rc = cgfdm::write_station_file(s, out, wave.data()))) return rc;
    }
    std::vector<float> pgv(2 * (size_t)s.p.NX * s.p.NY);
    if ((rc = eng->get_pgv(pgv.data()))) return rc;
    return cgfdm::write_pgv_file(s, out, pgv.data());
  });
}

}  // extern "C"
