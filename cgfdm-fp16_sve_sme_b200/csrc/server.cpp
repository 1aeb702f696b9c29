// Request loop with continuous batching (cgfdm_server_* of the C ABI).
//
// Requests (one simulation each: grid, model, sources, stations, precision)
// are queued by submit() from any host thread.  Two threads do the work:
//   * admission thread: queued requests are admitted in arrival order while
//     their device footprint (engine_device_bytes) fits the HBM budget; it
//     creates each engine and uploads the inputs on the engine's own stream,
//     overlapping the rounds that are running; a request larger than the
//     whole budget fails at submission;
//   * worker thread, in rounds: all running requests of one precision
//     advance together as one batch (batched persistent streaming launches,
//     optionally one CUDA graph per step) by `chunk` steps, or fewer when a
//     member has fewer left; the FP32, FP16, BF16 and FP64 batches of a round
//     run on their own streams, so their work overlaps on the device; after a
//     round each member's new seismogram rows are copied into the request's
//     host buffer (streamed back chunk by chunk), finished requests copy
//     their PGV map, release their device memory and leave the batch, and the
//     requests admitted meanwhile join the next round, after a short first
//     round of their own (a tenth of the chunk, eager) that streams their
//     first seismogram rows back early.
// Wavefields stay resident on the device from admission to completion.
// Latencies are measured from submission: to the first streamed seismogram
// chunk, and to completion.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cgfdm_b200.h"
#include "engine.h"

namespace cgfdm {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  cgfdm_desc desc{};
  std::vector<float> cjm, rdz, rate;
  std::vector<int64_t> src_index;
  std::vector<int32_t> sta;
  int point = 0;
  int32_t point_xyz[3] = {0, 0, 0};
  float rickerfc = 0;
  int32_t src_nt = 0;
  float src_dt = 0;
  int64_t bytes = 0;
  bool admitted = false;  // its bytes count against the budget
  bool cancel = false;    // cancellation asked while admitted: retire after the round
  // results
  std::vector<float> wave, pgv;
  int steps = 0;          // steps whose seismograms are in `wave`
  int state = CGFDM_REQ_QUEUED;
  int error = CGFDM_OK;
  std::string error_text;
  Clock::time_point t_submit, t_first, t_done;
  std::unique_ptr<Engine> eng;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (pos - lo) * (v[hi] - v[lo]);
}

}  // namespace

class Server {
 public:
  explicit Server(const cgfdm_server_opts &o) : opts_(o) {
    if (opts_.chunk_steps <= 0) opts_.chunk_steps = 100;
  }
  ~Server() { stop(); }

  int start() {
    if (cudaSetDevice(opts_.device) != cudaSuccess) {
      set_error("server: no such CUDA device");
      return CGFDM_ERR_NO_KERNEL;
    }
    if (opts_.hbm_budget_bytes <= 0) {
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        set_error("server: cudaMemGetInfo failed");
        return CGFDM_ERR_CUDA;
      }
      const int64_t reserve = 4LL << 30;  // CUDA context, graphs, scratch
      budget_ = (int64_t)fr > reserve ? (int64_t)fr - reserve : (int64_t)fr / 2;
    } else {
      budget_ = opts_.hbm_budget_bytes;
    }
    for (int q = 0; q < 4; ++q)
      if (cudaStreamCreateWithFlags(&streams_[q], cudaStreamNonBlocking) != cudaSuccess) {
        set_error("server: stream creation failed");
        return CGFDM_ERR_CUDA;
      }
    worker_ = std::thread([this] { loop(); });
    admitter_ = std::thread([this] { admit_loop(); });
    return CGFDM_OK;
  }

  void stop() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (stopping_) return;
      stopping_ = true;
    }
    cv_.notify_all();
    work_cv_.notify_all();
    if (admitter_.joinable()) admitter_.join();
    if (worker_.joinable()) worker_.join();
    cudaSetDevice(opts_.device);
    batches_.clear();
    for (auto &kv : reqs_) kv.second->eng.reset();
    for (auto &s : streams_)
      if (s) cudaStreamDestroy(s);
  }

  int submit(std::unique_ptr<Request> r, int64_t *id) {
    int64_t bytes = engine_device_bytes(r->desc);
    if (bytes <= 0) {
      set_error("server: invalid request descriptor");
      return CGFDM_ERR_ARG;
    }
    if (bytes > budget_) {
      set_error("server: request needs " + std::to_string(bytes) + " device bytes, budget " +
                std::to_string(budget_));
      return CGFDM_ERR_NOMEM;
    }
    r->bytes = bytes;
    r->wave.assign((size_t)r->sta.size() / 3 * r->desc.nt * 9, 0.0f);
    r->pgv.assign((size_t)2 * r->desc.nx * r->desc.ny, 0.0f);
    r->t_submit = Clock::now();
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!have_first_) {
        have_first_ = true;
        t_first_submit_ = r->t_submit;
      }
      r->id = ++next_id_;
      *id = r->id;
      queue_.push_back(r->id);
      reqs_[r->id] = std::move(r);
    }
    cv_.notify_all();
    return CGFDM_OK;
  }

  int poll(int64_t id, int32_t *state, int32_t *steps) {
    std::lock_guard<std::mutex> lk(mu_);
    auto f = reqs_.find(id);
    if (f == reqs_.end()) {
      set_error("server: unknown request");
      return CGFDM_ERR_ARG;
    }
    if (state) *state = f->second->state;
    if (steps) *steps = f->second->steps;
    return CGFDM_OK;
  }

  // Copies seismogram rows [from, steps) (the rows streamed back so far).
  int read_rows(int64_t id, int32_t from, float *wave, int32_t *upto) {
    std::lock_guard<std::mutex> lk(mu_);
    auto f = reqs_.find(id);
    if (f == reqs_.end()) {
      set_error("server: unknown request");
      return CGFDM_ERR_ARG;
    }
    Request &r = *f->second;
    const int nsta = (int)r.sta.size() / 3, nt = r.desc.nt;
    from = std::max(0, std::min(from, r.steps));
    for (int s = 0; s < nsta; ++s)
      std::memcpy(wave + ((size_t)s * nt + from) * 9, r.wave.data() + ((size_t)s * nt + from) * 9,
                  sizeof(float) * 9 * (size_t)(r.steps - from));
    if (upto) *upto = r.steps;
    return CGFDM_OK;
  }

  int cancel(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto f = reqs_.find(id);
    if (f == reqs_.end()) {
      set_error("server: unknown request");
      return CGFDM_ERR_ARG;
    }
    Request &r = *f->second;
    if (r.state == CGFDM_REQ_QUEUED && !r.admitted) {
      queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
      r.state = CGFDM_REQ_CANCELLED;
      r.t_done = Clock::now();
      done_cv_.notify_all();
      cv_.notify_all();
      return CGFDM_OK;
    }
    if (r.state == CGFDM_REQ_QUEUED || r.state == CGFDM_REQ_RUNNING) {
      r.cancel = true;  // the worker retires it after its current round
      return CGFDM_OK;
    }
    set_error("server: the request has already ended");
    return CGFDM_ERR_STATE;
  }

  int wait(int64_t id, float *wave, float *pgv, double *lat_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto f = reqs_.find(id);
    if (f == reqs_.end()) {
      set_error("server: unknown request");
      return CGFDM_ERR_ARG;
    }
    Request *r = f->second.get();
    done_cv_.wait(lk, [&] {
      return r->state == CGFDM_REQ_DONE || r->state == CGFDM_REQ_FAILED ||
             r->state == CGFDM_REQ_CANCELLED;
    });
    if (r->state == CGFDM_REQ_CANCELLED) {
      set_error("server: the request was cancelled");
      reqs_.erase(f);
      return CGFDM_ERR_CANCELLED;
    }
    if (r->state == CGFDM_REQ_FAILED) {
      set_error(r->error_text);
      const int e = r->error;
      reqs_.erase(f);
      return e;
    }
    if (wave) std::memcpy(wave, r->wave.data(), sizeof(float) * r->wave.size());
    if (pgv) std::memcpy(pgv, r->pgv.data(), sizeof(float) * r->pgv.size());
    if (lat_ms) {
      lat_ms[0] = ms_between(r->t_submit, r->t_first);
      lat_ms[1] = ms_between(r->t_submit, r->t_done);
    }
    reqs_.erase(f);
    return CGFDM_OK;
  }

  int stats(double *out) {
    std::lock_guard<std::mutex> lk(mu_);
    out[0] = percentile(lat_first_, 0.5);
    out[1] = percentile(lat_first_, 0.99);
    out[2] = percentile(lat_done_, 0.5);
    out[3] = percentile(lat_done_, 0.99);
    const double span = have_first_ ? std::chrono::duration<double>(t_last_done_ - t_first_submit_).count() : 0.0;
    out[4] = span > 0 ? updates_ / span / 1e9 : 0.0;
    out[5] = (double)lat_done_.size();
    out[6] = busy_s_;
    out[7] = (double)peak_bytes_;
    return CGFDM_OK;
  }

 private:
  // Creates the request's engine and uploads its inputs (worker thread).
  int admit(Request &r) {
    int rc = make_engine(r.desc, r.eng);
    if (!rc) rc = r.eng->set_model(r.cjm.data(), r.rdz.data());
    if (!rc && r.point)
      rc = r.eng->set_point_source(r.point_xyz[0], r.point_xyz[1], r.point_xyz[2], r.rickerfc);
    if (!rc && !r.src_index.empty())
      rc = r.eng->set_fault_source(r.src_index.data(), r.rate.data(),
                                   (int64_t)r.src_index.size(), r.src_nt, r.src_dt, true);
    if (!rc) rc = r.eng->set_stations(r.sta.data(), (int)r.sta.size() / 3);
    if (!rc) rc = r.eng->set_tile_rows(16);
    if (!rc) rc = r.eng->synchronize();
    // the host copies of the inputs are not needed any more
    std::vector<float>().swap(r.cjm);
    std::vector<float>().swap(r.rdz);
    std::vector<float>().swap(r.rate);
    return rc;
  }

  void fail(Request &r, int rc) {
    r.error = rc;
    r.error_text = last_error();
    r.state = CGFDM_REQ_FAILED;
    r.t_done = Clock::now();
    r.eng.reset();
    if (r.admitted) used_ -= r.bytes;
    r.admitted = false;
  }

  // Admission thread: creates the engines of queued requests and uploads
  // their inputs (on each engine's own stream) while the worker's rounds run.
  void admit_loop() {
    cudaSetDevice(opts_.device);
    for (;;) {
      Request *r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] {
          return stopping_ ||
                 (!queue_.empty() && used_ + reqs_[queue_.front()]->bytes <= budget_);
        });
        if (stopping_) return;
        r = reqs_[queue_.front()].get();
        used_ += r->bytes;  // reserved before the engine exists
        r->admitted = true;
        peak_bytes_ = std::max(peak_bytes_, used_);
        queue_.pop_front();
      }
      int rc = admit(*r);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (rc) {
          fail(*r, rc);
        } else {
          r->state = CGFDM_REQ_RUNNING;
          ready_.push_back(r);
        }
      }
      done_cv_.notify_all();
      work_cv_.notify_all();
    }
  }

  using Slots = std::map<int, std::pair<std::vector<Engine *>, std::unique_ptr<BatchBase>>>;

  void loop() {
    cudaSetDevice(opts_.device);
    std::vector<Request *> active;
    // a newly admitted request first advances this many steps in a round of
    // its own (eager, no graphs), so that its first seismogram rows come back
    // without waiting for a full round of every running request
    const int first_chunk = std::max(1, opts_.chunk_steps / 10);
    for (;;) {
      std::vector<Request *> fresh;
      {
        std::unique_lock<std::mutex> lk(mu_);
        work_cv_.wait(lk, [&] { return stopping_ || !ready_.empty() || !active.empty(); });
        if (stopping_) return;
        // requests admitted since the last round join this one
        fresh = ready_;
        active.insert(active.end(), ready_.begin(), ready_.end());
        ready_.clear();
      }
      if (active.empty()) continue;
      if (!fresh.empty() && first_chunk < opts_.chunk_steps) {
        run_round(active, fresh, first_chunk, fresh_batches_, false);
        fresh_batches_.clear();  // one-off batches: their members join the main ones
      }
      if (!active.empty()) run_round(active, active, opts_.chunk_steps, batches_, opts_.use_graph);
    }
  }

  // One round over `members` (a subset of `active`): a batch per precision,
  // each on its own stream, advanced by at most `cap` steps; then the new
  // seismogram rows are streamed back and finished requests retired (and
  // removed from `active`).
  void run_round(std::vector<Request *> &active, std::vector<Request *> members, int cap,
             Slots &slots, bool graph) {
    const auto t0 = Clock::now();
    std::map<int, std::vector<Request *>> groups;
    for (Request *r : members) groups[r->desc.precision].push_back(r);
    std::vector<std::pair<std::vector<Request *>, int>> ran;
    int q = 0;
    for (auto &g : groups) {
      std::vector<Request *> &m = g.second;
      int k = cap;
      for (Request *r : m) k = std::min(k, r->desc.nt - r->eng->steps_done());
      std::vector<Engine *> e;
      for (Request *r : m) e.push_back(r->eng.get());
      BatchBase *b = batch_for(slots, g.first, e, graph);
      int rc = b ? b->run(k, streams_[q++ % 4]) : CGFDM_ERR_ARG;
      if (rc) {
        // before the members' engines go
        batches_.erase(g.first);
        fresh_batches_.erase(g.first);
        for (Request *r : m) r->eng.reset();
        std::lock_guard<std::mutex> lk(mu_);
        for (Request *r : m) {
          active.erase(std::remove(active.begin(), active.end(), r), active.end());
          fail(*r, rc);
        }
        done_cv_.notify_all();
        cv_.notify_all();
        continue;
      }
      ran.push_back({m, k});
    }
    // stream the new seismogram rows back; retire finished requests.  Order
    // matters: results are copied first, then the batches that hold a
    // finishing member are destroyed, then the members' engines, and only
    // then is a request marked (wait() may release it at once).
    struct Retire {
      Request *r;
      int rc;
    };
    std::vector<Retire> retire;
    for (auto &g : ran) {
      for (Request *r : g.first) {
        const int it1 = r->eng->steps_done(), it0 = it1 - g.second;
        int rc = r->eng->get_station_rows(r->wave.data(), it0, it1);
        const bool finished = it1 >= r->desc.nt;
        if (!rc && finished) rc = r->eng->get_pgv(r->pgv.data());
        std::lock_guard<std::mutex> lk(mu_);
        if (!rc) {
          updates_ += (double)r->desc.nx * r->desc.ny * r->desc.nz * g.second;
          if (r->steps == 0) {
            r->t_first = Clock::now();
            lat_first_.push_back(ms_between(r->t_submit, r->t_first));
          }
          r->steps = it1;
        }
        if (rc || finished || r->cancel) retire.push_back({r, rc});
      }
    }
    for (const Retire &x : retire) {
      batches_.erase(x.r->desc.precision);
      fresh_batches_.erase(x.r->desc.precision);
    }
    for (const Retire &x : retire) x.r->eng.reset();
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (const Retire &x : retire) {
        Request *r = x.r;
        active.erase(std::remove(active.begin(), active.end(), r), active.end());
        if (x.rc) {
          fail(*r, x.rc);
          continue;
        }
        used_ -= r->bytes;
        r->admitted = false;
        if (r->cancel && r->steps < r->desc.nt) {
          r->state = CGFDM_REQ_CANCELLED;
          r->t_done = Clock::now();
          continue;
        }
        r->t_done = Clock::now();
        t_last_done_ = r->t_done;
        lat_done_.push_back(ms_between(r->t_submit, r->t_done));
        r->state = CGFDM_REQ_DONE;
      }
      busy_s_ += std::chrono::duration<double>(Clock::now() - t0).count();
    }
    done_cv_.notify_all();
    if (!retire.empty()) cv_.notify_all();  // memory came free
  }

  // The batch of exactly these members (rebuilt when membership changes, so
  // that graphs are captured once per membership).
  BatchBase *batch_for(Slots &slots, int precision, const std::vector<Engine *> &m, bool graph) {
    auto &slot = slots[precision];
    if (slot.first != m || !slot.second) {
      slot.second.reset();
      slot.first = m;
      if (make_batch(m.data(), (int)m.size(), slot.second)) {
        slot.second.reset();
        return nullptr;
      }
      if (graph) slot.second->set_graph(true);
    }
    return slot.second.get();
  }

  cgfdm_server_opts opts_;
  int64_t budget_ = 0, used_ = 0, peak_bytes_ = 0;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_, work_cv_;  // admission, results, rounds
  std::vector<Request *> ready_;  // admitted, not yet in a round
  std::deque<int64_t> queue_;
  std::map<int64_t, std::unique_ptr<Request>> reqs_;
  int64_t next_id_ = 0;
  bool stopping_ = false;
  std::thread worker_, admitter_;
  cudaStream_t streams_[4] = {};
  Slots batches_;        // the main batch of each precision (graphs, when on)
  Slots fresh_batches_;  // the first, short round of newly admitted requests
  std::vector<double> lat_first_, lat_done_;
  double updates_ = 0, busy_s_ = 0;
  bool have_first_ = false;
  Clock::time_point t_first_submit_, t_last_done_;
};

}  // namespace cgfdm

struct cgfdm_server {
  std::unique_ptr<cgfdm::Server> s;
};

extern "C" {

int cgfdm_server_cancel(cgfdm_server *sv, int64_t id) {
  if (!sv || !sv->s) return CGFDM_ERR_ARG;
  return sv->s->cancel(id);
}

int cgfdm_server_create(const cgfdm_server_opts *opts, cgfdm_server **out) {
  if (!opts || !out) return CGFDM_ERR_ARG;
  *out = nullptr;
  try {
    auto *h = new cgfdm_server();
    h->s.reset(new cgfdm::Server(*opts));
    int rc = h->s->start();
    if (rc) {
      delete h;
      return rc;
    }
    *out = h;
    return CGFDM_OK;
  } catch (const std::exception &e) {
    cgfdm::set_error(e.what());
    return CGFDM_ERR_NOMEM;
  }
}

int cgfdm_server_submit(cgfdm_server *sv, const cgfdm_desc *desc, const float *cjm,
                        const float *rdz, int32_t point_src, const int32_t *point_xyz,
                        float rickerfc, const int64_t *src_index, const float *moment_rate,
                        int64_t npts, int32_t src_nt, float src_dt, const int32_t *sta_xyz,
                        int32_t nsta, int64_t *id) {
  if (!sv || !sv->s || !desc || !cjm || !rdz || !id || nsta < 0 || npts < 0) return CGFDM_ERR_ARG;
  if (desc->nx <= 0 || desc->ny <= 0 || desc->nz <= 0 || desc->nt <= 0) return CGFDM_ERR_ARG;
  try {
    std::unique_ptr<cgfdm::Request> r(new cgfdm::Request);
    r->desc = *desc;
    const size_t num = (size_t)(desc->nx + 6) * (desc->ny + 6) * (desc->nz + 6);
    const size_t nsurf = (size_t)(desc->nx + 6) * (desc->ny + 6);
    r->cjm.assign(cjm, cjm + 13 * num);
    r->rdz.assign(rdz, rdz + 18 * nsurf);
    r->point = point_src ? 1 : 0;
    if (point_src && point_xyz) std::memcpy(r->point_xyz, point_xyz, sizeof r->point_xyz);
    r->rickerfc = rickerfc;
    if (npts > 0 && src_index && moment_rate) {
      r->src_index.assign(src_index, src_index + npts);
      r->rate.assign(moment_rate, moment_rate + (size_t)npts * src_nt * 6);
      r->src_nt = src_nt;
      r->src_dt = src_dt;
    }
    if (nsta > 0 && sta_xyz) r->sta.assign(sta_xyz, sta_xyz + 3 * nsta);
    return sv->s->submit(std::move(r), id);
  } catch (const std::bad_alloc &) {
    cgfdm::set_error("server: host memory exhausted");
    return CGFDM_ERR_NOMEM;
  }
}

int cgfdm_server_poll(cgfdm_server *sv, int64_t id, int32_t *state, int32_t *steps) {
  if (!sv || !sv->s) return CGFDM_ERR_ARG;
  return sv->s->poll(id, state, steps);
}

int cgfdm_server_read_rows(cgfdm_server *sv, int64_t id, int32_t from, float *wave,
                           int32_t *upto) {
  if (!sv || !sv->s || !wave) return CGFDM_ERR_ARG;
  return sv->s->read_rows(id, from, wave, upto);
}

int cgfdm_server_wait(cgfdm_server *sv, int64_t id, float *wave, float *pgv, double *lat_ms) {
  if (!sv || !sv->s) return CGFDM_ERR_ARG;
  return sv->s->wait(id, wave, pgv, lat_ms);
}

int cgfdm_server_stats(cgfdm_server *sv, double *out8) {
  if (!sv || !sv->s || !out8) return CGFDM_ERR_ARG;
  return sv->s->stats(out8);
}

int cgfdm_server_destroy(cgfdm_server *sv) {
  delete sv;
  return CGFDM_OK;
}

}  // extern "C"
