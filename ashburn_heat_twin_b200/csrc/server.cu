// Continuous-batching server behind the C ABI (ahx_server_*, include/ahx.h): one scheduler thread per server owns
// a set of solver slots (handles) and one batch (ahx_batch_*) on one device.
//
// The reference serves one scenario per page (js/live.js:69-86: step, then read, in a loop). Here many scenario solves
// share the device: requests arrive through ahx_server_submit (host byte images, copied), queue in arrival order, and
// the scheduler loop
//   1. admits the head of the queue while the resident cells stay under max_cells and the slots' device memory under
//      the HBM budget (a finished request's slot of the same grid is reused; idle slots of other grids are released to
//      make room; the first request is always admitted);
//   2. configures the slot as the reference's resetFlow leaves a solver (parameter block, column records and ktop
//      uploaded, equilibrium flow, theta 0, parity 0; solver.js:380-398), so the answer is the one a fresh solver
//      would give;
//   3. steps every active request together for k = min(chunk, fewest steps left) steps with one batched launch
//      sequence (the member list follows the active requests, so requests join and leave between chunks), queueing at
//      most `depth` chunks ahead of the device;
//   4. answers a request whose steps are done with the read-back of its state (ahx_read_submit / ahx_read_wait on its
//      slot, ordered after the chunk), after which the slot returns to the idle pool of its grid.
// Device work is asynchronous throughout; the thread waits only for the chunk `depth` places back and polls read-backs
// without blocking. A CUDA error marks the server lost: every unanswered request ends with AHX_EDEVICE.
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

#include "ahx.h"
#include "handle.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  uint64_t ticket = 0, tag = 0;
  int nx = 0, ny = 0, nz = 0, steps = 0, nzv = 0, want_vol = 0, want_wind = 0;
  float conv = 0.f, volscale = 0.f;
  std::vector<unsigned char> params;
  std::vector<uint32_t> colv, ktop;
  double t_submit = 0, t_admit = -1, t_done = -1;
  bool done = false;
  int status = AHX_OK;
  std::string err;
  std::vector<float> surf;     // surf, u, v: 3 * NXY
  std::vector<uint8_t> vol;    // nzv * NXY
  float theta_max = 0.f;
  uint64_t grid_key() const { return ((uint64_t)nx << 42) | ((uint64_t)ny << 21) | (uint64_t)nz; }
  int64_t cells() const { return (int64_t)nx * ny * nz; }
};

struct Slot {
  ahx_handle* h = nullptr;
  uint64_t key = 0;
  int64_t cells = 0;
  uint64_t bytes = 0;
  std::shared_ptr<Req> req;
  int left = 0;
  uint64_t read_ticket = 0;
};

// a queued chunk: an event recorded on a member's stream after the batched steps (every member's stream waits for
// the batch), owned by the server so it outlives the member
struct Chunk {
  cudaEvent_t ev;
};

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

}  // namespace

struct ahx_server {
  ahx_server_config cfg{};
  int dev = 0;
  Clock::time_point t0;
  std::thread worker;
  // shared with the API threads (under mu)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Req>> incoming;
  std::map<uint64_t, std::shared_ptr<Req>> open;   // submitted, not yet collected by ahx_server_poll
  uint64_t next_ticket = 0;
  bool stop = false, destroyed = false, lost = false;
  std::string lost_msg;
  ahx_server_stats_out st{};
  // scheduler thread only
  std::deque<std::shared_ptr<Req>> pending;
  std::vector<Slot*> slots, active, draining;
  std::map<uint64_t, std::vector<Slot*>> idle;
  std::map<uint64_t, std::pair<int, int>> tuned;   // grid -> (block_y encoding, zslab)
  ahx_batch* batch = nullptr;
  std::vector<ahx_handle*> members;
  std::deque<Chunk> inflight;
  std::vector<cudaEvent_t> spare_events;
  uint64_t budget = 0, bytes_used = 0;
  int64_t resident = 0;
};

namespace {

std::string last_msg() { return std::string(ahx_last_error()); }

// end a request (under the caller's lock of S->mu)
void finish_locked(ahx_server* S, const std::shared_ptr<Req>& r, int status, const std::string& err) {
  r->done = true;
  r->status = status;
  r->err = err;
  r->t_done = seconds_since(S->t0);
  ++S->st.completed;
}

void finish(ahx_server* S, const std::shared_ptr<Req>& r, int status, const std::string& err = std::string()) {
  std::lock_guard<std::mutex> lk(S->mu);
  finish_locked(S, r, status, err);
  S->cv_done.notify_all();
}

void publish(ahx_server* S) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->st.queued = (int64_t)S->pending.size() + (int64_t)S->incoming.size();
  S->st.active = (int64_t)S->active.size();
  S->st.slots = (int64_t)S->slots.size();
  int64_t n = 0;
  for (auto& kv : S->idle) n += (int64_t)kv.second.size();
  S->st.idle_slots = n;
  S->st.resident_cells = S->resident;
  S->st.slot_bytes = S->bytes_used;
  S->st.hbm_budget_bytes = S->budget;
}

// the server cannot go on (device error): every request not yet answered ends with `status`
void go_lost(ahx_server* S, int status, const std::string& why) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->lost = true;
  S->lost_msg = why;
  for (auto& kv : S->open)
    if (!kv.second->done) finish_locked(S, kv.second, status, why);
  S->incoming.clear();
  S->pending.clear();
  S->cv_done.notify_all();
}

// release one idle slot of a grid other than `keep`; false when there is none
bool evict_idle(ahx_server* S, uint64_t keep) {
  for (auto& kv : S->idle) {
    if (kv.first == keep || kv.second.empty()) continue;
    Slot* sl = kv.second.back();
    kv.second.pop_back();
    ahx_destroy(sl->h);
    S->bytes_used -= std::min(S->bytes_used, sl->bytes);
    S->slots.erase(std::find(S->slots.begin(), S->slots.end(), sl));
    delete sl;
    std::lock_guard<std::mutex> lk(S->mu);
    ++S->st.evictions;
    return true;
  }
  return false;
}

int esize_f(int precision) { return precision == AHX_FP64 ? 8 : (precision == AHX_FP32 ? 4 : 2); }
int esize_g(int precision) {
  return precision == AHX_FP64 ? 8
         : (precision == AHX_FP32 || precision == AHX_FP16_G32 || precision == AHX_BF16_G32) ? 4
                                                                                              : 2;
}

// a slot for r: an idle one of its grid, or a new one while the budget allows. *status is set on a hard failure
// (then nullptr); nullptr with AHX_OK means "wait for memory".
Slot* take_slot(ahx_server* S, const Req& r, ahx_status* status) {
  *status = AHX_OK;
  const uint64_t key = r.grid_key();
  auto it = S->idle.find(key);
  if (it != S->idle.end() && !it->second.empty()) {
    Slot* sl = it->second.back();
    it->second.pop_back();
    return sl;
  }
  uint64_t need = 0;
  for (Slot* sl : S->slots)
    if (sl->key == key) need = sl->bytes;
  if (!need)
    need = (uint64_t)((double)r.cells() * 2.0 *
                      (19.0 * esize_f(S->cfg.precision) + 7.0 * esize_g(S->cfg.precision)) * 1.08);
  while (S->bytes_used + need > S->budget && evict_idle(S, key)) {
  }
  if (S->bytes_used + need > S->budget && !S->slots.empty()) return nullptr;
  size_t free0 = 0, free1 = 0, total = 0;
  cudaMemGetInfo(&free0, &total);
  ahx_dims d{};
  d.nx = r.nx;
  d.ny = r.ny;
  d.nz = r.nz;
  d.precision = S->cfg.precision;
  d.device_ordinal = S->dev;
  d.arith = S->cfg.arith;
  ahx_handle* h = nullptr;
  const ahx_status e = ahx_create(&d, &h);
  if (e != AHX_OK) {
    if (e == AHX_ENOMEM && !S->slots.empty()) return nullptr;   // wait for running requests to free memory
    *status = e;
    return nullptr;
  }
  cudaMemGetInfo(&free1, &total);
  Slot* sl = new Slot;
  sl->h = h;
  sl->key = key;
  sl->cells = r.cells();
  sl->bytes = std::max<uint64_t>(need, free0 > free1 ? (uint64_t)(free0 - free1) : 0);
  S->bytes_used += sl->bytes;
  S->slots.push_back(sl);
  return sl;
}

// the state resetFlow leaves behind for this request's images (solver.js:380-398)
ahx_status configure(ahx_server* S, Slot* sl, const Req& r) {
  ahx_handle* h = sl->h;
  ahx_status e;
  if ((e = ahx_set_params(h, r.params.data(), r.params.size())) != AHX_OK) return e;
  if ((e = ahx_set_ktop(h, r.ktop.data(), nullptr)) != AHX_OK) return e;
  if ((e = ahx_set_columns(h, r.colv.data())) != AHX_OK) return e;
  if ((e = ahx_init_flow(h)) != AHX_OK) return e;
  if ((e = ahx_clear_heat(h)) != AHX_OK) return e;
  if ((e = ahx_set_parity(h, 0)) != AHX_OK) return e;
  if (S->cfg.tune) {
    auto t = S->tuned.find(sl->key);
    if (t == S->tuned.end()) {
      int by = 0, zs = 0;
      float ms = 0;
      if ((e = ahx_autotune(h, 3, &by, &zs, &ms)) != AHX_OK) return e;   // trials on scratch copies of the state
      S->tuned[sl->key] = {by, zs};
    } else {
      if ((e = ahx_set_launch(h, t->second.first, t->second.second)) != AHX_OK) return e;
    }
  }
  return AHX_OK;
}

// keep the batch's member list equal to the active slots (stream-ordered, no synchronisation)
ahx_status sync_members(ahx_server* S) {
  std::vector<ahx_handle*> want;
  for (Slot* sl : S->active) want.push_back(sl->h);
  if (want == S->members) return AHX_OK;
  ahx_status e;
  if (!S->batch) {
    if (want.empty()) return AHX_OK;
    if ((e = ahx_batch_create(want.data(), (int)want.size(), &S->batch)) != AHX_OK) return e;
    e = S->cfg.batch_mode == 1 ? ahx_batch_set_launch(S->batch, 5, 8, 1, -1) : ahx_batch_set_launch(S->batch, 0, 0, 2, -1);
    if (e != AHX_OK) return e;
  } else if ((e = ahx_batch_set_members(S->batch, want.data(), (int)want.size())) != AHX_OK) {
    return e;
  }
  S->members = want;
  return AHX_OK;
}

// answer the requests whose read-back has arrived (without waiting)
ahx_status poll_reads(ahx_server* S) {
  std::vector<Slot*> keep;
  for (Slot* sl : S->draining) {
    Req& r = *sl->req;
    const size_t NXY = (size_t)r.nx * r.ny;
    const ahx_status e = ahx_read_wait(sl->h, sl->read_ticket, 0, r.surf.data(), r.surf.data() + NXY,
                                       r.surf.data() + 2 * NXY, r.want_vol ? r.vol.data() : nullptr, &r.theta_max);
    if (e == AHX_ETIMEOUT) {
      keep.push_back(sl);
      continue;
    }
    if (e != AHX_OK) return e;
    finish(S, sl->req, AHX_OK);
    sl->req.reset();
    S->idle[sl->key].push_back(sl);
  }
  S->draining.swap(keep);
  return AHX_OK;
}

// one pass of the scheduler loop; returns a non-OK status when the server cannot go on
ahx_status schedule(ahx_server* S) {
  ahx_status e;
  // 1-2: admission in arrival order
  while (!S->pending.empty()) {
    std::shared_ptr<Req> r = S->pending.front();
    if (!S->active.empty() && S->resident + r->cells() > S->cfg.max_cells) break;
    ahx_status se = AHX_OK;
    Slot* sl = take_slot(S, *r, &se);
    if (!sl) {
      if (se == AHX_OK) break;   // wait for memory
      S->pending.pop_front();
      finish(S, r, se, last_msg());
      continue;
    }
    if ((e = configure(S, sl, *r)) != AHX_OK) return e;
    S->pending.pop_front();
    sl->req = r;
    sl->left = r->steps;
    S->resident += sl->cells;
    r->t_admit = seconds_since(S->t0);
    r->surf.assign((size_t)3 * r->nx * r->ny, 0.f);
    if (r->want_vol) r->vol.assign((size_t)r->nzv * r->nx * r->ny, 0);
    S->active.push_back(sl);
    std::lock_guard<std::mutex> lk(S->mu);
    ++S->st.admitted;
  }
  // 3: one chunk over the active requests
  if (!S->active.empty()) {
    int k = S->cfg.chunk;
    for (Slot* sl : S->active) k = std::min(k, sl->left);
    if (k > 0) {
      if ((e = sync_members(S)) != AHX_OK) return e;
      if ((e = ahx_batch_step(S->batch, k)) != AHX_OK) return e;
      Chunk c{nullptr};
      if (!S->spare_events.empty()) {
        c.ev = S->spare_events.back();
        S->spare_events.pop_back();
      } else if (cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming) != cudaSuccess) {
        ahx::set_last_error("live solver: server: cudaEventCreate failed");
        return AHX_EDEVICE;
      }
      if (cudaEventRecord(c.ev, S->active[0]->h->s_step) != cudaSuccess) {
        S->spare_events.push_back(c.ev);
        ahx::set_last_error("live solver: server: cudaEventRecord failed");
        return AHX_EDEVICE;
      }
      S->inflight.push_back(c);
      std::lock_guard<std::mutex> lk(S->mu);
      ++S->st.chunks;
      S->st.batch_steps += k;
      S->st.cell_updates += (int64_t)k * S->resident;
    }
    // 4: requests whose steps are done: queue their read-back behind the chunk
    std::vector<Slot*> still;
    for (Slot* sl : S->active) {
      sl->left -= k;
      if (sl->left > 0) {
        still.push_back(sl);
        continue;
      }
      const Req& r = *sl->req;
      if ((e = ahx_read_submit(sl->h, r.conv, r.volscale, r.nzv, r.want_vol, r.want_wind, &sl->read_ticket)) !=
          AHX_OK)
        return e;
      S->resident -= sl->cells;
      S->draining.push_back(sl);
    }
    if (still.size() != S->active.size()) {
      S->active.swap(still);
      if ((e = sync_members(S)) != AHX_OK) return e;   // leavers are released at once
    }
  }
  // at most `depth` chunks queued ahead; all of them drained when nothing is active
  while (!S->inflight.empty() && ((int)S->inflight.size() > S->cfg.depth || S->active.empty())) {
    const cudaError_t q = cudaEventQuery(S->inflight.front().ev);
    if (q == cudaSuccess) {
      S->spare_events.push_back(S->inflight.front().ev);
      S->inflight.pop_front();
      continue;
    }
    if (q != cudaErrorNotReady) {
      ahx::set_last_error(std::string("live solver: server: batched chunk failed: ") + cudaGetErrorString(q));
      return AHX_EDEVICE;
    }
    if ((e = poll_reads(S)) != AHX_OK) return e;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (S->stop) return AHX_OK;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  return poll_reads(S);
}

void worker_main(ahx_server* S) {
  cudaSetDevice(S->dev);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->mu);
      const bool busy = !S->incoming.empty() || !S->pending.empty() || !S->active.empty() || !S->draining.empty();
      if ((!busy || S->lost) && !S->stop) S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
      if (S->stop) break;
      if (S->lost) continue;   // nothing more is scheduled; destroy releases the slots
      while (!S->incoming.empty()) {
        S->pending.push_back(S->incoming.front());
        S->incoming.pop_front();
      }
    }
    const ahx_status e = schedule(S);
    publish(S);
    if (e != AHX_OK) {
      go_lost(S, e == AHX_ENOMEM ? AHX_ENOMEM : AHX_EDEVICE, "live solver: server stopped: " + last_msg());
    } else if (!S->draining.empty() && S->active.empty()) {
      std::this_thread::sleep_for(std::chrono::microseconds(100));   // read-backs in flight, nothing to step
    }
  }
}

ahx_status fail(ahx_status st, const std::string& m) {
  ahx::set_last_error(m);
  return st;
}

}  // namespace

extern "C" {

ahx_status ahx_server_create(const ahx_server_config* cfg, ahx_server** out) {
  if (!cfg || !out) return fail(AHX_EINVAL, "live solver: null argument");
  *out = nullptr;
  if (cfg->precision < AHX_FP32 || cfg->precision > AHX_FP16_SR)
    return fail(AHX_EINVAL, "live solver: unknown precision");
  if (cfg->arith != AHX_ARITH_EXACT && cfg->arith != AHX_ARITH_FAST)
    return fail(AHX_EINVAL, "live solver: unknown arithmetic variant");
  if (cfg->batch_mode != 0 && cfg->batch_mode != 1) return fail(AHX_EINVAL, "live solver: bad batch mode");
  int dev = cfg->device_ordinal;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(AHX_EDEVICE, "live solver: no CUDA device");
  if (cudaSetDevice(dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(AHX_EDEVICE, "live solver: cannot use CUDA device " + std::to_string(dev));
  }
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return fail(AHX_EDEVICE, "live solver: cannot query device memory");
  }
  ahx_server* S = new ahx_server;
  S->cfg = *cfg;
  S->dev = dev;
  if (S->cfg.chunk <= 0) S->cfg.chunk = 256;
  if (S->cfg.max_cells <= 0) S->cfg.max_cells = 24000000;
  if (S->cfg.depth <= 0) S->cfg.depth = 2;
  S->budget = S->cfg.hbm_budget_bytes ? S->cfg.hbm_budget_bytes : (uint64_t)(0.8 * (double)free_b);
  S->cfg.hbm_budget_bytes = S->budget;
  S->st.hbm_budget_bytes = S->budget;
  S->t0 = Clock::now();
  S->worker = std::thread(worker_main, S);
  *out = S;
  return AHX_OK;
}

ahx_status ahx_server_submit(ahx_server* S, const ahx_request* q, uint64_t* ticket) {
  if (!S || !q || !ticket) return fail(AHX_EINVAL, "live solver: null argument");
  if (q->nx < 2 || q->ny < 2 || q->nz < 2) return fail(AHX_EINVAL, "live solver: grid must be at least 2 x 2 x 2");
  if (q->steps < 0) return fail(AHX_EINVAL, "live solver: negative step count");
  if (!q->params || q->params_bytes != 64 + 16 * (size_t)q->nz)
    return fail(AHX_EINVAL, "live solver: parameter block must be 64 + 16 * nz bytes");
  if (!q->colv || !q->ktop) return fail(AHX_EINVAL, "live solver: null column records or ktop plane");
  if (q->nzv < 0 || q->nzv > q->nz) return fail(AHX_EINVAL, "live solver: nzv out of range");
  const size_t NXY = (size_t)q->nx * q->ny;
  for (size_t c = 0; c < NXY; ++c)
    if (q->ktop[c] > ahx::kMaxLevel || q->colv[4 * c] > ahx::kMaxLevel || q->colv[4 * c + 1] != q->ktop[c])
      return fail(AHX_EINVAL, "live solver: column records and ktop plane disagree or exceed the level range");
  auto r = std::make_shared<Req>();
  r->tag = q->user_tag;
  r->nx = q->nx;
  r->ny = q->ny;
  r->nz = q->nz;
  r->steps = q->steps;
  r->nzv = q->nzv;
  r->want_vol = q->want_vol ? 1 : 0;
  r->want_wind = q->want_wind ? 1 : 0;
  r->conv = q->conv;
  r->volscale = q->volscale;
  r->params.assign(static_cast<const unsigned char*>(q->params),
                   static_cast<const unsigned char*>(q->params) + q->params_bytes);
  r->colv.assign(q->colv, q->colv + 4 * NXY);
  r->ktop.assign(q->ktop, q->ktop + NXY);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->destroyed) return fail(AHX_EDESTROYED, "live solver: server destroyed");
  if (S->lost) return fail(AHX_EDEVICE, S->lost_msg);
  r->ticket = ++S->next_ticket;
  r->t_submit = seconds_since(S->t0);
  S->open[r->ticket] = r;
  S->incoming.push_back(r);
  ++S->st.submitted;
  *ticket = r->ticket;
  S->cv_work.notify_one();
  return AHX_OK;
}

ahx_status ahx_server_poll(ahx_server* S, uint64_t ticket, int timeout_ms, ahx_server_result* info, float* surf,
                           float* u, float* v, uint8_t* vol) {
  if (!S) return fail(AHX_EINVAL, "live solver: null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->open.find(ticket);
  if (it == S->open.end()) return fail(AHX_EINVAL, "live solver: unknown request ticket");
  std::shared_ptr<Req> r = it->second;
  auto ready = [&] { return r->done || S->destroyed; };
  if (timeout_ms < 0) S->cv_done.wait(lk, ready);
  else S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
  if (!r->done) {
    if (S->destroyed) return fail(AHX_EDESTROYED, "live solver: server destroyed");
    return fail(AHX_ETIMEOUT, "live solver: request not finished yet");
  }
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->ticket = r->ticket;
    info->user_tag = r->tag;
    info->nx = r->nx;
    info->ny = r->ny;
    info->nz = r->nz;
    info->nzv = r->nzv;
    info->steps = r->steps;
    info->status = r->status;
    info->submitted_s = r->t_submit;
    info->admitted_s = r->t_admit;
    info->done_s = r->t_done;
    info->theta_max = r->theta_max;
    info->want_vol = r->want_vol;
    info->want_wind = r->want_wind;
  }
  const ahx_status status = (ahx_status)r->status;
  if (status == AHX_OK) {
    const size_t NXY = (size_t)r->nx * r->ny;
    if (surf) std::memcpy(surf, r->surf.data(), NXY * 4);
    if (r->want_wind) {
      if (u) std::memcpy(u, r->surf.data() + NXY, NXY * 4);
      if (v) std::memcpy(v, r->surf.data() + 2 * NXY, NXY * 4);
    }
    if (vol && r->want_vol) std::memcpy(vol, r->vol.data(), r->vol.size());
  }
  const std::string err = r->err;
  S->open.erase(it);
  if (status != AHX_OK) return fail(status, err.empty() ? "live solver: request failed" : err);
  return AHX_OK;
}

ahx_status ahx_server_stats(ahx_server* S, ahx_server_stats_out* out) {
  if (!S || !out) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->st;
  out->elapsed_s = seconds_since(S->t0);
  return AHX_OK;
}

ahx_status ahx_server_destroy(ahx_server* S) {
  if (!S) return fail(AHX_EINVAL, "live solver: null server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->destroyed) return AHX_OK;
    S->stop = true;
    S->cv_work.notify_all();
  }
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->dev);
  if (S->batch) {
    ahx_batch_sync(S->batch, -1);
    ahx_batch_destroy(S->batch);
    S->batch = nullptr;
  }
  for (Slot* sl : S->slots) {
    ahx_destroy(sl->h);
    delete sl;
  }
  for (const Chunk& c : S->inflight) cudaEventDestroy(c.ev);
  for (cudaEvent_t ev : S->spare_events) cudaEventDestroy(ev);
  S->inflight.clear();
  S->spare_events.clear();
  S->slots.clear();
  S->active.clear();
  S->draining.clear();
  S->idle.clear();
  std::lock_guard<std::mutex> lk(S->mu);
  S->destroyed = true;
  for (auto& kv : S->open)
    if (!kv.second->done) finish_locked(S, kv.second, AHX_EDESTROYED, "live solver: server destroyed");
  S->cv_done.notify_all();
  // the server object itself stays (a small tombstone), so later calls on it return AHX_EDESTROYED
  return AHX_OK;
}

}  // extern "C"
