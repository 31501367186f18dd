// Batched stepping (include/ahx.h, ahx_batch_*): many independent domains of one device stepped by one persistent
// launch per step, replayed from a CUDA graph.
//
// The reference steps one domain per device (solver.js:401-427); a batch groups existing handles so ensembles and
// the serving loop pay one launch per step for all of them and the persistent blocks balance unequal grids. Each
// member keeps its own buffers, parameter block, columns and ktop; the batch holds, per step parity, a device table
// of the members' views and a member-major tile list. Members stay usable on their own: before a batched launch the
// batch stream waits for every member's stream, and afterwards every member's stream waits for the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ahx.h"
#include "handle.h"
#include "launch.h"

using namespace ahx;

struct ahx_batch {
  std::mutex mu;
  bool destroyed = false, lost = false;
  std::string lost_msg;
  int dev = 0, precision = 0, arith = 0, minb = 5, grid = 0, max_nz = 0;
  std::vector<ahx_handle*> members;
  std::vector<int> zslab;          // tile depth per member
  std::vector<int> base_parity;    // each member's parity when the view table was written
  int phase = 0;                   // steps since then, mod 2
  int ntiles = 0;
  int64_t cells = 0;
  cudaStream_t s = nullptr;
  DomainView* d_views = nullptr;   // [2][members]: set p reads buffer base_parity ^ p
  BatchTile* d_tiles = nullptr;
  int* d_zslab = nullptr;
  DomainView* h_views = nullptr;   // pinned staging of the table
  cudaEvent_t ev_done = nullptr;
  std::vector<cudaEvent_t> ev_member;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // two steps starting at phase 0 / 1
  bool use_graph = true;
};

namespace {

ahx_status batch_fail(ahx_batch* b, cudaError_t e, const char* what) {
  const std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (b) {
    b->lost = true;
    b->lost_msg = m;
    for (ahx_handle* h : b->members) h->batch_lost.store(1);   // callers may hold member locks
  }
  return fail(AHX_EDEVICE, "live solver: CUDA error (" + m + ")");
}

#define AHX_BCUDA(b, call)                                    \
  do {                                                        \
    cudaError_t e__ = (call);                                 \
    if (e__ != cudaSuccess) return batch_fail(b, e__, #call); \
  } while (0)

ahx_status check_batch(ahx_batch* b) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  if (b->destroyed) return fail(AHX_EDESTROYED, "live solver: batch destroyed");
  if (b->lost) return fail(AHX_EDEVICE, "live solver: CUDA device lost (" + b->lost_msg + ")");
  return AHX_OK;
}

cudaError_t launch(const ahx_batch* b, int set, cudaStream_t s) {
  BatchLaunch L;
  L.precision = b->precision;
  L.minb = b->minb;
  L.max_nz = b->max_nz;
  L.grid = b->grid;
  L.ntiles = b->ntiles;
  L.views = b->d_views + (size_t)set * b->members.size();
  L.tiles = b->d_tiles;
  L.zslabs = b->d_zslab;
  return b->arith == AHX_ARITH_FAST ? fast::launch_batch(L, s, nullptr) : exact::launch_batch(L, s, nullptr);
}

int occupancy(const ahx_batch* b) {
  BatchLaunch L{};
  L.precision = b->precision;
  L.minb = b->minb;
  L.max_nz = b->max_nz;
  int occ = 0;
  const cudaError_t e =
      b->arith == AHX_ARITH_FAST ? fast::launch_batch(L, nullptr, &occ) : exact::launch_batch(L, nullptr, &occ);
  return e == cudaSuccess ? occ : 0;
}

// write both view sets from the members' current parities (members locked by the caller); stream-ordered upload
ahx_status write_views(ahx_batch* b) {
  const size_t M = b->members.size();
  AHX_BCUDA(b, cudaStreamSynchronize(b->s));   // the staging buffer may still feed an earlier upload
  for (size_t m = 0; m < M; ++m) {
    ahx_handle* h = b->members[m];
    b->base_parity[m] = h->parity;
    b->h_views[m] = view_at(h, h->parity);
    b->h_views[M + m] = view_at(h, h->parity ^ 1);
  }
  b->phase = 0;
  AHX_BCUDA(b, cudaMemcpyAsync(b->d_views, b->h_views, 2 * M * sizeof(DomainView), cudaMemcpyHostToDevice, b->s));
  return AHX_OK;
}

// capture the two-step graph starting at `phase` (sets phase, phase ^ 1)
ahx_status capture(ahx_batch* b, int phase) {
  cudaGraph_t g = nullptr;
  AHX_BCUDA(b, cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e1 = launch(b, phase, b->s);
  cudaError_t e2 = e1 == cudaSuccess ? launch(b, phase ^ 1, b->s) : e1;
  cudaError_t e3 = cudaStreamEndCapture(b->s, &g);
  if (e2 != cudaSuccess || e3 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return batch_fail(b, e2 != cudaSuccess ? e2 : e3, "batch graph capture");
  }
  const cudaError_t e4 = cudaGraphInstantiate(&b->graph[phase], g, 0);
  cudaGraphDestroy(g);
  if (e4 != cudaSuccess) return batch_fail(b, e4, "cudaGraphInstantiate");
  return AHX_OK;
}

void release(ahx_batch* b) {
  cudaSetDevice(b->dev);
  if (b->s) cudaStreamSynchronize(b->s);
  for (auto& g : b->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  if (b->d_views) cudaFree(b->d_views);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_zslab) cudaFree(b->d_zslab);
  if (b->h_views) cudaFreeHost(b->h_views);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  for (cudaEvent_t e : b->ev_member)
    if (e) cudaEventDestroy(e);
  if (b->s) cudaStreamDestroy(b->s);
  b->d_views = nullptr;
  b->d_tiles = nullptr;
  b->d_zslab = nullptr;
  b->h_views = nullptr;
  b->ev_done = nullptr;
  b->ev_member.clear();
  b->s = nullptr;
}

}  // namespace

extern "C" {

ahx_status ahx_batch_create(ahx_handle* const* members, int count, ahx_batch** out) {
  if (!members || !out || count < 1) return fail(AHX_EINVAL, "live solver: batch needs at least one member");
  *out = nullptr;
  if (count > 65535) return fail(AHX_EINVAL, "live solver: at most 65535 members per batch");
  for (int m = 0; m < count; ++m)
    for (int k = 0; k < m; ++k)
      if (members[k] == members[m]) return fail(AHX_EINVAL, "live solver: a handle appears twice in the batch");
  ahx_batch* b = new ahx_batch();
  std::vector<std::unique_lock<std::mutex>> locks;
  for (int m = 0; m < count; ++m) {
    ahx_handle* h = members[m];
    if (ahx_status st = check(h)) {
      delete b;
      return st;
    }
    locks.emplace_back(h->mu);
    if (m == 0) {
      b->dev = h->dev;
      b->precision = h->dims.precision;
      b->arith = h->dims.arith;
    } else if (h->dev != b->dev || h->dims.precision != b->precision || h->dims.arith != b->arith) {
      delete b;
      return fail(AHX_EINVAL, "live solver: batch members must share device, precision and arithmetic");
    }
    b->members.push_back(h);
  }
  // tiles: 32 x 4 columns x z-slab levels per member, member-major
  std::vector<BatchTile> tiles;
  std::vector<int> minbs;
  for (int m = 0; m < count; ++m) {
    const ahx_handle* h = members[m];
    const int nz = h->dims.nz;
    const int zs = h->zslab > 0 ? std::min(h->zslab, nz) : std::min(nz, 16);
    b->zslab.push_back(zs);
    b->max_nz = std::max(b->max_nz, nz);
    b->cells += (int64_t)h->dims.nx * h->dims.ny * nz;
    if (h->minb > 0) minbs.push_back(h->minb);
    const int gx = (h->dims.nx + 31) / 32, gy = (h->dims.ny + 3) / 4, gz = (nz + zs - 1) / zs;
    if (gx > 65535 || gy > 65535 || gz > 65535) {
      delete b;
      return fail(AHX_EINVAL, "live solver: member grid too large for a batch tile index");
    }
    for (int z = 0; z < gz; ++z)
      for (int y = 0; y < gy; ++y)
        for (int x = 0; x < gx; ++x) tiles.push_back(BatchTile{(uint16_t)m, (uint16_t)x, (uint16_t)y, (uint16_t)z});
  }
  if (tiles.size() > (size_t)INT32_MAX) {
    delete b;
    return fail(AHX_EINVAL, "live solver: too many tiles in one batch");
  }
  // register-budget variant: the members' tuned choice when they agree, else 5 (96 registers)
  if (!minbs.empty() && std::all_of(minbs.begin(), minbs.end(), [&](int v) { return v == minbs[0]; }))
    b->minb = minbs[0];
  b->ntiles = (int)tiles.size();
  b->base_parity.assign(count, 0);
  auto bail = [&](ahx_status st, const std::string& m) {
    release(b);
    delete b;
    cudaGetLastError();
    return fail(st, m);
  };
  if (cudaSetDevice(b->dev) != cudaSuccess) return bail(AHX_EDEVICE, "live solver: cannot use CUDA device");
  if (cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming) != cudaSuccess)
    return bail(AHX_EDEVICE, "live solver: batch stream creation failed");
  b->ev_member.assign(count, nullptr);
  for (auto& e : b->ev_member)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return bail(AHX_EDEVICE, "live solver: batch event creation failed");
  if (cudaMalloc(&b->d_views, 2 * count * sizeof(DomainView)) != cudaSuccess ||
      cudaMalloc(&b->d_tiles, tiles.size() * sizeof(BatchTile)) != cudaSuccess ||
      cudaMalloc(&b->d_zslab, count * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&b->h_views, 2 * count * sizeof(DomainView)) != cudaSuccess)
    return bail(AHX_ENOMEM, "live solver: batch table allocation failed");
  if (cudaMemcpy(b->d_tiles, tiles.data(), tiles.size() * sizeof(BatchTile), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_zslab, b->zslab.data(), count * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(AHX_EDEVICE, "live solver: batch table upload failed");
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->dev);
  const int occ = occupancy(b);
  if (occ < 1 || nsm < 1) return bail(AHX_EDEVICE, "live solver: batched step kernel cannot be resident");
  b->grid = std::min(b->ntiles, nsm * occ);
  if (ahx_status st = write_views(b)) {
    release(b);
    delete b;
    return st;
  }
  if (cudaStreamSynchronize(b->s) != cudaSuccess) return bail(AHX_EDEVICE, "live solver: batch set-up failed");
  for (ahx_handle* h : b->members) ++h->batch_refs;
  *out = b;
  return AHX_OK;
}

ahx_status ahx_batch_set_variant(ahx_batch* b, int minb, int use_graph) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (ahx_status st = check_batch(b)) return st;
  if (minb != 0 && minb != 4 && minb != 5 && minb != 6)
    return fail(AHX_EINVAL, "live solver: batch register-budget variant must be 4, 5 or 6 (0 = keep)");
  AHX_BCUDA(b, cudaSetDevice(b->dev));
  AHX_BCUDA(b, cudaStreamSynchronize(b->s));
  if (minb != 0 && minb != b->minb) {
    b->minb = minb;
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->dev);
    const int occ = occupancy(b);
    if (occ < 1) return fail(AHX_EDEVICE, "live solver: batched step kernel cannot be resident");
    b->grid = std::min(b->ntiles, nsm * occ);
    for (auto& g : b->graph)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
  }
  b->use_graph = use_graph != 0;
  return AHX_OK;
}

ahx_status ahx_batch_step(ahx_batch* b, int n) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (ahx_status st = check_batch(b)) return st;
  if (n < 0) return fail(AHX_EINVAL, "live solver: bad step count");
  if (n == 0) return AHX_OK;
  AHX_BCUDA(b, cudaSetDevice(b->dev));
  const size_t M = b->members.size();
  std::vector<std::unique_lock<std::mutex>> locks;
  locks.reserve(M);
  bool moved = false;
  for (size_t m = 0; m < M; ++m) {
    ahx_handle* h = b->members[m];
    locks.emplace_back(h->mu);
    if (ahx_status st = check(h)) return st;
    if (h->budget_on) return fail(AHX_EINVAL, "live solver: batched steps do not accumulate budgets (member " +
                                                  std::to_string(m) + " has them enabled)");
    if (h->parity != (b->base_parity[m] ^ b->phase)) moved = true;   // stepped on its own since
  }
  if (moved)
    if (ahx_status st = write_views(b)) return st;
  // the batch runs after everything already queued on each member's stream
  for (size_t m = 0; m < M; ++m) {
    AHX_BCUDA(b, cudaEventRecord(b->ev_member[m], b->members[m]->s_step));
    AHX_BCUDA(b, cudaStreamWaitEvent(b->s, b->ev_member[m], 0));
  }
  int left = n;
  if (b->use_graph) {
    if (!b->graph[b->phase])
      if (ahx_status st = capture(b, b->phase)) return st;
    for (; left >= 2; left -= 2) AHX_BCUDA(b, cudaGraphLaunch(b->graph[b->phase], b->s));
  }
  for (; left > 0; --left) {
    AHX_BCUDA(b, launch(b, b->phase, b->s));
    b->phase ^= 1;
  }
  AHX_BCUDA(b, cudaEventRecord(b->ev_done, b->s));
  for (size_t m = 0; m < M; ++m) {
    ahx_handle* h = b->members[m];
    AHX_BCUDA(b, cudaStreamWaitEvent(h->s_step, b->ev_done, 0));
    h->parity ^= (n & 1);
    h->steps += n;
  }
  return AHX_OK;
}

ahx_status ahx_batch_sync(ahx_batch* b, int timeout_ms) {
  cudaEvent_t ev = nullptr;
  {
    if (!b) return fail(AHX_EINVAL, "live solver: null batch");
    std::lock_guard<std::mutex> lk(b->mu);
    if (ahx_status st = check_batch(b)) return st;
    AHX_BCUDA(b, cudaSetDevice(b->dev));
    AHX_BCUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    AHX_BCUDA(b, cudaEventRecord(ev, b->s));
  }
  const ahx_status st = wait_event(nullptr, ev, timeout_ms);
  cudaEventDestroy(ev);
  if (st == AHX_EDEVICE) {
    std::lock_guard<std::mutex> lk(b->mu);
    b->lost = true;
    b->lost_msg = "batched step failed";
  }
  return st;
}

ahx_status ahx_batch_time_steps(ahx_batch* b, int n, int timeout_ms, float* ms) {
  if (!b || !ms) return fail(AHX_EINVAL, "live solver: null argument");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    if (ahx_status st = check_batch(b)) return st;
    AHX_BCUDA(b, cudaSetDevice(b->dev));
    AHX_BCUDA(b, cudaEventCreate(&e0));
    AHX_BCUDA(b, cudaEventCreate(&e1));
  }
  // e0 after the members' queued work: record it once the batch stream waits on them (a zero-step batch call)
  ahx_status st = AHX_OK;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    for (size_t m = 0; m < b->members.size() && st == AHX_OK; ++m) {
      std::lock_guard<std::mutex> lm(b->members[m]->mu);
      cudaError_t e = cudaEventRecord(b->ev_member[m], b->members[m]->s_step);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->s, b->ev_member[m], 0);
      if (e != cudaSuccess) st = batch_fail(b, e, "batch ordering");
    }
    if (st == AHX_OK) {
      const cudaError_t e = cudaEventRecord(e0, b->s);
      if (e != cudaSuccess) st = batch_fail(b, e, "cudaEventRecord");
    }
  }
  if (st == AHX_OK) st = ahx_batch_step(b, n);
  if (st == AHX_OK) {
    std::lock_guard<std::mutex> lk(b->mu);
    const cudaError_t e = cudaEventRecord(e1, b->s);
    if (e != cudaSuccess) st = batch_fail(b, e, "cudaEventRecord");
  }
  if (st == AHX_OK) st = wait_event(nullptr, e1, timeout_ms);
  if (st == AHX_OK) {
    const cudaError_t e = cudaEventElapsedTime(ms, e0, e1);
    if (e != cudaSuccess) st = batch_fail(b, e, "cudaEventElapsedTime");
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

ahx_status ahx_batch_get_info(ahx_batch* b, ahx_batch_info_out* out) {
  if (!b || !out) return fail(AHX_EINVAL, "live solver: null argument");
  std::lock_guard<std::mutex> lk(b->mu);
  std::memset(out, 0, sizeof(*out));
  out->members = (int)b->members.size();
  out->tiles = b->ntiles;
  out->grid = b->grid;
  out->minb = b->minb;
  out->use_graph = b->use_graph ? 1 : 0;
  out->cells = b->cells;
  return check_batch(b);
}

ahx_status ahx_batch_destroy(ahx_batch* b) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (b->destroyed) return AHX_OK;
  b->destroyed = true;
  release(b);
  for (ahx_handle* h : b->members) {
    std::lock_guard<std::mutex> lm(h->mu);
    --h->batch_refs;
  }
  // the batch object stays allocated so later calls report "batch destroyed"
  return AHX_OK;
}

}  // extern "C"
