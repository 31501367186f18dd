// Batched stepping (include/ahx.h, ahx_batch_*): many independent domains of one device stepped by one persistent
// launch per step, replayed from a CUDA graph.
//
// The reference steps one domain per device (solver.js:401-427); a batch groups existing handles so ensembles and
// the serving loop pay one launch per step for all of them and the persistent blocks balance unequal grids. Each
// member keeps its own buffers, parameter block, columns and ktop. The batch owns device tables sized for a capacity
// (members, tiles, levels): per step parity a table of the members' views, a member-major tile list, the tile depth
// per member and the tile count, which the kernel reads from device memory. The launch shape (grid = resident blocks
// on every SM, shared memory for the capacity's levels) therefore does not depend on the membership, so the captured
// two-step graph stays valid and a membership change is a stream-ordered table upload: no synchronisation, no
// allocation unless the capacity grows. Members stay usable on their own: before batched launches the batch stream
// waits for every member's stream, and afterwards every member's stream waits for the batch.
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

namespace {

// pinned host images of one table upload; two alternate so an upload never waits for the one before it
struct Staging {
  DomainView* views = nullptr;   // [2][cap_members]
  BatchTile* tiles = nullptr;    // [cap_tiles]
  int* zslab = nullptr;          // [cap_members]
  int* ntiles = nullptr;         // [1]
  cudaEvent_t ev = nullptr;      // recorded after the copies that read this image
  bool used = false;
};

}  // namespace

struct ahx_batch {
  std::mutex mu;
  bool destroyed = false, lost = false;
  std::string lost_msg;
  int dev = 0, precision = 0, arith = 0, minb = 4, nsm = 0, occ = 0, grid = 0;
  bool pairs = false;              // paired levels on packed f32x2 arithmetic (FMA build)
  int cap_members = 0, cap_nz = 0;
  int64_t cap_tiles = 0;
  std::vector<ahx_handle*> members;
  std::vector<int> zslab;          // tile depth per member
  std::vector<int> base_parity;    // each member's parity when the view table was written
  int phase = 0;                   // steps since then, mod 2
  int zs_policy = 8;               // tile-depth policy (build_plan)
  int ntiles = 0;
  int64_t cells = 0;
  cudaStream_t s = nullptr;
  DomainView* d_views = nullptr;   // [2][cap_members]: set p makes member m read buffer base_parity[m] ^ p
  BatchTile* d_tiles = nullptr;
  int* d_zslab = nullptr;
  int* d_ntiles = nullptr;
  int* d_sched = nullptr;          // tile counter and finished-block counter of the running launch
  Staging stage[2];
  int stage_next = 0;
  cudaEvent_t ev_done = nullptr;
  std::vector<cudaEvent_t> ev_member;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // two steps starting at phase 0 / 1
  bool use_graph = true;
  // branch mode: each member's own solo step kernels on parallel graph branches (side streams during capture)
  bool branches = false;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  cudaGraphExec_t bgraph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [steps - 1][phase]
  uint64_t bkey[2][2] = {{0, 0}, {0, 0}};
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

BatchLaunch launch_args(const ahx_batch* b, int set) {
  BatchLaunch L{};
  L.precision = b->precision;
  L.minb = b->minb;
  L.pairs = b->pairs;
  L.max_nz = b->cap_nz;
  L.grid = b->grid;
  L.views = b->d_views + (size_t)set * b->cap_members;
  L.tiles = b->d_tiles;
  L.zslabs = b->d_zslab;
  L.ntiles = b->d_ntiles;
  L.sched = b->d_sched;
  return L;
}

cudaError_t launch(const ahx_batch* b, int set, cudaStream_t s) {
  const BatchLaunch L = launch_args(b, set);
  return b->arith == AHX_ARITH_FAST ? fast::launch_batch(L, s, nullptr) : exact::launch_batch(L, s, nullptr);
}

// resident blocks per SM of the batched kernel for the current variant and level capacity
int occupancy(const ahx_batch* b) {
  const BatchLaunch L = launch_args(b, 0);
  int occ = 0;
  const cudaError_t e =
      b->arith == AHX_ARITH_FAST ? fast::launch_batch(L, nullptr, &occ) : exact::launch_batch(L, nullptr, &occ);
  return e == cudaSuccess ? occ : 0;
}

void drop_graphs(ahx_batch* b) {
  for (auto& g : b->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  for (auto& row : b->bgraph)
    for (auto& g : row)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
}

constexpr int kMaxBranches = 32;   // concurrent branches of a branch-mode graph (members share them round-robin)

// what a branch-mode graph depends on: the members, the parities they read at phase 0 and their launch shapes
uint64_t branch_key(const ahx_batch* b) {
  uint64_t k = 1469598103934665603ull;
  for (size_t m = 0; m < b->members.size(); ++m) {
    const ahx_handle* h = b->members[m];
    for (uint64_t x : {(uint64_t)(uintptr_t)h, (uint64_t)b->base_parity[m], solo_launch_key(h)})
      k = (k ^ x) * 1099511628211ull;
  }
  return k | 1;
}

// capture `nsteps` (1 or 2) steps starting at `phase` as one graph: member m's solo kernels, in step order, on branch
// m mod K, the K branches forked from and joined back to the batch stream
ahx_status capture_branches(ahx_batch* b, int phase, int nsteps) {
  const size_t M = b->members.size();
  const size_t K = std::min<size_t>(M, kMaxBranches);
  if (!b->fork_ev) AHX_BCUDA(b, cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
  while (b->side.size() < K) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    AHX_BCUDA(b, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->side.push_back(s);
    AHX_BCUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->side_ev.push_back(e);
  }
  cudaGraphExec_t& slot = b->bgraph[nsteps - 1][phase];
  if (slot) cudaGraphExecDestroy(slot), slot = nullptr;
  cudaGraph_t g = nullptr;
  AHX_BCUDA(b, cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaEventRecord(b->fork_ev, b->s);
  for (size_t k = 0; k < K && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(b->side[k], b->fork_ev, 0);
  for (size_t m = 0; m < M && e == cudaSuccess; ++m)
    for (int s = 0; s < nsteps && e == cudaSuccess; ++s)
      e = solo_step(b->members[m], b->base_parity[m] ^ phase ^ s, b->side[m % K]);
  for (size_t k = 0; k < K && e == cudaSuccess; ++k) {
    e = cudaEventRecord(b->side_ev[k], b->side[k]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->s, b->side_ev[k], 0);
  }
  const cudaError_t e2 = cudaStreamEndCapture(b->s, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return batch_fail(b, e != cudaSuccess ? e : e2, "batch branch graph capture");
  }
  const cudaError_t e3 = cudaGraphInstantiate(&slot, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) {
    slot = nullptr;
    return batch_fail(b, e3, "cudaGraphInstantiate");
  }
  b->bkey[nsteps - 1][phase] = branch_key(b);
  return AHX_OK;
}

// the branch-mode graph of `nsteps` steps from the current phase, captured again when its key is stale
ahx_status branch_graph(ahx_batch* b, int nsteps, cudaGraphExec_t* out) {
  if (!b->bgraph[nsteps - 1][b->phase] || b->bkey[nsteps - 1][b->phase] != branch_key(b))
    if (ahx_status st = capture_branches(b, b->phase, nsteps)) return st;
  *out = b->bgraph[nsteps - 1][b->phase];
  return AHX_OK;
}

ahx_status resize_grid(ahx_batch* b) {
  b->occ = occupancy(b);
  if (b->occ < 1 || b->nsm < 1) return fail(AHX_EDEVICE, "live solver: batched step kernel cannot be resident");
  b->grid = b->nsm * b->occ;
  drop_graphs(b);
  return AHX_OK;
}

void free_tables(ahx_batch* b) {
  if (b->d_views) cudaFree(b->d_views);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_zslab) cudaFree(b->d_zslab);
  if (b->d_ntiles) cudaFree(b->d_ntiles);
  if (b->d_sched) cudaFree(b->d_sched);
  b->d_sched = nullptr;
  b->d_views = nullptr;
  b->d_tiles = nullptr;
  b->d_zslab = nullptr;
  b->d_ntiles = nullptr;
  for (Staging& g : b->stage) {
    if (g.ev && g.used) cudaEventSynchronize(g.ev);
    if (g.views) cudaFreeHost(g.views);
    if (g.tiles) cudaFreeHost(g.tiles);
    if (g.zslab) cudaFreeHost(g.zslab);
    if (g.ntiles) cudaFreeHost(g.ntiles);
    g.views = nullptr;
    g.tiles = nullptr;
    g.zslab = g.ntiles = nullptr;
    g.used = false;
  }
}

// (re)allocate the tables for at least these capacities (with headroom); the batch stream is drained first
ahx_status ensure_capacity(ahx_batch* b, int members, int64_t tiles, int nz) {
  if (members <= b->cap_members && tiles <= b->cap_tiles && nz <= b->cap_nz && b->d_views) return AHX_OK;
  AHX_BCUDA(b, cudaStreamSynchronize(b->s));
  free_tables(b);
  const int cm = std::max({members, b->cap_members, 16});
  const int64_t ct = std::max<int64_t>({tiles + tiles / 2, b->cap_tiles, 4096});
  const int cz = std::max({nz, b->cap_nz, 64});
  if (ct > (int64_t)INT32_MAX) return fail(AHX_EINVAL, "live solver: too many tiles in one batch");
  b->cap_members = 0;
  b->cap_tiles = 0;
  if (cudaMalloc(&b->d_views, 2 * (size_t)cm * sizeof(DomainView)) != cudaSuccess ||
      cudaMalloc(&b->d_tiles, (size_t)ct * sizeof(BatchTile)) != cudaSuccess ||
      cudaMalloc(&b->d_zslab, (size_t)cm * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_ntiles, sizeof(int)) != cudaSuccess || cudaMalloc(&b->d_sched, 2 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    free_tables(b);
    return fail(AHX_ENOMEM, "live solver: batch table allocation failed");
  }
  AHX_BCUDA(b, cudaMemsetAsync(b->d_sched, 0, 2 * sizeof(int), b->s));
  for (Staging& g : b->stage) {
    if (cudaMallocHost(&g.views, 2 * (size_t)cm * sizeof(DomainView)) != cudaSuccess ||
        cudaMallocHost(&g.tiles, (size_t)ct * sizeof(BatchTile)) != cudaSuccess ||
        cudaMallocHost(&g.zslab, (size_t)cm * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&g.ntiles, sizeof(int)) != cudaSuccess ||
        (!g.ev && cudaEventCreateWithFlags(&g.ev, cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      free_tables(b);
      return fail(AHX_ENOMEM, "live solver: batch staging allocation failed");
    }
  }
  while ((int)b->ev_member.size() < cm) {
    cudaEvent_t e = nullptr;
    AHX_BCUDA(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_member.push_back(e);
  }
  b->cap_members = cm;
  b->cap_tiles = ct;
  const bool nz_grew = cz != b->cap_nz;
  b->cap_nz = cz;
  if (nz_grew || b->grid == 0)
    if (ahx_status st = resize_grid(b)) return st;
  drop_graphs(b);   // the graphs hold the old table addresses
  return AHX_OK;
}

// tiles of a member domain in x and y (32 x 4 columns per tile): the main tiles, then the strip tiles of its column
// split (a batch member is a whole domain)
struct TileGrid {
  int gx, gy;
};
TileGrid tile_grid(const ahx_handle* h) {
  const int nx = h->dims.nx, ny = h->dims.ny;
  const StepSplit SP = step_split(nx, 0, ny, 0, 0, ny, strip_width(h->esize, nx));
  return TileGrid{SP.gx, main_blocks_y(ny, 0, 4) + strip_blocks_y(SP, 4)};
}

// Tile plan for depth policy `policy` (> 0: that depth for every member, clipped to its nz, 8 levels by default;
// -1: whole columns when that still gives at least 4 tiles per persistent block, else each member's own z-slab or
// 16 levels).
ahx_status build_plan(const std::vector<ahx_handle*>& mem, int policy, int grid, std::vector<BatchTile>& tiles,
                      std::vector<int>& zslab) {
  auto own = [](const ahx_handle* h) {
    return h->zslab > 0 ? std::min(h->zslab, h->dims.nz) : std::min(h->dims.nz, 16);
  };
  int64_t whole_tiles = 0;
  for (const ahx_handle* h : mem) whole_tiles += (int64_t)tile_grid(h).gx * tile_grid(h).gy;
  const bool whole = policy < 0 && whole_tiles >= 4 * (int64_t)std::max(grid, 1);
  tiles.clear();
  zslab.clear();
  for (size_t m = 0; m < mem.size(); ++m) {
    const ahx_handle* h = mem[m];
    const int nz = h->dims.nz;
    const int zs = policy > 0 ? std::min(policy, nz) : (whole ? nz : own(h));
    zslab.push_back(zs);
    const TileGrid tg = tile_grid(h);
    const int gx = tg.gx, gy = tg.gy, gz = (nz + zs - 1) / zs;
    if (gx > 65535 || gy > 65535 || gz > 65535)
      return fail(AHX_EINVAL, "live solver: member grid too large for a batch tile index");
    if (tiles.size() + (size_t)gx * gy * gz > (size_t)INT32_MAX / 2)
      return fail(AHX_EINVAL, "live solver: too many tiles in one batch");
    for (int z = 0; z < gz; ++z)
      for (int y = 0; y < gy; ++y)
        for (int x = 0; x < gx; ++x) tiles.push_back(BatchTile{(uint16_t)m, (uint16_t)x, (uint16_t)y, (uint16_t)z});
  }
  return AHX_OK;
}

// stream-ordered upload of the tables for `mem` (locked by the caller) from their current parities
ahx_status upload(ahx_batch* b, const std::vector<ahx_handle*>& mem, const std::vector<BatchTile>& tiles,
                  const std::vector<int>& zslab) {
  Staging& g = b->stage[b->stage_next];
  b->stage_next ^= 1;
  if (g.used) AHX_BCUDA(b, cudaEventSynchronize(g.ev));   // the copies of two uploads ago have read this image
  const size_t M = mem.size(), C = (size_t)b->cap_members;
  for (size_t m = 0; m < M; ++m) {
    ahx_handle* h = mem[m];
    g.views[m] = view_at(h, h->parity);
    g.views[C + m] = view_at(h, h->parity ^ 1);
    // tiles of this member in one step (its blocks report done to its step counter)
    const uint32_t nt = (uint32_t)tile_grid(h).gx * (uint32_t)tile_grid(h).gy *
                        (uint32_t)((h->dims.nz + zslab[m] - 1) / zslab[m]);
    g.views[m].tick_blocks = g.views[C + m].tick_blocks = nt;
    g.zslab[m] = zslab[m];
  }
  if (!tiles.empty()) std::memcpy(g.tiles, tiles.data(), tiles.size() * sizeof(BatchTile));
  *g.ntiles = (int)tiles.size();
  if (M) {
    AHX_BCUDA(b, cudaMemcpyAsync(b->d_views, g.views, M * sizeof(DomainView), cudaMemcpyHostToDevice, b->s));
    AHX_BCUDA(b, cudaMemcpyAsync(b->d_views + C, g.views + C, M * sizeof(DomainView), cudaMemcpyHostToDevice, b->s));
    AHX_BCUDA(b, cudaMemcpyAsync(b->d_zslab, g.zslab, M * sizeof(int), cudaMemcpyHostToDevice, b->s));
  }
  if (!tiles.empty())
    AHX_BCUDA(b, cudaMemcpyAsync(b->d_tiles, g.tiles, tiles.size() * sizeof(BatchTile), cudaMemcpyHostToDevice, b->s));
  AHX_BCUDA(b, cudaMemcpyAsync(b->d_ntiles, g.ntiles, sizeof(int), cudaMemcpyHostToDevice, b->s));
  AHX_BCUDA(b, cudaEventRecord(g.ev, b->s));
  g.used = true;
  b->base_parity.assign(M, 0);
  for (size_t m = 0; m < M; ++m) b->base_parity[m] = mem[m]->parity;
  b->phase = 0;
  b->zslab = zslab;
  b->ntiles = (int)tiles.size();
  b->cells = 0;
  for (const ahx_handle* h : mem) b->cells += (int64_t)h->dims.nx * h->dims.ny * h->dims.nz;
  return AHX_OK;
}

// plan + capacity + upload for `mem` (locked by the caller)
ahx_status install(ahx_batch* b, const std::vector<ahx_handle*>& mem) {
  std::vector<BatchTile> tiles;
  std::vector<int> zslab;
  int nz = 0;
  for (const ahx_handle* h : mem) nz = std::max(nz, h->dims.nz);
  if (ahx_status st = build_plan(mem, b->zs_policy, b->grid, tiles, zslab)) return st;
  const int grid_before = b->grid;
  if (ahx_status st = ensure_capacity(b, (int)mem.size(), (int64_t)tiles.size(), nz)) return st;
  if (b->grid != grid_before) {
    // the whole-column choice depends on the grid, which the first allocation sets
    if (ahx_status st = build_plan(mem, b->zs_policy, b->grid, tiles, zslab)) return st;
    if (ahx_status st = ensure_capacity(b, (int)mem.size(), (int64_t)tiles.size(), nz)) return st;
  }
  return upload(b, mem, tiles, zslab);
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
  drop_graphs(b);
  free_tables(b);
  for (Staging& g : b->stage)
    if (g.ev) cudaEventDestroy(g.ev), g.ev = nullptr;
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  for (cudaEvent_t e : b->ev_member)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : b->side)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->side_ev)
    if (e) cudaEventDestroy(e);
  if (b->fork_ev) cudaEventDestroy(b->fork_ev);
  b->side.clear();
  b->side_ev.clear();
  b->fork_ev = nullptr;
  if (b->s) cudaStreamDestroy(b->s);
  b->ev_done = nullptr;
  b->ev_member.clear();
  b->s = nullptr;
}

// locks a set of handles in address order (so two batches sharing members cannot deadlock)
struct MemberLocks {
  std::vector<std::unique_lock<std::mutex>> locks;
  explicit MemberLocks(std::vector<ahx_handle*> hs) {
    std::sort(hs.begin(), hs.end());
    hs.erase(std::unique(hs.begin(), hs.end()), hs.end());
    for (ahx_handle* h : hs) locks.emplace_back(h->mu);
  }
};

// membership checks for a new member list (not locked yet: only fields fixed at creation and flags are read)
ahx_status check_members(const ahx_batch* b, ahx_handle* const* members, int count) {
  if (count < 0 || (count > 0 && !members)) return fail(AHX_EINVAL, "live solver: bad member list");
  if (count > 65535) return fail(AHX_EINVAL, "live solver: at most 65535 members per batch");
  std::vector<ahx_handle*> v(members, members + count);
  std::sort(v.begin(), v.end());
  if (std::adjacent_find(v.begin(), v.end()) != v.end())
    return fail(AHX_EINVAL, "live solver: a handle appears twice in the batch");
  for (int m = 0; m < count; ++m) {
    ahx_handle* h = members[m];
    if (ahx_status st = check(h)) return st;
    if (b && (h->dev != b->dev || h->dims.precision != b->precision || h->dims.arith != b->arith))
      return fail(AHX_EINVAL, "live solver: batch members must share device, precision and arithmetic");
    if (h->nyg > 0) return fail(AHX_EINVAL, "live solver: a slab of a larger domain cannot join a batch");
  }
  return AHX_OK;
}

}  // namespace

extern "C" {

ahx_status ahx_batch_create(ahx_handle* const* members, int count, ahx_batch** out) {
  if (!members || !out || count < 1) return fail(AHX_EINVAL, "live solver: batch needs at least one member");
  *out = nullptr;
  if (ahx_status st = check_members(nullptr, members, count)) return st;
  ahx_batch* b = new ahx_batch();
  b->dev = members[0]->dev;
  b->precision = members[0]->dims.precision;
  b->arith = members[0]->dims.arith;
  if (ahx_status st = check_members(b, members, count)) {
    delete b;
    return st;
  }
  std::vector<ahx_handle*> mem(members, members + count);
  MemberLocks lock(mem);
  // register-budget variant: the members' tuned choice when they agree, else 4 (128 registers)
  std::vector<int> minbs;
  for (const ahx_handle* h : mem)
    if (h->minb > 0) minbs.push_back(h->minb);
  if (!minbs.empty() && std::all_of(minbs.begin(), minbs.end(), [&](int v) { return v == minbs[0]; }))
    b->minb = minbs[0];
  auto bail = [&](ahx_status st) {
    release(b);
    delete b;
    cudaGetLastError();
    return st;
  };
  if (cudaSetDevice(b->dev) != cudaSuccess) return bail(fail(AHX_EDEVICE, "live solver: cannot use CUDA device"));
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
  if (cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(AHX_EDEVICE, "live solver: batch stream creation failed"));
  if (ahx_status st = install(b, mem)) return bail(st);
  if (cudaStreamSynchronize(b->s) != cudaSuccess) return bail(fail(AHX_EDEVICE, "live solver: batch set-up failed"));
  b->members = mem;
  for (ahx_handle* h : mem) ++h->batch_refs;
  *out = b;
  return AHX_OK;
}

ahx_status ahx_batch_set_members(ahx_batch* b, ahx_handle* const* members, int count) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (ahx_status st = check_batch(b)) return st;
  if (ahx_status st = check_members(b, members, count)) return st;
  AHX_BCUDA(b, cudaSetDevice(b->dev));
  std::vector<ahx_handle*> mem(members, members + count);
  std::vector<ahx_handle*> all = mem;
  all.insert(all.end(), b->members.begin(), b->members.end());
  MemberLocks lock(all);
  for (ahx_handle* h : mem)
    if (ahx_status st = check(h)) return st;
  if (ahx_status st = install(b, mem)) return st;
  for (ahx_handle* h : b->members) --h->batch_refs;
  for (ahx_handle* h : mem) ++h->batch_refs;
  b->members = mem;
  return AHX_OK;
}

ahx_status ahx_batch_set_launch(ahx_batch* b, int minb, int zslab, int use_graph, int pairs) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (ahx_status st = check_batch(b)) return st;
  if (minb != 0 && minb != 4 && minb != 5 && minb != 6)
    return fail(AHX_EINVAL, "live solver: batch register-budget variant must be 4, 5 or 6 (0 = keep)");
  if (zslab < -1) return fail(AHX_EINVAL, "live solver: batch z-slab must be > 0, 0 (keep) or -1 (automatic)");
  if (use_graph < 0 || use_graph > 2) return fail(AHX_EINVAL, "live solver: use_graph must be 0, 1 or 2");
  AHX_BCUDA(b, cudaSetDevice(b->dev));
  if (pairs > 0 && (b->arith != AHX_ARITH_FAST || b->precision == AHX_FP64))
    return fail(AHX_EINVAL, "live solver: paired levels need the FMA build and f32 arithmetic");
  const bool new_pairs = pairs < 0 ? b->pairs : pairs > 0;
  if ((minb != 0 && minb != b->minb) || new_pairs != b->pairs) {
    AHX_BCUDA(b, cudaStreamSynchronize(b->s));
    const int old = b->minb;
    const bool old_pairs = b->pairs;
    if (minb != 0) b->minb = minb;
    b->pairs = new_pairs;
    if (ahx_status st = resize_grid(b)) {
      b->minb = old;
      b->pairs = old_pairs;
      resize_grid(b);
      return st;
    }
  }
  if (zslab != 0 || minb != 0 || pairs >= 0) {
    if (zslab != 0) b->zs_policy = zslab;
    MemberLocks lock(b->members);
    if (ahx_status st = install(b, b->members)) return st;
  }
  b->use_graph = use_graph != 0;
  b->branches = use_graph == 2;
  return AHX_OK;
}

ahx_status ahx_batch_step(ahx_batch* b, int n) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (ahx_status st = check_batch(b)) return st;
  if (n < 0) return fail(AHX_EINVAL, "live solver: bad step count");
  if (n == 0 || b->members.empty()) return AHX_OK;
  AHX_BCUDA(b, cudaSetDevice(b->dev));
  const size_t M = b->members.size();
  MemberLocks lock(b->members);
  bool moved = false;
  for (size_t m = 0; m < M; ++m) {
    ahx_handle* h = b->members[m];
    if (ahx_status st = check(h)) return st;
    if (h->budget_on || h->accum_on)
      return fail(AHX_EINVAL, "live solver: batched steps do not accumulate budgets or time sums (member " +
                                  std::to_string(m) + " has them enabled)");
    if (h->parity != (b->base_parity[m] ^ b->phase)) moved = true;   // stepped on its own since
  }
  if (moved)
    if (ahx_status st = install(b, b->members)) return st;
  // the batch runs after everything already queued on each member's stream
  for (size_t m = 0; m < M; ++m) {
    AHX_BCUDA(b, cudaEventRecord(b->ev_member[m], b->members[m]->s_step));
    AHX_BCUDA(b, cudaStreamWaitEvent(b->s, b->ev_member[m], 0));
  }
  int left = n;
  if (b->branches) {
    cudaGraphExec_t g = nullptr;
    if (left >= 2) {
      if (ahx_status st = branch_graph(b, 2, &g)) return st;
      for (; left >= 2; left -= 2) AHX_BCUDA(b, cudaGraphLaunch(g, b->s));
    }
    if (left == 1) {
      if (ahx_status st = branch_graph(b, 1, &g)) return st;
      AHX_BCUDA(b, cudaGraphLaunch(g, b->s));
      b->phase ^= 1;
      left = 0;
    }
  }
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
  ahx_status st = AHX_OK;
  {
    std::lock_guard<std::mutex> lk(b->mu);
    if (ahx_status c = check_batch(b)) return c;
    AHX_BCUDA(b, cudaSetDevice(b->dev));
    AHX_BCUDA(b, cudaEventCreate(&e0));
    AHX_BCUDA(b, cudaEventCreate(&e1));
    // e0 after the members' queued work, so the interval holds only the batched steps
    MemberLocks lock(b->members);
    for (size_t m = 0; m < b->members.size() && st == AHX_OK; ++m) {
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
  out->use_graph = b->branches ? 2 : (b->use_graph ? 1 : 0);
  out->pairs = b->pairs ? 1 : 0;
  out->zslab_max = b->zslab.empty() ? 0 : *std::max_element(b->zslab.begin(), b->zslab.end());
  out->cells = b->cells;
  return check_batch(b);
}

ahx_status ahx_batch_destroy(ahx_batch* b) {
  if (!b) return fail(AHX_EINVAL, "live solver: null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (b->destroyed) return AHX_OK;
  b->destroyed = true;
  release(b);
  MemberLocks lock(b->members);
  for (ahx_handle* h : b->members) --h->batch_refs;
  // the batch object stays allocated so later calls report "batch destroyed"
  return AHX_OK;
}

}  // extern "C"
