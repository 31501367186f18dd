// Internal state of a live-solver handle, shared by the C ABI translation units (api.cu, batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "ahx.h"
#include "launch.h"

namespace ahx {

constexpr int kUploadSlots = 4;
// column levels (kt, ktop) are validated against this bound so every level index stays a small non-negative int
constexpr uint32_t kMaxLevel = 65535;

struct ReadSlot {
  bool busy = false;
  uint64_t ticket = 0;
  int nzv = 0, want_vol = 0, want_wind = 0;
  float* d_surf = nullptr;     // 3*NXY
  uint32_t* d_vol = nullptr;   // ceil(nz*NXY/4)
  unsigned* d_tmax = nullptr;
  float* h_surf = nullptr;     // pinned
  uint8_t* h_vol = nullptr;    // pinned
  unsigned* h_tmax = nullptr;  // pinned
  cudaEvent_t ev_kernels = nullptr, ev_done = nullptr;
};

struct UploadSlot {
  void* h = nullptr;   // pinned
  size_t bytes = 0;
  cudaEvent_t ev = nullptr;
  bool used = false;
};

struct Fence {
  uint64_t ticket;
  cudaEvent_t ev;
};

}  // namespace ahx

struct ahx_handle {
  std::mutex mu;
  int dev = 0;
  bool destroyed = false;
  bool lost = false;
  std::string lost_msg;
  cudaStream_t s_step = nullptr, s_copy = nullptr;
  ahx_dims dims{};
  int esize = 4, esize_g = 4, px = 0;   // bytes per stored f / g population; x pitch in elements
  uint32_t ps = 0, qs = 0;
  void* f[2] = {nullptr, nullptr};
  void* g[2] = {nullptr, nullptr};
  unsigned char* d_params = nullptr;
  uint4* d_colv = nullptr;
  uint32_t* d_ktop = nullptr;
  uint32_t* d_oldk = nullptr;
  float4* d_dbg = nullptr;
  double* d_budget = nullptr;
  bool budget_on = false;
  bool accum_on = false;                  // FP64 time accumulators (near-ground and lateral faces)
  double* d_sacc = nullptr;               // 3 * NXY
  double* d_facc = nullptr;               // 2 * (2 ny nz + 2 nx nz)
  int64_t accum_steps = 0;
  ahx::StatsScratch* d_stats = nullptr;
  int parity = 0;
  int64_t steps = 0;
  int block_y = 4, zslab = 0, minb = 0;
  bool pairs = false;                     // paired levels on packed f32x2 arithmetic (FMA build)
  int jg0 = 0, nyg = 0, jlo = 0, jhi = 0;   // y-slab of a larger domain (nyg = 0: the whole domain)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // two plain steps starting at parity 0 / 1
  uint64_t graph_key[2] = {0, 0};                 // launch set-up each graph was captured with
  int tma_ty = 0, tma_depth = 0;          // staged kernel selected when tma_ty > 0
  bool maps_ok = false;
  ahx::TmaMaps maps[2][2];                     // [TY 4 / 8][parity]: tensor maps of the state read by a step
  bool pmaps_ok = false;
  ahx::TmaMaps pmaps[2][2];                    // the same over the 32-bit words of level-paired 16-bit planes
  int* d_err = nullptr;                   // error word the staged kernel sets
  bool prefetch = false;                  // next-level L2 prefetch in the step (launch option, FMA build)
  uint32_t* d_tick = nullptr;             // step counter pair of the stochastic-rounding storage, then the tuner's
  ahx::ReadSlot reads[AHX_MAX_READS];
  uint64_t next_read = 0;
  ahx::UploadSlot up[ahx::kUploadSlots];
  int up_next = 0;
  std::vector<ahx::Fence> fences;
  uint64_t next_fence = 0;
  char name[64] = {0};
  int batch_refs = 0;                     // batches this handle belongs to (it cannot be destroyed meanwhile)
  std::atomic<int> batch_lost{0};         // set (without the lock) when a batched step over this handle failed
};


namespace ahx {

// helpers of api.cu that batch.cu uses
ahx_status fail(ahx_status st, const std::string& msg);                      // sets ahx_last_error()
ahx_status cuda_fail(ahx_handle* h, cudaError_t e, const char* what);       // marks h lost (if non-null)
ahx_status check(ahx_handle* h);                                             // null / destroyed / lost
DomainView view_at(ahx_handle* h, int parity);                               // the state read at this parity
StepLaunch solo_launch(const ahx_handle* h, int parity);   // a plain step of this handle (its launch shape) at a parity
uint64_t solo_launch_key(const ahx_handle* h);             // everything solo_launch depends on besides the parity
// the tensor maps a staged launch reads at a parity (single-level or paired-word maps), or null for a plain launch
const TmaMaps* stage_maps(const ahx_handle* h, const StepLaunch& L, int parity);
cudaError_t solo_step(ahx_handle* h, int parity, cudaStream_t s);   // launch one plain step reading that parity
ahx_status wait_event(ahx_handle* h, cudaEvent_t ev, int timeout_ms);        // bounded, lock not held

}  // namespace ahx
