// Internal launcher interface between the C ABI (api.cu) and the kernel translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "lattice.cuh"
#include "tma.cuh"

namespace ahx {

struct StepLaunch {
  int precision;   // ahx_precision
  int mode;        // 0 none, 1 out, 2 acc
  bool budget;
  int block_y;     // threads per block in y (x is one warp)
  int zslab;       // levels per block
  int minb = 0;    // 0, or 4 / 5 / 6 resident 128-thread blocks per SM (register budget 128 / 96 / 80)
  bool pairs = false;   // FMA build: two interior levels per thread on packed f32x2 arithmetic
  int tma_ty = 0;  // > 0: the TMA-staged kernel with 32 x tma_ty columns per block ...
  int tma_depth = 0;               // ... and this many levels staged ahead
  const TmaMaps* maps = nullptr;   // tensor maps of the state being read
};

// one tile of a batched step: block (bx, by, bz) of member `member`'s 32 x 4 x zslab decomposition
struct BatchTile {
  uint16_t member, bx, by, bz;
};

struct BatchLaunch {
  int precision;                 // ahx_precision, the same for every member
  int minb;                      // 4 / 5 / 6 resident 128-thread blocks per SM
  bool pairs;                    // FMA build: two interior levels per thread on packed f32x2 arithmetic
  int max_nz;                    // level capacity (sizes the staged inflow profile in shared memory)
  int grid;                      // persistent blocks
  const DomainView* views;       // device: one view per member
  const BatchTile* tiles;        // device: *ntiles tiles, member-major
  const int* zslabs;             // device: z-slab depth per member
  const int* ntiles;             // device: tile count
  int* sched;                    // device: [next tile, blocks done], zero between launches
};

// fused step, IEEE-exact arithmetic (step_exact.cu, built with -fmad=false)
namespace exact {
cudaError_t launch_step(const DomainView& D, const StepLaunch& L, cudaStream_t s);
// with occupancy != nullptr: only report resident blocks per SM for this configuration
cudaError_t launch_batch(const BatchLaunch& B, cudaStream_t s, int* occupancy);
}
// fused step, contracted arithmetic (step_fast.cu, built with -fmad=true)
namespace fast {
cudaError_t launch_step(const DomainView& D, const StepLaunch& L, cudaStream_t s);
cudaError_t launch_batch(const BatchLaunch& B, cudaStream_t s, int* occupancy);
}

// aux.cu
cudaError_t launch_init(const DomainView& D, int precision, void* f0, void* f1, cudaStream_t s);
cudaError_t launch_reinit(const DomainView& D, int precision, const uint32_t* oldk, void* f, void* g,
                          cudaStream_t s);
cudaError_t launch_surf(const DomainView& D, int precision, float conv, float* sout, cudaStream_t s);
cudaError_t launch_vol(const DomainView& D, int precision, int nzv, float volscale, uint32_t* vout,
                       unsigned* tmax_bits, cudaStream_t s);

struct StatsScratch {
  double sum[4];          // theta, ke, rho - 1, count
  unsigned tmax_bits;     // max(theta, 0) as f32 bits
  unsigned umax_bits;     // max |j|/rho as f32 bits
  unsigned non_finite;
  unsigned pad;
};
cudaError_t launch_stats(const DomainView& D, int precision, StatsScratch* out, cudaStream_t s);

// layout conversion of one population plane q between the reference layout (f32 or f64, [cell]) and the internal
// pitched storage; is_g selects the theta codec
cudaError_t launch_import_plane(const DomainView& D, int precision, const void* ref_plane, int ref_is_f64, void* dst,
                                int q, int is_g, cudaStream_t s);
cudaError_t launch_export_plane(const DomainView& D, int precision, const void* src, void* ref_plane, int ref_is_f64,
                                int q, int is_g, cudaStream_t s);

// copy local row j of all 26 planes of the current state (D.fA / D.gA) to (to_buffer) or from a packed device buffer
cudaError_t launch_row_copy(const DomainView& D, int precision, int j, void* buf, int to_buffer, cudaStream_t s);
// copy the halo of local row j (the 6 planes with c_y = dir) of the current state (next = 0: D.fA / D.gA) or of the
// state the step in progress writes (next = 1: D.fB / D.gB) to (to_buffer) or from a packed device buffer
cudaError_t launch_halo_copy(const DomainView& D, int precision, int j, int dir, int next, void* buf, int to_buffer,
                             cudaStream_t s);

int element_bytes(int precision);     // bytes of one stored flow population f
int element_bytes_g(int precision);   // bytes of one stored temperature population g

// the thread-local message ahx_last_error() returns (api.cu)
void set_last_error(const std::string& m);

}  // namespace ahx
