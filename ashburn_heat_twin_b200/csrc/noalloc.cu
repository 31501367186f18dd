// Diagnostics over a caller-owned state with no allocation of any kind: ahx_stats_noalloc (include/ahx.h).
//
// Who needs this: callers that cannot allocate device memory at the moment they want diagnostics, such as an engine
// that has handed all device memory to a fixed pool up front (an allocation outside the pool can fail or break its
// budget), or code on a latency-critical path where cudaMalloc / cudaFree would synchronise the device. They still own the state (populations f, g and the ktop plane, in device memory, reference layout) and an
// output record in device memory; this entry point only launches kernels on the caller's stream.
//
// The reduction's per-block partial sums live in one file-scope device array, g_stats_partials, of a fixed size
// (kMaxBlocks records of 8 doubles = 1 MiB). Every GPU that loads this library holds that array until the process
// exits. Every call on a device shares it and it keeps the last call's contents; each call overwrites every slot it
// later reads, so nothing has to start at zero. Two calls whose kernels overlap on the GPU (different streams without
// ordering between them) race on the array: order them, or use ahx_stats on a handle.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "ahx.h"
#include "fused.cuh"
#include "launch.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerBlock = 8192;       // cells one block reduces
constexpr int kMaxBlocks = 16384;          // capacity of the partials array
constexpr long long kMaxCells = (long long)kMaxBlocks * kCellsPerBlock;   // 134,217,728 cells

struct Partial {
  double sum[4];       // theta, ke, rho - 1, count
  unsigned tmax_bits;  // max(theta, 0) as f32 bits
  unsigned umax_bits;  // max |j|/rho as f32 bits
  unsigned non_finite;
  unsigned pad[5];
};
static_assert(sizeof(Partial) == 64, "one partial is 64 bytes");

// the scratch: file scope, 256-byte aligned, fixed size (1 MiB)
static __device__ __align__(256) Partial g_stats_partials[kMaxBlocks];

ahx_status fail(ahx_status st, const std::string& m) {
  ahx::set_last_error(m);   // read back with ahx_last_error(), like every other entry point
  return st;
}

// Per-device address of g_stats_partials, looked up once per device (with that device current) and again whenever
// the device's current context is a different one than at the look-up (after cudaDeviceReset, or a context the
// caller made itself): an address belongs to the context it was resolved in.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
Partial* g_addr[kMaxDevices] = {nullptr};
unsigned long long g_ctx[kMaxDevices] = {0};

// unique id of the calling thread's current context (driver entry points found through the runtime, so the library
// needs no link to the driver library); 0 when there is no current context or the driver cannot say
unsigned long long current_context_id() {
  using CtxGetCurrentFn = CUresult (*)(CUcontext*);
  using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || c == nullptr || get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Block b reduces cells [b*kCellsPerBlock, (b+1)*kCellsPerBlock) of the reference layout (cell = (k*ny + j)*nx + i)
// in a fixed order and writes its partial record; the same per-cell f32 values as the stats kernel (kernel.js:580-633).
__global__ void __launch_bounds__(kThreads) partial_kernel(const float* __restrict__ f, const float* __restrict__ g,
                                                           const uint32_t* __restrict__ ktop, int nx, int ny,
                                                           long long N, Partial* parts) {
  __shared__ double s_sum[4][kThreads / 32];
  __shared__ float s_tmax[kThreads / 32], s_umax[kThreads / 32];
  __shared__ unsigned s_nonf[kThreads / 32];
  const long long c0 = (long long)blockIdx.x * kCellsPerBlock;
  const long long c1 = min(N, c0 + kCellsPerBlock);
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  float tmax = 0.f, umax = 0.f;
  unsigned nonf = 0;
  const long long NXY = (long long)nx * ny;
  for (long long c = c0 + threadIdx.x; c < c1; c += kThreads) {
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / NXY);
    if (k < (int)__ldg(ktop + (long long)j * nx + i)) continue;
    float fq[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) fq[q] = __ldg(f + (long long)q * N + c);
    float rho = fq[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) rho = rho + fq[q];
    auto fv = [&](int q) { return fq[q]; };
    const float jx = ahx::moment1<float, 0>(fv), jy = ahx::moment1<float, 1>(fv), jz = ahx::moment1<float, 2>(fv);
    float th = __ldg(g + c);
#pragma unroll
    for (int q = 1; q < 7; ++q) th = th + __ldg(g + (long long)q * N + c);
    const unsigned br = __float_as_uint(rho) & 0x7f800000u, bt = __float_as_uint(th) & 0x7f800000u;
    if (br == 0x7f800000u || bt == 0x7f800000u) {
      ++nonf;
      continue;
    }
    s0 += (double)th;
    s1 += (double)(0.5f * (jx * jx + jy * jy + jz * jz) / rho);
    s2 += (double)(rho - 1.0f);
    s3 += 1.0;
    tmax = fmaxf(tmax, fmaxf(th, 0.f));
    umax = fmaxf(umax, sqrtf(jx * jx + jy * jy + jz * jz) / rho);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
    umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, o));
    nonf += __shfl_xor_sync(0xffffffffu, nonf, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_sum[0][w] = s0;
    s_sum[1][w] = s1;
    s_sum[2][w] = s2;
    s_sum[3][w] = s3;
    s_tmax[w] = tmax;
    s_umax[w] = umax;
    s_nonf[w] = nonf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p;
    for (int a = 0; a < 4; ++a) {
      double t = 0;
      for (int b = 0; b < kThreads / 32; ++b) t += s_sum[a][b];
      p.sum[a] = t;
    }
    float tm = 0.f, um = 0.f;
    unsigned nf = 0;
    for (int b = 0; b < kThreads / 32; ++b) {
      tm = fmaxf(tm, s_tmax[b]);
      um = fmaxf(um, s_umax[b]);
      nf += s_nonf[b];
    }
    p.tmax_bits = __float_as_uint(tm);
    p.umax_bits = __float_as_uint(um);
    p.non_finite = nf;
    for (int a = 0; a < 5; ++a) p.pad[a] = 0;
    parts[blockIdx.x] = p;
  }
}

// one block sums the partials in block order (deterministic) into the caller's ahx_stats_out
__global__ void __launch_bounds__(kThreads) final_kernel(const Partial* parts, int nblocks, ahx_stats_out* out) {
  __shared__ double s[4][kThreads];
  __shared__ float st[kThreads], su[kThreads];
  __shared__ unsigned sn[kThreads];
  double a[4] = {0, 0, 0, 0};
  float tm = 0.f, um = 0.f;
  unsigned nf = 0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) {
    for (int q = 0; q < 4; ++q) a[q] += parts[b].sum[q];
    tm = fmaxf(tm, __uint_as_float(parts[b].tmax_bits));
    um = fmaxf(um, __uint_as_float(parts[b].umax_bits));
    nf += parts[b].non_finite;
  }
  for (int q = 0; q < 4; ++q) s[q][threadIdx.x] = a[q];
  st[threadIdx.x] = tm;
  su[threadIdx.x] = um;
  sn[threadIdx.x] = nf;
  __syncthreads();
  if (threadIdx.x == 0) {
    ahx_stats_out o;
    double t[4] = {0, 0, 0, 0};
    float m = 0.f, u = 0.f;
    unsigned n = 0;
    for (int b = 0; b < kThreads; ++b) {
      for (int q = 0; q < 4; ++q) t[q] += s[q][b];
      m = fmaxf(m, st[b]);
      u = fmaxf(u, su[b]);
      n += sn[b];
    }
    o.sum_theta = t[0];
    o.sum_ke = t[1];
    o.sum_rho_dev = t[2];
    o.count = t[3];
    o.theta_max = m;
    o.umax = u;
    o.non_finite = n;
    o.pad = 0;
    *out = o;
  }
}

}  // namespace

extern "C" ahx_status ahx_stats_noalloc(int nx, int ny, int nz, const float* f, const float* g, const uint32_t* ktop,
                                        ahx_stats_out* out, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !f || !g || !ktop || !out)
    return fail(AHX_EINVAL, "live solver: ahx_stats_noalloc: bad grid or null pointer");
  const long long N = (long long)nx * ny * nz;
  if (N > kMaxCells)
    return fail(AHX_EINVAL, "live solver: ahx_stats_noalloc handles at most " + std::to_string(kMaxCells) +
                                " cells (its fixed scratch holds " + std::to_string(kMaxBlocks) +
                                " partial sums); use ahx_stats on a handle for larger grids");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(AHX_EDEVICE, "live solver: ahx_stats_noalloc: no usable current CUDA device");
  Partial* parts = nullptr;
  {
    // set-up, once per device and context, with that device current: the device address of the scratch array
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_addr[dev] || ctx == 0 || ctx != g_ctx[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_stats_partials);
      if (e != cudaSuccess || !p) {
        g_addr[dev] = nullptr;
        return fail(AHX_EDEVICE, std::string("live solver: ahx_stats_noalloc: cannot resolve its scratch (") +
                                     cudaGetErrorString(e) + ")");
      }
      g_addr[dev] = static_cast<Partial*>(p);
      g_ctx[dev] = current_context_id();   // the look-up made the device's primary context current if none was
    }
    parts = g_addr[dev];
  }
  const int nblocks = (int)((N + kCellsPerBlock - 1) / kCellsPerBlock);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  partial_kernel<<<nblocks, kThreads, 0, s>>>(f, g, ktop, nx, ny, N, parts);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    final_kernel<<<1, kThreads, 0, s>>>(parts, nblocks, out);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return fail(AHX_EDEVICE, std::string("live solver: ahx_stats_noalloc: launch failed (") + cudaGetErrorString(e) +
                                 ")");
  return AHX_OK;
}
