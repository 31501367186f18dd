// Satellite kernels of the live solver for sm_100a: near-surface and volume read-back, flow initialisation,
// solid->fluid re-initialisation, diagnostics, and the layout conversion between the reference's [q][cell] f32
// layout and the pitched internal storage. Built with -fmad=false like the exact step, so the read-back of the
// moments is bit-identical to the CPU restatement of the reference kernels.
#include "fused.cuh"
#include "launch.h"

namespace ahx {

int element_bytes(int precision) {
  switch (precision) {
    case 0: return 4;
    case 1: return 2;
    case 2: return 2;
    case 3: return 8;
    case 4: return 2;   // f FP16, g f32
    case 5: return 2;   // f BF16, g f32
    case 6: return 2;   // FP16, stochastic rounding in the step
    default: return 0;
  }
}

int element_bytes_g(int precision) { return precision == 4 || precision == 5 ? 4 : element_bytes(precision); }

namespace {

__device__ __forceinline__ void load_params_smem(const DomainView& D, ParamsHead& sP, float4* prof) {
  const int tid = threadIdx.x;
  if (tid < 16) reinterpret_cast<int*>(&sP)[tid] = reinterpret_cast<const int*>(D.params)[tid];
  const float4* g = reinterpret_cast<const float4*>(D.params + 64);
  for (int z = tid; z < D.nz; z += blockDim.x) prof[z] = g[z];
  __syncthreads();
}

// genSurfWGSL (kernel.js:435-471): pre-collision theta and force-corrected (u, v)*conv of the first fluid cell of
// every column, north-up [row][col]; zeros where ktop >= nz.
template <class S>
__global__ void __launch_bounds__(128) surf_kernel(DomainView D, float conv, float* sout) {
  using R = RealOf<S>;
  extern __shared__ float4 prof[];
  __shared__ ParamsHead sP;
  load_params_smem(D, sP, prof);
  const int NXY = D.nx * D.ny;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= NXY) return;
  const int i = c % D.nx, j = c / D.nx;
  const int o = (D.ny - 1 - j) * D.nx + i;
  const uint4 cv = __ldg(D.colv + c);
  const int k = (int)cv.y;
  if (k < 0 || k >= D.nz) {
    sout[o] = 0.f;
    sout[NXY + o] = 0.f;
    sout[2 * NXY + o] = 0.f;
    return;
  }
  Column<R> C;
  load_column(D, sP, i, j, C);
  Cell<R> X;
  stream_cell<S>(D, sP, prof, C, k, (uint32_t)j * (uint32_t)D.px + (uint32_t)i, X);
  Macro<R> M;
  moments_forces<R>(sP, C, k, D.nz, X, M);
  sout[o] = (float)M.th;
  sout[NXY + o] = (float)M.ux * conv;
  sout[2 * NXY + o] = (float)M.uy * conv;
}

// genVolWGSL (kernel.js:475-520): theta (streamed g, summed) of the lowest nzv levels, north-up [k][row][col],
// quantised to u8 round(theta*volscale) clamped to 0..255, 4 cells per u32 (little-endian); solid cells are 0; the
// max theta (>= 0) over these cells into *tmax_bits (f32 bits, non-negative floats order as unsigned).
template <class S>
__global__ void __launch_bounds__(256) vol_kernel(DomainView D, int nzv, float volscale, uint32_t* vout,
                                                  unsigned* tmax_bits) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  __shared__ ParamsHead sP;
  __shared__ unsigned wmax;
  const int tid = threadIdx.x;
  if (tid < 16) reinterpret_cast<int*>(&sP)[tid] = reinterpret_cast<const int*>(D.params)[tid];
  if (tid == 0) wmax = 0u;
  __syncthreads();
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const long NXY = (long)nx * ny;
  const long NVOL = (long)nzv * NXY;
  const long NW = (NVOL + 3) / 4;
  const long t = (long)blockIdx.x * blockDim.x + tid;
  const StoreG<S>* gA = static_cast<const StoreG<S>*>(D.gA);
  float tmax = 0.f;
  if (t < NW) {
    uint32_t packed = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const long p = 4 * t + e;
      if (p < NVOL) {
        const int k = (int)(p / NXY);
        const long rem = p % NXY;
        const int i = (int)(rem % nx);
        const int j = ny - 1 - (int)(rem / nx);
        const int kg = (int)__ldg(D.ktop + (long)j * nx + i);
        R th = R(0);
        if (k >= kg) {
          using TG = StoreG<S>;
          const uint32_t m = (uint32_t)j * (uint32_t)D.px + (uint32_t)i, n = lvl<TG>(k, m, D.ps);
          R g[7];
          g[0] = KG::dec_g(KG::load(gA + n));
          static_for<6>([&](auto Qm1) {
            constexpr int q = Qm1 + 1;
            constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
            const int si = i - cx, sj = j - cy, sk = k - cz;
            R gv;
            if (sk >= nz) {
              gv = KG::dec_g(KG::load(gA + (uint32_t)q * D.qs + n));
            } else if (si < 0 || si >= nx || sj < 0 || sj >= ny) {
              bool inflow = false;
              if constexpr (cx == 1) inflow = inflow || (si < 0 && sP.inflow_w != 0);
              if constexpr (cx == -1) inflow = inflow || (si >= nx && sP.inflow_e != 0);
              if constexpr (cy == 1) inflow = inflow || (sj < 0 && sP.inflow_s != 0);
              if constexpr (cy == -1) inflow = inflow || (sj >= ny && sP.inflow_n != 0);
              gv = inflow ? R(0) : KG::dec_g(KG::load(gA + (uint32_t)q * D.qs + n));
            } else if (sk < (int)__ldg(D.ktop + (long)sj * nx + si)) {
              gv = KG::dec_g(KG::load(gA + (uint32_t)opp7(q) * D.qs + n));
            } else {
              // the offset wraps in 32 bits before it touches the pointer (cx = -1 gives a negative shift)
              const uint32_t off = (uint32_t)q * D.qs + lvl<TG>(sk, m - (uint32_t)(cx + cy * D.px), D.ps);
              gv = KG::dec_g(KG::load(gA + off));
            }
            g[q] = gv;
          });
          th = g[0];
#pragma unroll
          for (int q = 1; q < 7; ++q) th = th + g[q];
        }
        const float thf = (float)th;
        const float r = rintf(thf * volscale);   // WGSL round(): half to even
        const uint32_t qv = (uint32_t)fminf(fmaxf(r, 0.f), 255.f);
        packed |= qv << (8u * (uint32_t)e);
        tmax = fmaxf(tmax, thf);
      }
    }
    vout[t] = packed;
  }
  // block max of the non-negative f32 bits, then one global atomic per block
  unsigned b = __float_as_uint(fmaxf(tmax, 0.f));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((tid & 31) == 0) atomicMax(&wmax, b);
  __syncthreads();
  if (tid == 0 && wmax != 0u) atomicMax(tmax_bits, wmax);
}

// genInitWGSL (kernel.js:524-553): equilibrium with the inflow profile at the local height above terrain in every
// cell (solid ones included), written to both population buffers.
template <class S>
__global__ void __launch_bounds__(256) init_kernel(DomainView D, StoreF<S>* f0, StoreF<S>* f1) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  const float4* prof = reinterpret_cast<const float4*>(D.params + 64);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= D.nx) return;
  const int ktc = (int)__ldg(D.colv + (size_t)j * D.nx + i).x;
  const int zagl = min(max(k - ktc, 0), D.nz - 1);
  const float4 pr = __ldg(prof + zagl);
  const R U = R(pr.x), V = R(pr.y);
  const R usq = U * U + V * V;
  const uint32_t n = lvl<StoreF<S>>(k, (uint32_t)j * (uint32_t)D.px + (uint32_t)i, D.ps);
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    const R cu = R(kC19[q][0]) * U + R(kC19[q][1]) * V;
    const R fq = R(w19(q)) * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usq);
    const StoreF<S> e = KF::enc_f(fq, R(w19(q)));
    f0[(uint32_t)q * D.qs + n] = e;
    f1[(uint32_t)q * D.qs + n] = e;
  });
}

// genReinitWGSL (kernel.js:557-575): cells that turned from solid to fluid (k in [ktop, min(oldk, nz))) get rest
// equilibrium f = w and theta = 0.
template <class S>
__global__ void __launch_bounds__(256) reinit_kernel(DomainView D, const uint32_t* oldk, StoreF<S>* f,
                                                      StoreG<S>* g) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int NXY = D.nx * D.ny;
  if (c >= NXY) return;
  const int i = c % D.nx, j = c / D.nx;
  const int k1 = min((int)oldk[c], D.nz);
  for (int k = (int)D.ktop[c]; k < k1; ++k) {
    const uint32_t m = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
    const uint32_t nf = lvl<StoreF<S>>(k, m, D.ps), ng = lvl<StoreG<S>>(k, m, D.ps);
    static_for<19>([&](auto Q) {
      constexpr int q = Q;
      f[(uint32_t)q * D.qs + nf] = KF::enc_f(R(w19(q)), R(w19(q)));
    });
    static_for<7>([&](auto Q) {
      constexpr int q = Q;
      g[(uint32_t)q * D.qs + ng] = KG::enc_g(R(0));
    });
  }
}

// genStatsWGSL (kernel.js:580-633) over the fluid cells of the current state: per-cell f32 values (theta,
// 0.5|j|^2/rho, rho - 1, 1) summed in FP64, max theta (>= 0), non-finite count (rho or theta), max |j|/rho.
template <class S>
__global__ void __launch_bounds__(256) stats_kernel(DomainView D, StatsScratch* out) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  const StoreF<S>* fA = static_cast<const StoreF<S>*>(D.fA);
  const StoreG<S>* gA = static_cast<const StoreG<S>*>(D.gA);
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  const long total = (long)nx * ny * nz;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  float tmax = 0.f, umax = 0.f;
  unsigned nonf = 0;
  for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (long)gridDim.x * blockDim.x) {
    const int i = (int)(c % nx);
    const int j = (int)((c / nx) % ny);
    const int k = (int)(c / ((long)nx * ny));
    if (j < D.jlo || j >= D.jhi) continue;   // ghost rows of a slab belong to its neighbour
    if (k < (int)__ldg(D.ktop + (long)j * nx + i)) continue;
    const uint32_t m = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
    const uint32_t nf = lvl<StoreF<S>>(k, m, D.ps), ng = lvl<StoreG<S>>(k, m, D.ps);
    R f[19];
    static_for<19>([&](auto Q) {
      constexpr int q = Q;
      f[q] = KF::dec_f(KF::load(fA + (uint32_t)q * D.qs + nf), R(w19(q)));
    });
    float rho = (float)f[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) rho = rho + (float)f[q];
    auto fq = [&](int q) { return (float)f[q]; };
    const float jx = moment1<float, 0>(fq), jy = moment1<float, 1>(fq), jz = moment1<float, 2>(fq);
    float th = (float)KG::dec_g(KG::load(gA + ng));
#pragma unroll
    for (int q = 1; q < 7; ++q) th = th + (float)KG::dec_g(KG::load(gA + (uint32_t)q * D.qs + ng));
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
  if ((threadIdx.x & 31) == 0) {
    if (s3 != 0.0 || s0 != 0.0) {
      atomicAdd(&out->sum[0], s0);
      atomicAdd(&out->sum[1], s1);
      atomicAdd(&out->sum[2], s2);
      atomicAdd(&out->sum[3], s3);
    }
    atomicMax(&out->tmax_bits, __float_as_uint(tmax));
    atomicMax(&out->umax_bits, __float_as_uint(umax));
    if (nonf) atomicAdd(&out->non_finite, nonf);
  }
}

// reference plane [cell] (f32 or f64) <-> internal pitched plane q
template <class T>
__global__ void __launch_bounds__(256) import_plane_kernel(DomainView D, const void* ref, int ref_is_f64, T* dst,
                                                           int q, int is_g) {
  using R = typename Codec<T>::Real;
  using K = Codec<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= D.nx) return;
  const size_t c = ((size_t)k * D.ny + j) * D.nx + i;
  const R v = ref_is_f64 ? R(static_cast<const double*>(ref)[c]) : R(static_cast<const float*>(ref)[c]);
  const double w = q == 0 ? 1.0 / 3 : (q < 7 ? 1.0 / 18 : 1.0 / 36);
  const uint32_t n = lvl<T>(k, (uint32_t)j * (uint32_t)D.px + (uint32_t)i, D.ps);
  dst[(uint32_t)q * D.qs + n] = is_g ? K::enc_g(v) : K::enc_f(v, R(w));
}

template <class T>
__global__ void __launch_bounds__(256) export_plane_kernel(DomainView D, const T* src, void* ref, int ref_is_f64,
                                                           int q, int is_g) {
  using R = typename Codec<T>::Real;
  using K = Codec<T>;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= D.nx) return;
  const size_t c = ((size_t)k * D.ny + j) * D.nx + i;
  const double w = q == 0 ? 1.0 / 3 : (q < 7 ? 1.0 / 18 : 1.0 / 36);
  const uint32_t n = lvl<T>(k, (uint32_t)j * (uint32_t)D.px + (uint32_t)i, D.ps);
  const T e = src[(uint32_t)q * D.qs + n];
  const R v = is_g ? K::dec_g(e) : K::dec_f(e, R(w));
  if (ref_is_f64) static_cast<double*>(ref)[c] = (double)v;
  else static_cast<float*>(ref)[c] = (float)v;
}

// one local row j of all 26 population planes <-> a packed buffer [f: 19][nz][nx], then (from the next 16-byte
// boundary) [g: 7][nz][nx]; raw storage elements
template <class TF, class TG>
__global__ void __launch_bounds__(256) row_copy_kernel(DomainView D, int j, const void* f, const void* g, void* buf,
                                                       int to_buffer) {
  const long per = (long)D.nz * D.nx;
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 26 * per) return;
  const int q = (int)(e / per);
  const int k = (int)((e % per) / D.nx), i = (int)(e % D.nx);
  const uint32_t m = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
  if (q < 19) {
    TF* s = const_cast<TF*>(static_cast<const TF*>(f)) + (uint32_t)q * D.qs + lvl<TF>(k, m, D.ps);
    TF* b = static_cast<TF*>(buf) + (long)q * per + (long)k * D.nx + i;
    if (to_buffer) *b = *s;
    else *s = *b;
  } else {
    TG* s = const_cast<TG*>(static_cast<const TG*>(g)) + (uint32_t)(q - 19) * D.qs + lvl<TG>(k, m, D.ps);
    // the g part starts at the next 16-byte boundary after the f part
    const size_t goff = (19 * (size_t)per * sizeof(TF) + 15) & ~(size_t)15;
    TG* b = reinterpret_cast<TG*>(static_cast<unsigned char*>(buf) + goff) + (long)(q - 19) * per + (long)k * D.nx + i;
    if (to_buffer) *b = *s;
    else *s = *b;
  }
}

// The halo of a y-slab boundary: of row j, only the populations that cross the boundary toward the neighbour, c_y =
// dir (+1: the 5 flow populations and 1 temperature population moving north, which the north neighbour's first row
// pulls from its ghost row; -1: those moving south). Packed as [5][nz][nx] f, padded to 16 bytes, then [nz][nx] g.
// `src` selects the buffers (the state a step reads, or the one the step in progress writes).
struct HaloPlanes {
  int f[5], g;
};
__host__ __device__ constexpr HaloPlanes halo_planes(int dir) {
  HaloPlanes h{{0, 0, 0, 0, 0}, 0};
  int n = 0;
  for (int q = 0; q < 19; ++q)
    if (kC19[q][1] == dir) h.f[n++] = q;
  for (int q = 0; q < 7; ++q)
    if (kC7[q][1] == dir) h.g = q;
  return h;
}
static_assert(halo_planes(1).f[4] != 0 && halo_planes(-1).f[4] != 0, "five flow populations cross each boundary");

template <class TF, class TG, int DIR>
__global__ void __launch_bounds__(256) halo_copy_kernel(DomainView D, int j, const void* f, const void* g, void* buf,
                                                        int to_buffer) {
  const long per = (long)D.nz * D.nx;
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 6 * per) return;
  const int slot = (int)(e / per);
  const int k = (int)((e % per) / D.nx), i = (int)(e % D.nx);
  const uint32_t m = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
  constexpr HaloPlanes H = halo_planes(DIR);
  if (slot < 5) {
    TF* s = const_cast<TF*>(static_cast<const TF*>(f)) + (uint32_t)H.f[slot] * D.qs + lvl<TF>(k, m, D.ps);
    TF* b = static_cast<TF*>(buf) + (long)slot * per + (long)k * D.nx + i;
    if (to_buffer) *b = *s;
    else *s = *b;
  } else {
    TG* s = const_cast<TG*>(static_cast<const TG*>(g)) + (uint32_t)H.g * D.qs + lvl<TG>(k, m, D.ps);
    const size_t goff = (5 * (size_t)per * sizeof(TF) + 15) & ~(size_t)15;
    TG* b = reinterpret_cast<TG*>(static_cast<unsigned char*>(buf) + goff) + (long)k * D.nx + i;
    if (to_buffer) *b = *s;
    else *s = *b;
  }
}

template <class F>
cudaError_t dispatch(int precision, F&& f) {
  switch (precision) {
    case 0: return f(float{});
    case 1: return f(__half{});
    case 2: return f(__nv_bfloat16{});
    case 3: return f(double{});
    case 4: return f(Mixed<__half, float>{});
    case 5: return f(Mixed<__nv_bfloat16, float>{});
    case 6: return f(half_sr{});
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_init(const DomainView& D, int precision, void* f0, void* f1, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    dim3 grid((D.nx + 255) / 256, D.ny, D.nz);
    init_kernel<S><<<grid, 256, 0, s>>>(D, static_cast<StoreF<S>*>(f0), static_cast<StoreF<S>*>(f1));
    return cudaGetLastError();
  });
}

cudaError_t launch_reinit(const DomainView& D, int precision, const uint32_t* oldk, void* f, void* g,
                          cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    const int NXY = D.nx * D.ny;
    reinit_kernel<S><<<(NXY + 255) / 256, 256, 0, s>>>(D, oldk, static_cast<StoreF<S>*>(f),
                                                       static_cast<StoreG<S>*>(g));
    return cudaGetLastError();
  });
}

cudaError_t launch_surf(const DomainView& D, int precision, float conv, float* sout, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    const int NXY = D.nx * D.ny;
    surf_kernel<S><<<(NXY + 127) / 128, 128, (size_t)D.nz * sizeof(float4), s>>>(D, conv, sout);
    return cudaGetLastError();
  });
}

cudaError_t launch_vol(const DomainView& D, int precision, int nzv, float volscale, uint32_t* vout,
                       unsigned* tmax_bits, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    const long NW = ((long)nzv * D.nx * D.ny + 3) / 4;
    if (NW == 0) return cudaSuccess;
    vol_kernel<S><<<(unsigned)((NW + 255) / 256), 256, 0, s>>>(D, nzv, volscale, vout, tmax_bits);
    return cudaGetLastError();
  });
}

cudaError_t launch_stats(const DomainView& D, int precision, StatsScratch* out, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    stats_kernel<S><<<sms * 8, 256, 0, s>>>(D, out);
    return cudaGetLastError();
  });
}

cudaError_t launch_import_plane(const DomainView& D, int precision, const void* ref_plane, int ref_is_f64, void* dst,
                                int q, int is_g, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    dim3 grid((D.nx + 255) / 256, D.ny, D.nz);
    if (is_g)
      import_plane_kernel<StoreG<S>><<<grid, 256, 0, s>>>(D, ref_plane, ref_is_f64, static_cast<StoreG<S>*>(dst), q, 1);
    else
      import_plane_kernel<StoreF<S>><<<grid, 256, 0, s>>>(D, ref_plane, ref_is_f64, static_cast<StoreF<S>*>(dst), q, 0);
    return cudaGetLastError();
  });
}

cudaError_t launch_export_plane(const DomainView& D, int precision, const void* src, void* ref_plane, int ref_is_f64,
                                int q, int is_g, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    dim3 grid((D.nx + 255) / 256, D.ny, D.nz);
    if (is_g)
      export_plane_kernel<StoreG<S>><<<grid, 256, 0, s>>>(D, static_cast<const StoreG<S>*>(src), ref_plane,
                                                          ref_is_f64, q, 1);
    else
      export_plane_kernel<StoreF<S>><<<grid, 256, 0, s>>>(D, static_cast<const StoreF<S>*>(src), ref_plane,
                                                          ref_is_f64, q, 0);
    return cudaGetLastError();
  });
}

cudaError_t launch_halo_copy(const DomainView& D, int precision, int j, int dir, int next, void* buf, int to_buffer,
                             cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    const long total = 6L * D.nz * D.nx;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    const void* f = next ? D.fB : D.fA;
    const void* g = next ? D.gB : D.gA;
    if (dir > 0) halo_copy_kernel<StoreF<S>, StoreG<S>, 1><<<blocks, 256, 0, s>>>(D, j, f, g, buf, to_buffer);
    else halo_copy_kernel<StoreF<S>, StoreG<S>, -1><<<blocks, 256, 0, s>>>(D, j, f, g, buf, to_buffer);
    return cudaGetLastError();
  });
}

cudaError_t launch_row_copy(const DomainView& D, int precision, int j, void* buf, int to_buffer, cudaStream_t s) {
  return dispatch(precision, [&](auto tag) {
    using S = decltype(tag);
    const long total = 26L * D.nz * D.nx;
    row_copy_kernel<StoreF<S>, StoreG<S>><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(D, j, D.fA, D.gA, buf,
                                                                                          to_buffer);
    return cudaGetLastError();
  });
}

}  // namespace ahx
