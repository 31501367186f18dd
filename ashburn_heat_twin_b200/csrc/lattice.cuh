// D3Q19 / D3Q7 lattice tables, compile-time q loops and the population storage codecs of the B200 live solver.
//
// Lattice tables follow js/live/kernel.js:19-28 of the reference (velocity order, weights 1/3, 1/18, 1/36 and
// 1/4, 1/8, opposite and z-mirror maps); literals are rounded the way kernel.js:31-33 (fmt) rounds them: the f64
// fraction rounded once to the arithmetic type.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "split.h"

#include <type_traits>
#include <utility>

namespace ahx {

constexpr int kC19[19][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                             {1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1}, {-1, 0, -1}, {1, 0, -1},
                             {-1, 0, 1}, {0, 1, 1}, {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};
constexpr int kC7[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

__host__ __device__ constexpr int find19(int a, int b, int c) {
  for (int q = 0; q < 19; ++q)
    if (kC19[q][0] == a && kC19[q][1] == b && kC19[q][2] == c) return q;
  return -1;
}
__host__ __device__ constexpr int find7(int a, int b, int c) {
  for (int q = 0; q < 7; ++q)
    if (kC7[q][0] == a && kC7[q][1] == b && kC7[q][2] == c) return q;
  return -1;
}
__host__ __device__ constexpr int opp19(int q) { return find19(-kC19[q][0], -kC19[q][1], -kC19[q][2]); }
__host__ __device__ constexpr int mirz19(int q) { return find19(kC19[q][0], kC19[q][1], -kC19[q][2]); }
__host__ __device__ constexpr int opp7(int q) { return find7(-kC7[q][0], -kC7[q][1], -kC7[q][2]); }
__host__ __device__ constexpr double w19(int q) { return q == 0 ? 1.0 / 3 : (q < 7 ? 1.0 / 18 : 1.0 / 36); }
__host__ __device__ constexpr double w7(int q) { return q == 0 ? 1.0 / 4 : 1.0 / 8; }

// compile-time loop: f(std::integral_constant<int, 0>) ... f(std::integral_constant<int, N-1>)
template <int... Qs, class F>
__host__ __device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Qs...>, F&& f) {
  (f(std::integral_constant<int, Qs>{}), ...);
}
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// Population storage codecs. The state lives in HBM in one of four formats; collision and forcing always run in the
// arithmetic type Real (f32, or f64 for the FP64 build). 16-bit formats store (f_q - w_q) * scale: the rest
// equilibrium w_q is subtracted so the stored magnitude is the small deviation, which keeps FP16/BF16 relative
// rounding on the deviation instead of on O(w) values. Temperature populations g have rest state 0 and are stored
// scaled only.
constexpr float kScaleF16 = 16.0f;      // |f - w| < ~0.2 in the UI range: stays well inside FP16 normal range
constexpr float kScaleG16 = 16.0f;      // theta populations up to ~10 K x w: < 4096 after scaling
constexpr float kScaleBF16 = 1.0f;      // BF16 has the f32 exponent range: no scaling needed

template <class S>
struct Codec;

template <>
struct Codec<float> {
  using Real = float;
  static constexpr bool kDither = false;
  static constexpr int kBytes = 4;
  __device__ __forceinline__ static float load(const float* p) { return __ldg(p); }
  __device__ __forceinline__ static void store(float* p, float v) { __stcs(p, v); }
  __device__ __forceinline__ static float dec_f(float v, float /*w*/) { return v; }
  __device__ __forceinline__ static float dec_g(float v) { return v; }
  __device__ __forceinline__ static float enc_f(float v, float /*w*/) { return v; }
  __device__ __forceinline__ static float enc_g(float v) { return v; }
};

template <>
struct Codec<double> {
  using Real = double;
  static constexpr bool kDither = false;
  static constexpr int kBytes = 8;
  __device__ __forceinline__ static double load(const double* p) { return __ldg(p); }
  __device__ __forceinline__ static void store(double* p, double v) { __stcs(p, v); }
  __device__ __forceinline__ static double dec_f(double v, double /*w*/) { return v; }
  __device__ __forceinline__ static double dec_g(double v) { return v; }
  __device__ __forceinline__ static double enc_f(double v, double /*w*/) { return v; }
  __device__ __forceinline__ static double enc_g(double v) { return v; }
};

// The 16-bit codecs scale by powers of two, so (f - w)*s and h/s + w written as one FMA round exactly like the
// separate multiply and add (the product is exact): the contraction changes no bits.
template <>
struct Codec<__half> {
  using Real = float;
  static constexpr bool kDither = false;
  static constexpr int kBytes = 2;
  // 16-bit traffic goes through the unsigned short load / store builtins (the __half overloads are inline-asm
  // wrappers the scheduler cannot reason about)
  __device__ __forceinline__ static __half load(const __half* p) {
    return __ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(p)));
  }
  __device__ __forceinline__ static void store(__half* p, __half v) {
    __stcs(reinterpret_cast<unsigned short*>(p), __half_as_ushort(v));
  }
  __device__ __forceinline__ static float dec_f(__half v, float w) {
    return __fmaf_rn(__half2float(v), 1.0f / kScaleF16, w);
  }
  __device__ __forceinline__ static float dec_g(__half v) { return __fmul_rn(__half2float(v), 1.0f / kScaleG16); }
  __device__ __forceinline__ static __half enc_f(float v, float w) {
    return __float2half_rn(__fmaf_rn(v, kScaleF16, -kScaleF16 * w));
  }
  __device__ __forceinline__ static __half enc_g(float v) { return __float2half_rn(__fmul_rn(v, kScaleG16)); }
  // the pieces of the codec, for paired (two-lane) decoding and encoding with identical rounding
  static constexpr float kF = kScaleF16, kG = kScaleG16;
  __device__ __forceinline__ static float raw(__half v) { return __half2float(v); }
  __device__ __forceinline__ static __half cvt(float v) { return __float2half_rn(v); }
  // a level-pair word (low half: the even level): load, store, both halves widened, two values narrowed
  __device__ __forceinline__ static uint32_t load_w(const __half* p) { return __ldg(reinterpret_cast<const unsigned*>(p)); }
  __device__ __forceinline__ static void store_w(__half* p, uint32_t w) { __stcs(reinterpret_cast<unsigned*>(p), w); }
  __device__ __forceinline__ static float2 raw2(uint32_t w) {
    return make_float2(__half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu))),
                       __half2float(__ushort_as_half((unsigned short)(w >> 16))));
  }
  __device__ __forceinline__ static uint32_t cvt2(float lo, float hi) {
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
};

template <>
struct Codec<__nv_bfloat16> {
  using Real = float;
  static constexpr bool kDither = false;
  static constexpr int kBytes = 2;
  __device__ __forceinline__ static __nv_bfloat16 load(const __nv_bfloat16* p) {
    return __ushort_as_bfloat16(__ldg(reinterpret_cast<const unsigned short*>(p)));
  }
  __device__ __forceinline__ static void store(__nv_bfloat16* p, __nv_bfloat16 v) {
    __stcs(reinterpret_cast<unsigned short*>(p), __bfloat16_as_ushort(v));
  }
  __device__ __forceinline__ static float dec_f(__nv_bfloat16 v, float w) {
    return __fmaf_rn(__bfloat162float(v), 1.0f / kScaleBF16, w);
  }
  __device__ __forceinline__ static float dec_g(__nv_bfloat16 v) {
    return __fmul_rn(__bfloat162float(v), 1.0f / kScaleBF16);
  }
  __device__ __forceinline__ static __nv_bfloat16 enc_f(float v, float w) {
    return __float2bfloat16_rn(__fmaf_rn(v, kScaleBF16, -kScaleBF16 * w));
  }
  __device__ __forceinline__ static __nv_bfloat16 enc_g(float v) {
    return __float2bfloat16_rn(__fmul_rn(v, kScaleBF16));
  }
  // the pieces of the codec, for paired (two-lane) decoding and encoding with identical rounding
  static constexpr float kF = kScaleBF16, kG = kScaleBF16;
  __device__ __forceinline__ static float raw(__nv_bfloat16 v) { return __bfloat162float(v); }
  __device__ __forceinline__ static __nv_bfloat16 cvt(float v) { return __float2bfloat16_rn(v); }
  __device__ __forceinline__ static uint32_t load_w(const __nv_bfloat16* p) {
    return __ldg(reinterpret_cast<const unsigned*>(p));
  }
  __device__ __forceinline__ static void store_w(__nv_bfloat16* p, uint32_t w) {
    __stcs(reinterpret_cast<unsigned*>(p), w);
  }
  // a BF16 value is the high half of its f32 (exact widening)
  __device__ __forceinline__ static float2 raw2(uint32_t w) {
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xFFFF0000u));
  }
  __device__ __forceinline__ static uint32_t cvt2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
};

// FP16 storage whose step stores round stochastically: the same bits in memory as the __half codec ((f - w) * 16
// and g * 16), decoded alike, but the fused step encodes each population with Blackwell's stochastic-rounding
// conversion (cvt.rs.f16x2.f32): a 13-bit dither supplied by the kernel is added below the kept mantissa bits of the
// magnitude and the result truncated, so a value rounds away from zero with probability equal to the dropped
// fraction (unbiased, including the f16 subnormal range). The instruction converts two values at once: the low half
// of its result takes its dither from bits 0-12 of the random operand, the high half from bits 16-28. Round-to-nearest
// keeps a quasi-steady state's rounding error the same step after step, a persistent bias the flow integrates; the
// dither makes it zero-mean noise. Conversions outside the step (state upload, initialisation) round to nearest like
// the __half codec.
struct half_sr {
  unsigned short x;
};
template <>
struct Codec<half_sr> {
  using Real = float;
  static constexpr bool kDither = true;
  static constexpr int kBytes = 2;
  __device__ __forceinline__ static half_sr load(const half_sr* p) {
    return half_sr{__ldg(reinterpret_cast<const unsigned short*>(p))};
  }
  __device__ __forceinline__ static void store(half_sr* p, half_sr v) {
    __stcs(reinterpret_cast<unsigned short*>(p), v.x);
  }
  __device__ __forceinline__ static float raw(half_sr v) { return __half2float(__ushort_as_half(v.x)); }
  __device__ __forceinline__ static half_sr cvt(float v) { return half_sr{__half_as_ushort(__float2half_rn(v))}; }
  // two values at once: lo with dither bits 16-28 of r_lo, hi with bits 16-28 of r_hi; returns hi << 16 | lo
  __device__ __forceinline__ static uint32_t cvt_sr2(float lo, float hi, uint32_t r_lo, uint32_t r_hi) {
    const uint32_t rb = __byte_perm(r_lo, r_hi, 0x7632);   // r_lo[31:16] in the low half, r_hi[31:16] in the high
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rb));
    return d;
  }
  // one value, dither bits 16-28 of r (the same bits cvt_sr2 gives the low half, so a cell converts identically alone
  // or paired)
  __device__ __forceinline__ static half_sr cvt_sr(float v, uint32_t r) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.0f), "f"(v), "r"(r >> 16));
    return half_sr{(unsigned short)(d & 0xFFFFu)};
  }
  __device__ __forceinline__ static void store_bits(half_sr* p, uint32_t b16) {
    __stcs(reinterpret_cast<unsigned short*>(p), (unsigned short)b16);
  }
  __device__ __forceinline__ static uint32_t load_w(const half_sr* p) { return __ldg(reinterpret_cast<const unsigned*>(p)); }
  __device__ __forceinline__ static void store_w(half_sr* p, uint32_t w) { __stcs(reinterpret_cast<unsigned*>(p), w); }
  __device__ __forceinline__ static float2 raw2(uint32_t w) {
    return make_float2(__half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu))),
                       __half2float(__ushort_as_half((unsigned short)(w >> 16))));
  }
  __device__ __forceinline__ static float dec_f(half_sr v, float w) { return __fmaf_rn(raw(v), 1.0f / kScaleF16, w); }
  __device__ __forceinline__ static float dec_g(half_sr v) { return __fmul_rn(raw(v), 1.0f / kScaleG16); }
  __device__ __forceinline__ static half_sr enc_f(float v, float w) {
    return cvt(__fmaf_rn(v, kScaleF16, -kScaleF16 * w));
  }
  __device__ __forceinline__ static half_sr enc_g(float v) { return cvt(__fmul_rn(v, kScaleG16)); }
  __device__ __forceinline__ static half_sr enc_f_sr(float v, float w, uint32_t r) {
    return cvt_sr(__fmaf_rn(v, kScaleF16, -kScaleF16 * w), r);
  }
  __device__ __forceinline__ static half_sr enc_g_sr(float v, uint32_t r) { return cvt_sr(__fmul_rn(v, kScaleG16), r); }
  static constexpr float kF = kScaleF16, kG = kScaleG16;
};

// Dithers of one cell update: a 32-bit seed from the cell's global index and the step counter through an integer
// finaliser (the "lowbias32" xorshift-multiply hash published by C. Wellons); population slot p (f: q, g: 19 + q)
// uses bits 16-28 of seed x M_p, M_p an odd constant per slot (the finaliser of a slot number), so each dither is
// uniform (x -> x M_p is a bijection of the seed) and the 26 products are independent instructions.
__host__ __device__ constexpr uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
template <int P>
inline constexpr uint32_t kDitherMul = mix32(0x2545f491u + 0x9e3779b9u * (uint32_t)P) | 1u;

// encode through a codec, with the dither of population slot P of the cell seeded h when it rounds stochastically
template <class K, int P, class R>
__device__ __forceinline__ auto enc_f_d(R v, R w, uint32_t h) {
  if constexpr (K::kDither) return K::enc_f_sr(v, w, h * kDitherMul<P>);
  else return K::enc_f(v, w);
}
// encode flow population P given as x = f / w: full-width storages store w x; the 16-bit codecs store
// (f - w) s = x (s w) - s w, formed by one multiply-add
template <class K, int P, class R>
__device__ __forceinline__ auto enc_f_x(R x, R w, uint32_t h) {
  if constexpr (K::kBytes == 8) {
    return K::enc_f(__dmul_rn(x, w), w);
  } else if constexpr (K::kBytes == 4) {
    return K::enc_f(__fmul_rn(x, w), w);
  } else {
    const float e = __fmaf_rn(x, K::kF * w, -(K::kF * w));
    if constexpr (K::kDither) return K::cvt_sr(e, h * kDitherMul<P>);
    else return K::cvt(e);
  }
}
template <class K, int P, class R>
__device__ __forceinline__ auto enc_g_d(R v, uint32_t h) {
  if constexpr (K::kDither) return K::enc_g_sr(v, h * kDitherMul<19 + P>);
  else return K::enc_g(v);
}

// Population layout in HBM. A population plane holds the levels of px x ny pitched rows (m = j px + i in a level).
// 32- and 64-bit elements keep each level as its own plane: element k ps + m. 16-bit elements keep the two levels of
// a pair (2t, 2t + 1) side by side in one 32-bit word: element t (2 ps) + 2 m + (k & 1), so the paired step loads and
// stores both levels of a column with one 32-bit access (a plane then holds nz rounded up to even levels).
template <class T>
inline constexpr bool kLevelPairs = sizeof(T) == 2;
// element offset of level k, row-column m in a population plane; unsigned arithmetic, so a neighbour offset that
// steps below 0 wraps and comes back when the population plane's offset is added
template <class T>
__host__ __device__ __forceinline__ uint32_t lvl(int k, uint32_t m, uint32_t ps) {
  if constexpr (kLevelPairs<T>) return (uint32_t)(k >> 1) * (2u * ps) + 2u * m + (uint32_t)(k & 1);
  else return (uint32_t)k * ps + m;
}

// element offset of the neighbour (k - cz, m - d) of the cell (k, m) whose own offset is n (= lvl<T>(k, m, ps))
template <class T>
__host__ __device__ __forceinline__ uint32_t lvl_nbr(int k, uint32_t m, uint32_t n, int cz, uint32_t d, uint32_t ps) {
  if constexpr (kLevelPairs<T>) {
    // from the own offset n: the lateral shift moves 2 d elements; level k - cz is the other half of the own word
    // (k even, cz = -1: + 1; k odd, cz = +1: - 1) or a half of the word one pair down / up (k even, cz = +1:
    // + 1 - 2 ps; k odd, cz = -1: - 1 + 2 ps). Equal to lvl(k - cz, m - d) (m is implied by n)
    (void)m;
    const uint32_t dz = cz == 0 ? 0u
                        : cz > 0 ? ((k & 1) ? 0xFFFFFFFFu : 1u - 2u * ps)
                                 : ((k & 1) ? 2u * ps - 1u : 1u);
    return n - 2u * d + dz;
  } else {
    return n - (d + (uint32_t)(cz * (int)ps));
  }
}

// Storage of a state: a plain type stores f and g alike; Mixed<SF, SG> stores the flow populations f as SF and the
// temperature populations g as SG (16-bit f with f32 g keeps the heat budget: a per-step source increment can be
// far below half an ulp of a 16-bit g).
template <class SF, class SG>
struct Mixed {};
template <class S>
struct StorageOf {
  using F = S;
  using G = S;
};
template <class SF, class SG>
struct StorageOf<Mixed<SF, SG>> {
  using F = SF;
  using G = SG;
};
template <class S>
using CodecF = Codec<typename StorageOf<S>::F>;
template <class S>
using CodecG = Codec<typename StorageOf<S>::G>;
template <class S>
using RealOf = typename CodecF<S>::Real;
template <class S>
using StoreF = typename StorageOf<S>::F;
template <class S>
using StoreG = typename StorageOf<S>::G;
// whether the step's stores of storage S draw dithers (and so read and advance the step counter)
template <class S>
inline constexpr bool kDitherOf = Codec<typename StorageOf<S>::F>::kDither || Codec<typename StorageOf<S>::G>::kDither;

// Parameter block (kernel.js:44-50): 16 four-byte scalars, then nz x float4 (uin, vin, kbg, 0)
struct ParamsHead {
  float tau0, cs2smag, gbeta, prt, kfloor, momfac, srcscale, sigmax;
  int32_t inflow_w, inflow_e, inflow_s, inflow_n, nsp, nsw, oclip, pad1;
};
static_assert(sizeof(ParamsHead) == 64, "parameter head is 64 bytes");

constexpr int kBudgetSlots = 32;    // the budget record is replicated to spread FP64 atomics over 32 addresses
constexpr int kBudgetStride = 16;   // doubles per slot (11 used)

// One domain's device view. Populations are stored [q][k][j][i] with an x pitch `px` (elements) so every x row
// starts on a 128-byte boundary: element (q, k, j, i) is at q*qs + (k*ny + j)*px + i.
struct DomainView {
  const unsigned char* params;  // ParamsHead + nz float4 profile
  const uint4* colv;            // NXY records (kt, ktop, cd bits, q bits), row j = 0 south, no pitch
  const uint32_t* ktop;         // NXY
  const void* fA;               // current state
  void* fB;                     // next state
  const void* gA;
  void* gB;
  float4* dbg;                  // (theta, ux, uy, uz) per cell (pitched), or null
  double* budget;               // per-step FP64 budget accumulators, or null
  // FP64 time accumulators (budget variant only), or null: per column at the first fluid cell (theta, ux, uy);
  // per lateral-face cell (theta, u_n): west / east [k][j], then south / north [k][i]
  double* sacc;
  double* facc;
  int* err;                     // error word: a staged copy that did not arrive in time sets it
  // stochastic-rounding storages: [0] steps taken (seeds the dithers), [1] blocks (tiles) of the current step done;
  // the last block of a step to finish advances [0]. tick_blocks: blocks (tiles) of one step in a batched launch
  uint32_t* tick;
  uint32_t tick_blocks;
  int pf;                       // 1: the FMA build's plain step prefetches the next level's source rows into L2
  int nx, ny, nz, px;
  // y-slab of a larger domain: local row 0 is global row jg0 of nyg; only local rows [jlo, jhi) are updated (the
  // others are ghost rows refreshed from the neighbouring slabs); a whole domain has jg0 0, nyg ny, [0, ny)
  int jg0, nyg, jlo, jhi;
  int jbase;                    // first local row the launch's grid covers (0 unless a step of a band of rows)
  int strip;                    // strip width of the column split (step_split)
  uint32_t ps;                  // level stride px*ny (a 16-bit plane's level pair: 2 ps, lvl)
  uint32_t qs;                  // population plane stride: ps x (nz, rounded up to even with a 16-bit population)
  // element offset of the interior pull source of population q relative to the cell: q*qs - (cx + cy*px + cz*ps);
  // level-paired planes: of the first source word of a level pair (pull_offset). Kernel-parameter tables, so each
  // gather is one add of a constant operand
  uint32_t pull_f[19], pull_g[7];
  uint32_t plane[19];           // q*qs
  // interior accesses as (base pointer + cell index): the pull source of each population (fA / gA + pull offset) and
  // each population plane of the next state (fB / gB + q*qs), filled by set_pointers
  const void* src_f[19];
  const void* src_g[7];
  void* dst_f[19];
  void* dst_g[7];
};

// pull offset of population q with velocity (cx, cy, cz) for one storage element size (host only): the element offset
// of the interior pull source relative to the cell. Level-paired 16-bit planes (esize 2): the offset of the first of
// the source words of a level pair (2t, 2t + 1) relative to the pair's word: the pair's sources are levels 2t - cz and
// 2t + 1 - cz, in one word for cz = 0, else in this word and the next one up (2 ps further).
inline uint32_t pull_offset(int esize, uint32_t qs, uint32_t px, uint32_t ps, int q, int cx, int cy, int cz) {
  if (esize == 2) return (uint32_t)q * qs - 2u * (uint32_t)(cx + cy * (int)px) - (cz == 1 ? 2u * ps : 0u);
  return (uint32_t)q * qs - (uint32_t)(cx + cy * (int)px + cz * (int)ps);
}

// fill the offset tables of a view from its strides and element sizes (host only)
inline void set_offsets(DomainView& D, int esize_f, int esize_g) {
  for (int q = 0; q < 19; ++q) {
    D.plane[q] = (uint32_t)q * D.qs;
    D.pull_f[q] = pull_offset(esize_f, D.qs, (uint32_t)D.px, D.ps, q, kC19[q][0], kC19[q][1], kC19[q][2]);
  }
  for (int q = 0; q < 7; ++q) D.pull_g[q] = pull_offset(esize_g, D.qs, (uint32_t)D.px, D.ps, q, kC7[q][0], kC7[q][1], kC7[q][2]);
}

// fill the interior base pointers of a view from its state pointers and offset tables (host only; call again when
// fA / fB / gA / gB change)
inline void set_pointers(DomainView& D, int esize_f, int esize_g) {
  for (int q = 0; q < 19; ++q) {
    D.src_f[q] = static_cast<const unsigned char*>(D.fA) + (size_t)D.pull_f[q] * esize_f;
    D.dst_f[q] = static_cast<unsigned char*>(D.fB) + (size_t)D.plane[q] * esize_f;
  }
  for (int q = 0; q < 7; ++q) {
    D.src_g[q] = static_cast<const unsigned char*>(D.gA) + (size_t)D.pull_g[q] * esize_g;
    D.dst_g[q] = static_cast<unsigned char*>(D.gB) + (size_t)D.plane[q] * esize_g;
  }
}

}  // namespace ahx
