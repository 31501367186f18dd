// Relaxation of the FMA build written once for one cell (V = float or double) and for two cells at once (V = float2,
// the packed f32x2 instructions of sm_100: one FFMA2 does the work of two FFMAs).
//
// Every operation is an explicit round-to-nearest multiply, add, subtract or fused multiply-add, and the packed forms
// round each lane exactly like the scalar ones, so a cell relaxed on one lane of a pair gets the same bits as the same
// cell relaxed alone. That keeps results independent of how cells are paired (launch shape, batch tiles).
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "lattice.cuh"

namespace ahx {

__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vrcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ float vsqrt(float a) { return sqrtf(a); }

__device__ __forceinline__ double vfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double vmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double vadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double vsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double vrcp(double a) { return 1.0 / a; }
__device__ __forceinline__ double vsqrt(double a) { return sqrt(a); }

__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as one packed multiply-add, b (-1) + a: the product is exact, so each lane rounds exactly like a - b (a
// negated operand would cost two scalar negations first)
__device__ __forceinline__ float2 vsub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 vrcp(float2 a) { return make_float2(vrcp(a.x), vrcp(a.y)); }
__device__ __forceinline__ float vneg(float a) { return -a; }
__device__ __forceinline__ double vneg(double a) { return -a; }
__device__ __forceinline__ float2 vneg(float2 a) { return __fmul2_rn(a, make_float2(-1.0f, -1.0f)); }
__device__ __forceinline__ float2 vsqrt(float2 a) { return make_float2(vsqrt(a.x), vsqrt(a.y)); }

// a constant in lane type V
template <class V>
__device__ __forceinline__ V vc(double c);
template <>
__device__ __forceinline__ float vc<float>(double c) { return (float)c; }
template <>
__device__ __forceinline__ double vc<double>(double c) { return c; }
template <>
__device__ __forceinline__ float2 vc<float2>(double c) { return make_float2((float)c, (float)c); }

// c.(a, b, c) over the nonzero components of a compile-time direction (x, y, z order)
template <class V, int cx, int cy, int cz>
__device__ __forceinline__ V vdot(V a, V b, V c) {
  V acc = vc<V>(0.0);
  bool first = true;
  auto term = [&](V x, int s) {
    if (first) acc = s > 0 ? x : vneg(x);
    else acc = s > 0 ? vadd(acc, x) : vsub(acc, x);
    first = false;
  };
  if constexpr (cx != 0) term(a, cx);
  if constexpr (cy != 0) term(b, cy);
  if constexpr (cz != 0) term(c, cz);
  return acc;
}

// first moments and the pair sums of the streamed populations
template <class V>
struct Moments {
  V sp9[9], dp9[9];
  V rho, irho, jx, jy, jz, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, th;
};

template <class V>
__device__ __forceinline__ void lane_moments(const V (&f)[19], const V (&g)[7], Moments<V>& m) {
  static_for<9>([&](auto Pi) {
    constexpr int p = Pi;
    m.sp9[p] = vadd(f[2 * p + 1], f[2 * p + 2]);
    m.dp9[p] = vsub(f[2 * p + 1], f[2 * p + 2]);
  });
  V rho = f[0];
#pragma unroll
  for (int p = 0; p < 9; ++p) rho = vadd(rho, m.sp9[p]);
  V jx = vc<V>(0.0), jy = jx, jz = jx, Pxx = jx, Pyy = jx, Pzz = jx, Pxy = jx, Pxz = jx, Pyz = jx;
  static_for<9>([&](auto Pi) {
    constexpr int p = Pi;
    constexpr int q = 2 * p + 1;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    if constexpr (cx != 0) {
      jx = cx > 0 ? vadd(jx, m.dp9[p]) : vsub(jx, m.dp9[p]);
      Pxx = vadd(Pxx, m.sp9[p]);
    }
    if constexpr (cy != 0) {
      jy = cy > 0 ? vadd(jy, m.dp9[p]) : vsub(jy, m.dp9[p]);
      Pyy = vadd(Pyy, m.sp9[p]);
    }
    if constexpr (cz != 0) {
      jz = cz > 0 ? vadd(jz, m.dp9[p]) : vsub(jz, m.dp9[p]);
      Pzz = vadd(Pzz, m.sp9[p]);
    }
    if constexpr (cx != 0 && cy != 0) Pxy = cx * cy > 0 ? vadd(Pxy, m.sp9[p]) : vsub(Pxy, m.sp9[p]);
    if constexpr (cx != 0 && cz != 0) Pxz = cx * cz > 0 ? vadd(Pxz, m.sp9[p]) : vsub(Pxz, m.sp9[p]);
    if constexpr (cy != 0 && cz != 0) Pyz = cy * cz > 0 ? vadd(Pyz, m.sp9[p]) : vsub(Pyz, m.sp9[p]);
  });
  m.rho = rho;
  m.irho = vrcp(rho);
  m.jx = jx;
  m.jy = jy;
  m.jz = jz;
  m.Pxx = Pxx;
  m.Pyy = Pyy;
  m.Pzz = Pzz;
  m.Pxy = Pxy;
  m.Pxz = Pxz;
  m.Pyz = Pyz;
  m.th = vadd(vadd(vadd(g[0], vadd(g[1], g[2])), vadd(g[3], g[4])), vadd(g[5], g[6]));
}

// the macroscopic values the output modes and budgets use
template <class V>
struct Relaxed {
  V Fx, Fy, Fz, ux, uy, uz;
};

// Parameter-derived constants of the FMA build's relaxation: formed in double precision from the f32 parameters and
// rounded once to f32, once per block instead of once per cell (the double arithmetic is not free on the GPU).
struct RelaxConst {
  float momfac3;   // 3 * momfac
  float iprt;      // 1 / prt
};
__device__ __forceinline__ RelaxConst relax_const(const ParamsHead& P) {
  return RelaxConst{(float)(3.0 * (double)P.momfac), (float)(1.0 / (double)P.prt)};
}

// Regularised BGK + Smagorinsky + Guo forcing (secForces / secRelax / secCollision, kernel.js:279-367) and the
// scalar collision (secScalarCollision, kernel.js:369-386), q paired with its opposite. Fx0, Fy0: drag force (0 away
// from the ground cell); sg: top-sponge strength (0 below it); Ssrc: heat source (0 off the first fluid cell);
// tb_add: outflow-sponge addition to the background tau (0 outside it). Each post-collision flow population is handed
// to put_f(q, x) as x = f_q / w_q (the storage codec applies the weight, so a 16-bit codec folds it into its scaled
// deviation (f - w) s = (x - 1) w s in one multiply-add), each temperature population to put_g(q, g_q), as soon as it
// is formed, so the caller can store it without holding all 26.
//
// With E0 = rho (1 - 1.5 u.u) - 4.5 om trN / 3 - 3 fpre u.F (the rest population's bracket), the bracket of a moving
// pair (q, opp q) is E0 + cu (4.5 rho cu + 9 fpre cF) + 4.5 om Q:N +- 3 (rho cu + fpre cF).
template <class V, class PutF, class PutG>
__device__ __forceinline__ void lane_relax(const ParamsHead& P, const RelaxConst& K, const Moments<V>& m,
                                           const V (&g)[7], V uI, V vI, V kb, V sg, V Fx0, V Fy0, V Ssrc, V tb_add,
                                           Relaxed<V>& o, PutF&& put_f, PutG&& put_g) {
  const V rho = m.rho, irho = m.irho, jx = m.jx, jy = m.jy, jz = m.jz;
  const V rs = vmul(rho, sg);
  const V Fx = vfma(rs, vfma(vneg(jx), irho, uI), Fx0);
  const V Fy = vfma(rs, vfma(vneg(jy), irho, vI), Fy0);
  const V Fz = vfma(vneg(rs), vmul(jz, irho), vmul(vmul(rho, vc<V>(P.gbeta)), m.th));
  const V half = vc<V>(0.5);
  const V ux = vmul(vfma(half, Fx, jx), irho), uy = vmul(vfma(half, Fy, jy), irho), uz = vmul(vfma(half, Fz, jz), irho);
  const V usq = vfma(uz, uz, vfma(uy, uy, vmul(ux, ux)));
  const V r3 = vmul(rho, vc<V>(1.0 / 3.0));
  const V rux = vmul(rho, ux), ruy = vmul(rho, uy), ruz = vmul(rho, uz);
  const V Nxx = vfma(vneg(rux), ux, vsub(m.Pxx, r3));
  const V Nyy = vfma(vneg(ruy), uy, vsub(m.Pyy, r3));
  const V Nzz = vfma(vneg(ruz), uz, vsub(m.Pzz, r3));
  const V Nxy = vfma(vneg(rux), uy, m.Pxy);
  const V Nxz = vfma(vneg(rux), uz, m.Pxz);
  const V Nyz = vfma(vneg(ruy), uz, m.Pyz);
  const V off2 = vfma(Nyz, Nyz, vfma(Nxz, Nxz, vmul(Nxy, Nxy)));
  const V Pn = vsqrt(vfma(vc<V>(2.0), off2, vfma(Nzz, Nzz, vfma(Nyy, Nyy, vmul(Nxx, Nxx)))));
  const V tb = vadd(vfma(vc<V>(K.momfac3), kb, vc<V>(P.tau0)), tb_add);
  const V tau = vmul(half, vadd(tb, vsqrt(vfma(tb, tb, vmul(vmul(vc<V>(P.cs2smag), Pn), irho)))));
  const V itau = vrcp(tau);
  const V nusgs = vmul(vsub(tau, tb), vc<V>(1.0 / 3.0));
  const V kap = vadd(vfma(nusgs, vc<V>(K.iprt), kb), vc<V>(P.kfloor));
  const V taug = vfma(vc<V>(4.0), kap, half);
  const V om = vsub(vc<V>(1.0), itau);
  const V fpre = vfma(vc<V>(-0.5), itau, vc<V>(1.0));
  const V trN = vmul(vadd(vadd(Nxx, Nyy), Nzz), vc<V>(1.0 / 3.0));
  const V uF = vfma(uz, Fz, vfma(uy, Fy, vmul(ux, Fx)));
  const V base = vfma(vc<V>(-1.5), usq, vc<V>(1.0));
  const V m3uF = vmul(vc<V>(-3.0), uF);
  const V omtr = vmul(om, trN);
  // rho base - 4.5 om trN - 3 fpre uF: the rest population's bracket and the common part of every other one
  const V E0 = vfma(fpre, m3uF, vfma(vc<V>(-4.5), omtr, vmul(rho, base)));
  put_f(std::integral_constant<int, 0>{}, E0);
  const V r45 = vmul(vc<V>(4.5), rho), f9 = vmul(vc<V>(9.0), fpre), o45 = vmul(vc<V>(4.5), om);
  const V r3x = vmul(vc<V>(3.0), rho), f3 = vmul(vc<V>(3.0), fpre);
  static_for<9>([&](auto Pi) {
    constexpr int p = Pi;
    constexpr int q = 2 * p + 1;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    const V cu = vdot<V, cx, cy, cz>(ux, uy, uz);
    const V cF = vdot<V, cx, cy, cz>(Fx, Fy, Fz);
    V qn = vc<V>(0.0);
    bool first = true;
    auto add = [&](V x) {
      qn = first ? x : vadd(qn, x);
      first = false;
    };
    if constexpr (cx != 0) add(Nxx);
    if constexpr (cy != 0) add(Nyy);
    if constexpr (cz != 0) add(Nzz);
    if constexpr (cx != 0 && cy != 0) qn = vfma(vc<V>(2 * cx * cy), Nxy, qn);
    if constexpr (cx != 0 && cz != 0) qn = vfma(vc<V>(2 * cx * cz), Nxz, qn);
    if constexpr (cy != 0 && cz != 0) qn = vfma(vc<V>(2 * cy * cz), Nyz, qn);
    // even part: E0 + cu (4.5 rho cu + 9 fpre cF) + 4.5 om qn
    const V ev = vfma(cu, vfma(r45, cu, vmul(f9, cF)), vfma(o45, qn, E0));
    // odd part: 3 (rho cu + fpre cF)
    const V od = vfma(r3x, cu, vmul(f3, cF));
    put_f(std::integral_constant<int, q>{}, vadd(ev, od));
    put_f(std::integral_constant<int, q + 1>{}, vsub(ev, od));
  });
  const V omg = vrcp(taug);
  const V a = vsub(vc<V>(1.0), omg), one_sg = vsub(vc<V>(1.0), sg);
  const V omth = vmul(omg, m.th);
  put_g(std::integral_constant<int, 0>{}, vmul(vfma(a, g[0], vmul(vc<V>(w7(0)), vadd(omth, Ssrc))), one_sg));
  static_for<3>([&](auto Pi) {
    constexpr int p = Pi;
    constexpr int q = 2 * p + 1;
    constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    const V w = vc<V>(w7(q));
    const V b = vmul(w, vadd(omth, Ssrc));
    const V c4 = vmul(vmul(vc<V>(4.0 * w7(q)), omth), vdot<V, cx, cy, cz>(ux, uy, uz));
    put_g(std::integral_constant<int, q>{}, vmul(vadd(vfma(a, g[q], b), c4), one_sg));
    put_g(std::integral_constant<int, q + 1>{}, vmul(vsub(vfma(a, g[q + 1], b), c4), one_sg));
  });
  o.Fx = Fx;
  o.Fy = Fy;
  o.Fz = Fz;
  o.ux = ux;
  o.uy = uy;
  o.uz = uz;
}

}  // namespace ahx
