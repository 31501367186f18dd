// ORACLE — test infrastructure, not product code.
//
// CPU restatement of the live solver's device kernels, generated in the reference as WGSL by js/live/kernel.js
// (alanhuang116/ashburn-heat-twin). Only the tests, the smoke check and the benchmark's CPU-baseline leg load this
// library: it is the checker the CUDA path is compared with, and the timed CPU baseline. The product never links it.
//
// Every function follows one generated WGSL kernel section by section, in the same order of operations, with the
// same literals rounded the same way (kernel.js:31-33 fmt(): float32-rounded decimal), and no floating-point
// contraction (build with -ffp-contract=off). Storage layout is the reference's: populations [q][cell] with
// cell = (k*ny + j)*nx + i, j = 0 at the south edge (kernel.js:17).
//
// Two arithmetic builds from one template: Real = float (the reference arithmetic, f32 everywhere) and Real = double
// (the FP64 precision oracle; parameters are the same f32 block widened to f64, lattice weights exact in f64).
//
// Pinning: the FP32 build reproduces the reference's archived scalar results (tests/live/validation_summary.json of
// the reference: read().thetaMax, surfMean, windMean after 300..2300 steps on the real Ashburn domain) — see the
// tests under tests/ that load this library.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>
#include <xmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Subnormal f32 values are flushed to zero (inputs and results), as the CUDA path does (-ftz=true): the WGSL
// reference runs with the GPU's f32 denormal mode, where flushing is the norm, and on the CPU subnormal arithmetic
// would otherwise be orders of magnitude slower. Every parallel region holds one of these per thread: it sets
// flush-to-zero and denormals-are-zero (MXCSR bits 15 and 6) for the region and restores the thread's previous mode
// when the region ends, so the calling process (numpy, the host metrics) keeps its own floating-point mode.
struct FlushSubnormals {
  unsigned saved;
  FlushSubnormals() : saved(_mm_getcsr()) { _mm_setcsr(saved | 0x8040u); }
  ~FlushSubnormals() { _mm_setcsr(saved); }
  FlushSubnormals(const FlushSubnormals&) = delete;
  FlushSubnormals& operator=(const FlushSubnormals&) = delete;
};

// lattice tables (kernel.js:19-28); OPP/MIRZ derived as the reference derives them (find the reversed / z-mirrored
// velocity), weights as the reference's f64 fractions
constexpr int C19[19][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                            {1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1}, {-1, 0, -1}, {1, 0, -1},
                            {-1, 0, 1}, {0, 1, 1}, {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};
constexpr int C7[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

constexpr int find19(int a, int b, int c) {
  for (int q = 0; q < 19; ++q)
    if (C19[q][0] == a && C19[q][1] == b && C19[q][2] == c) return q;
  return -1;
}
constexpr int find7(int a, int b, int c) {
  for (int q = 0; q < 7; ++q)
    if (C7[q][0] == a && C7[q][1] == b && C7[q][2] == c) return q;
  return -1;
}
constexpr int OPP19(int q) { return find19(-C19[q][0], -C19[q][1], -C19[q][2]); }
constexpr int MIRZ19(int q) { return find19(C19[q][0], C19[q][1], -C19[q][2]); }
constexpr int OPP7(int q) { return find7(-C7[q][0], -C7[q][1], -C7[q][2]); }
constexpr double W19d(int q) { return q == 0 ? 1.0 / 3 : (q < 7 ? 1.0 / 18 : 1.0 / 36); }
constexpr double W7d(int q) { return q == 0 ? 1.0 / 4 : 1.0 / 8; }

// compile-time loop over q = 0..N-1 (the reference's generator unrolls every q loop into straight-line WGSL)
template <int... Qs, class F>
inline void static_for_impl(std::integer_sequence<int, Qs...>, F&& f) {
  (f(std::integral_constant<int, Qs>{}), ...);
}
template <int N, class F>
inline void static_for(F&& f) {
  static_for_impl(std::make_integer_sequence<int, N>{}, f);
}

// Params block (kernel.js:44-50): 16 x 4-byte scalars then nz x vec4<f32> (uin, vin, kbg, 0)
struct Params {
  float tau0, cs2smag, gbeta, prt, kfloor, momfac, srcscale, sigmax;
  int32_t inflow_w, inflow_e, inflow_s, inflow_n, nsp, nsw, oclip, pad1;
  const float* prof;
};

Params parse_params(const void* blk) {
  Params P;
  std::memcpy(&P, blk, 64);
  P.prof = reinterpret_cast<const float*>(static_cast<const char*>(blk) + 64);
  return P;
}

template <class R>
struct Grid {
  int NX, NY, NZ;
  long N, NXY;
  Params P;
  const uint32_t* colv;   // 4 x u32 per column
  const uint32_t* ktopc;  // u32 per column
};

// sum of the terms of a moment: q in order, sign by c[comp] (kernel.js:245-252 mom(); 127-134 prelude)
template <class R, int comp, class F>
inline R first_moment(const F& fq) {
  R acc = 0;
  bool first = true;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int c = C19[q][comp];
    if constexpr (c != 0) {
      const R v = fq(q);
      if (first) acc = c > 0 ? v : -v;
      else acc = c > 0 ? acc + v : acc - v;
      first = false;
    }
  });
  return acc;
}

// mom2(p, r) (kernel.js:254-262)
template <class R, int p, int r>
inline R second_moment(const R* f) {
  R acc = 0;
  bool first = true;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int v = C19[q][p] * C19[q][r];
    if constexpr (v != 0) {
      if (first) acc = v > 0 ? f[q] : -f[q];
      else acc = v > 0 ? acc + f[q] : acc - f[q];
      first = false;
    }
  });
  return acc;
}

// (cx)*a + (cy)*b + (cz)*c over the nonzero components in x, y, z order; 0.0 if none (kernel.js:184-199,342-345)
template <class R, int cx, int cy, int cz>
inline R cdot(R a, R b, R c) {
  R acc = 0;
  bool first = true;
  if constexpr (cx != 0) { acc = R(cx) * a; first = false; }
  if constexpr (cy != 0) { acc = first ? R(cy) * b : acc + R(cy) * b; first = false; }
  if constexpr (cz != 0) { acc = first ? R(cz) * c : acc + R(cz) * c; first = false; }
  (void)first;
  return acc;
}

// inflowCond (kernel.js:150-157)
template <int cx, int cy>
inline bool inflow_cond(const Params& P, int si, int sj, int NX, int NY) {
  bool r = false;
  if constexpr (cx == 1) r = r || (si < 0 && P.inflow_w != 0);
  if constexpr (cx == -1) r = r || (si >= NX && P.inflow_e != 0);
  if constexpr (cy == 1) r = r || (sj < 0 && P.inflow_s != 0);
  if constexpr (cy == -1) r = r || (sj >= NY && P.inflow_n != 0);
  return r;
}

// State of one cell after the stream phase (pre-collision), shared by step / surf.
template <class R>
struct Streamed {
  R f[19], g[7];
  int ktc, kg, zagl;
  R uI, vI;
};

// secProfile + secNeighbourCache + secOutflowPrelude + secStreamF + secStreamG (kernel.js:102-243)
template <class R>
void stream_cell(const Grid<R>& G, const R* fA, const R* gA, int i, int j, int k, Streamed<R>& S) {
  const int NX = G.NX, NY = G.NY, NZ = G.NZ;
  const long N = G.N;
  const Params& P = G.P;
  const long n = ((long)k * NY + j) * NX + i;
  const long col = (long)j * NX + i;
  const int ktc = (int)G.colv[4 * col + 0];
  const int kg = (int)G.colv[4 * col + 1];
  S.ktc = ktc;
  S.kg = kg;
  // secProfile
  int zagl = k - ktc;
  if (zagl < 0) zagl = 0;
  S.zagl = zagl;
  const R uI = R(P.prof[4 * zagl + 0]);
  const R vI = R(P.prof[4 * zagl + 1]);
  S.uI = uI;
  S.vI = vI;
  // secNeighbourCache (cacheNbr = true)
  const int im = std::max(i - 1, 0), ip = std::min(i + 1, NX - 1), jm = std::max(j - 1, 0),
            jp = std::min(j + 1, NY - 1);
  const int xs[3] = {im, i, ip}, ys[3] = {jm, j, jp};
  int kn[3][3];
  for (int ox = -1; ox <= 1; ++ox)
    for (int oy = -1; oy <= 1; ++oy)
      kn[ox + 1][oy + 1] = (ox == 0 && oy == 0) ? kg : (int)G.ktopc[(long)ys[oy + 1] * NX + xs[ox + 1]];
  // secOutflowPrelude
  R rn = 1, uxn = 0, uyn = 0, uzn = 0;
  const bool onb = (i == 0 && P.inflow_w == 0) || (i == NX - 1 && P.inflow_e == 0) || (j == 0 && P.inflow_s == 0) ||
                   (j == NY - 1 && P.inflow_n == 0);
  auto own = [&](int q) { return fA[(long)q * N + n]; };
  if (onb) {
    rn = own(0);
    for (int q = 1; q < 19; ++q) rn = rn + own(q);
    uxn = first_moment<R, 0>(own) / rn;
    uyn = first_moment<R, 1>(own) / rn;
    uzn = first_moment<R, 2>(own) / rn;
  }
  const R usqn = uxn * uxn + uyn * uyn + uzn * uzn;
  R uxc = uxn, uyc = uyn;
  if (P.oclip != 0) {
    if (i == 0 && P.inflow_w == 0 && uxc > R(0)) uxc = 0;
    if (i == NX - 1 && P.inflow_e == 0 && uxc < R(0)) uxc = 0;
    if (j == 0 && P.inflow_s == 0 && uyc > R(0)) uyc = 0;
    if (j == NY - 1 && P.inflow_n == 0 && uyc < R(0)) uyc = 0;
  }
  const R usqc = uxc * uxc + uyc * uyc + uzn * uzn;
  // secStreamF
  S.f[0] = fA[n];
  static_for<18>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = C19[q][0], cy = C19[q][1], cz = C19[q][2];
    const R w = R(W19d(q));
    const int si = i - cx, sj = j - cy, sk = k - cz;
    const bool outx = (si < 0) || (si >= NX);
    const bool outy = (sj < 0) || (sj >= NY);
    R fv;
    if (sk >= NZ) {
      // free-slip lid: mirrored population from the same layer
      constexpr int m = MIRZ19(q);
      const int ti = si, tj = sj;
      if (ti < 0 || ti >= NX || tj < 0 || tj >= NY) {
        fv = fA[(long)m * N + n];
      } else {
        const long t = ((long)k * NY + tj) * NX + ti;
        if (k < kn[-cx + 1][-cy + 1]) fv = fA[(long)m * N + n];
        else fv = fA[(long)m * N + t];
      }
    } else if (outx || outy) {
      if (inflow_cond<cx, cy>(P, si, sj, NX, NY)) {
        const R cu = cdot<R, cx, cy, 0>(uI, vI, R(0));
        fv = w * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * (uI * uI + vI * vI));
      } else {
        const R cu = cdot<R, cx, cy, cz>(uxn, uyn, uzn);
        if (P.oclip != 0) {
          const R cuc = cdot<R, cx, cy, cz>(uxc, uyc, uzn);
          fv = fA[(long)q * N + n] + w * ((R(1.0) + R(3.0) * cuc + R(4.5) * cuc * cuc - R(1.5) * usqc) -
                                          rn * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usqn));
        } else {
          fv = fA[(long)q * N + n] + w * (R(1.0) - rn) * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usqn);
        }
      }
    } else {
      const long s = ((long)sk * NY + sj) * NX + si;
      if (sk < kn[-cx + 1][-cy + 1]) fv = fA[(long)OPP19(q) * N + n];
      else fv = fA[(long)q * N + s];
    }
    S.f[q] = fv;
  });
  // secStreamG
  S.g[0] = gA[n];
  static_for<6>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = C7[q][0], cy = C7[q][1], cz = C7[q][2];
    const int si = i - cx, sj = j - cy, sk = k - cz;
    R gv;
    if (sk >= NZ) {
      gv = gA[(long)q * N + n];
    } else if (si < 0 || si >= NX || sj < 0 || sj >= NY) {
      if (inflow_cond<cx, cy>(P, si, sj, NX, NY)) gv = 0;
      else gv = gA[(long)q * N + n];
    } else {
      const long s = ((long)sk * NY + sj) * NX + si;
      if (sk < kn[-cx + 1][-cy + 1]) gv = gA[(long)OPP7(q) * N + n];
      else gv = gA[(long)q * N + s];
    }
    S.g[q] = gv;
  });
}

template <class R>
struct Moments {
  R rho, jx, jy, jz, th, Pxx, Pyy, Pzz, Pxy, Pxz, Pyz;
};

// secMoments (kernel.js:264-277)
template <class R>
void moments(const Streamed<R>& S, bool second, Moments<R>& M) {
  M.rho = S.f[0];
  for (int q = 1; q < 19; ++q) M.rho = M.rho + S.f[q];
  auto fq = [&](int q) { return S.f[q]; };
  M.jx = first_moment<R, 0>(fq);
  M.jy = first_moment<R, 1>(fq);
  M.jz = first_moment<R, 2>(fq);
  M.th = S.g[0];
  for (int q = 1; q < 7; ++q) M.th = M.th + S.g[q];
  if (!second) return;
  M.Pxx = second_moment<R, 0, 0>(S.f);
  M.Pyy = second_moment<R, 1, 1>(S.f);
  M.Pzz = second_moment<R, 2, 2>(S.f);
  M.Pxy = second_moment<R, 0, 1>(S.f);
  M.Pxz = second_moment<R, 0, 2>(S.f);
  M.Pyz = second_moment<R, 1, 2>(S.f);
}

template <class R>
struct Forces {
  R Fx, Fy, Fz, sg, ux, uy, uz;
};

// secForces (kernel.js:279-306)
template <class R>
void forces(const Grid<R>& G, const Streamed<R>& S, const Moments<R>& M, R cd, int k, Forces<R>& F) {
  const Params& P = G.P;
  const int NZ = G.NZ;
  const R rho = M.rho, jx = M.jx, jy = M.jy, jz = M.jz;
  R Fx = 0, Fy = 0;
  R Fz = rho * R(P.gbeta) * M.th;
  if (k == S.kg && S.kg == S.ktc) {
    const R ux0 = jx / rho, uy0 = jy / rho;
    const R sp = std::sqrt(ux0 * ux0 + uy0 * uy0);
    Fx = -rho * cd * sp * ux0;
    Fy = -rho * cd * sp * uy0;
    const R lim = R(0.5) * rho;
    if (cd * sp > R(0.5)) {
      Fx = -lim * ux0;
      Fy = -lim * uy0;
    }
  }
  R sg = 0;
  if (k >= NZ - P.nsp) {
    const R aa = (R(k - (NZ - P.nsp)) + R(1.0)) / R(P.nsp);
    sg = R(P.sigmax) * aa * aa;
    Fx += rho * sg * (S.uI - jx / rho);
    Fy += rho * sg * (S.vI - jy / rho);
    Fz += -rho * sg * (jz / rho);
  }
  F.Fx = Fx;
  F.Fy = Fy;
  F.Fz = Fz;
  F.sg = sg;
  F.ux = (jx + R(0.5) * Fx) / rho;
  F.uy = (jy + R(0.5) * Fy) / rho;
  F.uz = (jz + R(0.5) * Fz) / rho;
}

// One full fused step of cell (i, j, k): kernel.js:395-431 (genStepWGSL main)
template <class R>
void step_cell(const Grid<R>& G, const R* fA, R* fB, const R* gA, R* gB, R* dbg, int mode, int i, int j, int k) {
  const int NX = G.NX, NY = G.NY;
  const long N = G.N;
  const Params& P = G.P;
  const long col = (long)j * NX + i;
  const int kg = (int)G.colv[4 * col + 1];
  if (k < kg) return;  // flag[n] != 0
  const long n = ((long)k * NY + j) * NX + i;
  Streamed<R> S;
  stream_cell(G, fA, gA, i, j, k, S);
  Moments<R> M;
  moments(S, true, M);
  float cdf;
  std::memcpy(&cdf, &G.colv[4 * col + 2], 4);
  Forces<R> F;
  forces(G, S, M, R(cdf), k, F);
  const R rho = M.rho, ux = F.ux, uy = F.uy, uz = F.uz, Fx = F.Fx, Fy = F.Fy, Fz = F.Fz;
  // secRelax (kernel.js:308-338)
  const R usq = ux * ux + uy * uy + uz * uz;
  const R r3 = rho * R(1.0 / 3.0);
  const R Nxx = M.Pxx - r3 - rho * ux * ux;
  const R Nyy = M.Pyy - r3 - rho * uy * uy;
  const R Nzz = M.Pzz - r3 - rho * uz * uz;
  const R Nxy = M.Pxy - rho * ux * uy;
  const R Nxz = M.Pxz - rho * ux * uz;
  const R Nyz = M.Pyz - rho * uy * uz;
  const R Pn = std::sqrt(Nxx * Nxx + Nyy * Nyy + Nzz * Nzz + R(2.0) * (Nxy * Nxy + Nxz * Nxz + Nyz * Nyz));
  const R kb = R(P.prof[4 * S.zagl + 2]);
  R tb = R(P.tau0) + R(3.0) * R(P.momfac) * kb;
  int dmin = 1000;
  if (P.inflow_w == 0 && i < dmin) dmin = i;
  if (P.inflow_e == 0 && NX - 1 - i < dmin) dmin = NX - 1 - i;
  if (P.inflow_s == 0 && j < dmin) dmin = j;
  if (P.inflow_n == 0 && NY - 1 - j < dmin) dmin = NY - 1 - j;
  if (dmin < P.nsw) {
    const R rr = (R(P.nsw) - R(dmin)) / R(P.nsw);
    tb += R(0.15) * rr * rr;
  }
  const R tau = R(0.5) * (tb + std::sqrt(tb * tb + R(P.cs2smag) * Pn / rho));
  const R nusgs = (tau - tb) * R(1.0 / 3.0);
  const R kap = nusgs / R(P.prt) + kb + R(P.kfloor);
  const R taug = R(0.5) + R(4.0) * kap;
  const R om = R(1.0) - R(1.0) / tau;
  const R fpre = R(1.0) - R(0.5) / tau;
  const R trN = (Nxx + Nyy + Nzz) * R(1.0 / 3.0);
  // secCollision (kernel.js:340-367)
  const R uF = ux * Fx + uy * Fy + uz * Fz;   // the same subexpression in every q
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = C19[q][0], cy = C19[q][1], cz = C19[q][2];
    const R w = R(W19d(q));
    const R w45 = R(4.5 * W19d(q));
    const R cu = cdot<R, cx, cy, cz>(ux, uy, uz);
    const R feq = w * rho * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usq);
    // Q:Pi^neq: Nxx/Nyy/Nzz for the nonzero components, then the cross terms 2*(c_a c_b)*N_ab
    R qn = 0;
    bool first = true;
    auto addq = [&](R v) {
      qn = first ? v : qn + v;
      first = false;
    };
    if constexpr (cx != 0) addq(Nxx);
    if constexpr (cy != 0) addq(Nyy);
    if constexpr (cz != 0) addq(Nzz);
    if constexpr (cx != 0 && cy != 0) addq(R(2.0) * R(cx * cy) * Nxy);
    if constexpr (cx != 0 && cz != 0) addq(R(2.0) * R(cx * cz) * Nxz);
    if constexpr (cy != 0 && cz != 0) addq(R(2.0) * R(cy * cz) * Nyz);
    const R fr = w45 * (qn - trN);
    const R cF = cdot<R, cx, cy, cz>(Fx, Fy, Fz);
    const R Fq = fpre * w * (R(3.0) * (cF - uF) + R(9.0) * cu * cF);
    fB[(long)q * N + n] = feq + om * fr + Fq;
  });
  // secScalarCollision (kernel.js:369-386)
  R Ssrc = 0;
  if (k == S.kg) {
    float qf;
    std::memcpy(&qf, &G.colv[4 * col + 3], 4);
    Ssrc = R(qf) * R(P.srcscale);
  }
  const R omg = R(1.0) / taug;
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = C7[q][0], cy = C7[q][1], cz = C7[q][2];
    const R w = R(W7d(q));
    const R geq = w * M.th * (R(1.0) + R(4.0) * cdot<R, cx, cy, cz>(ux, uy, uz));
    gB[(long)q * N + n] = (S.g[q] + omg * (geq - S.g[q]) + w * Ssrc) * (R(1.0) - F.sg);
  });
  if (mode == 1) {
    dbg[4 * n + 0] = M.th;
    dbg[4 * n + 1] = ux;
    dbg[4 * n + 2] = uy;
    dbg[4 * n + 3] = uz;
  } else if (mode == 2) {
    dbg[4 * n + 0] = dbg[4 * n + 0] + M.th;
    dbg[4 * n + 1] = dbg[4 * n + 1] + ux;
    dbg[4 * n + 2] = dbg[4 * n + 2] + uy;
    dbg[4 * n + 3] = dbg[4 * n + 3] + uz;
  }
}

template <class R>
Grid<R> make_grid(int nx, int ny, int nz, const void* params, const uint32_t* colv, const uint32_t* ktopc) {
  Grid<R> G;
  G.NX = nx;
  G.NY = ny;
  G.NZ = nz;
  G.NXY = (long)nx * ny;
  G.N = G.NXY * nz;
  G.P = parse_params(params);
  G.colv = colv;
  G.ktopc = ktopc;
  return G;
}

template <class R>
void step_all(int nx, int ny, int nz, const void* params, const uint32_t* colv, const uint32_t* ktopc, const R* fA,
              R* fB, const R* gA, R* gB, R* dbg, int mode) {
  const Grid<R> G = make_grid<R>(nx, ny, nz, params, colv, ktopc);
#pragma omp parallel
  {
    const FlushSubnormals ftz;
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) step_cell(G, fA, fB, gA, gB, dbg, mode, i, j, k);
  }
}

// genInitWGSL (kernel.js:524-553): equilibrium with the inflow profile at the local height above terrain
template <class R>
void init_all(int nx, int ny, int nz, const void* params, const uint32_t* colv, R* f0, R* f1) {
  const Params P = parse_params(params);
  const long NXY = (long)nx * ny, N = NXY * nz;
#pragma omp parallel
  {
  const FlushSubnormals ftz;
#pragma omp for schedule(static)
  for (long n = 0; n < N; ++n) {
    const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / NXY);
    const int ktc = (int)colv[4 * ((long)j * nx + i)];
    const int zagl = std::min(std::max(k - ktc, 0), nz - 1);
    const R U = R(P.prof[4 * zagl + 0]), V = R(P.prof[4 * zagl + 1]);
    const R usq = U * U + V * V;
    static_for<19>([&](auto Q) {
      constexpr int q = Q;
      const R cu = R(C19[q][0]) * U + R(C19[q][1]) * V;
      const R fq = R(W19d(q)) * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usq);
      f0[(long)q * N + n] = fq;
      if (f1) f1[(long)q * N + n] = fq;
    });
  }
  }
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// mode: 0 plain step, 1 write (theta, ux, uy, uz) to dbg, 2 accumulate into dbg (kernel.js:427-428)
void orc_step_f32(int nx, int ny, int nz, const void* params, const uint32_t* colv, const uint32_t* ktopc,
                  const float* fA, float* fB, const float* gA, float* gB, float* dbg, int mode) {
  step_all<float>(nx, ny, nz, params, colv, ktopc, fA, fB, gA, gB, dbg, mode);
}

void orc_step_f64(int nx, int ny, int nz, const void* params, const uint32_t* colv, const uint32_t* ktopc,
                  const double* fA, double* fB, const double* gA, double* gB, double* dbg, int mode) {
  step_all<double>(nx, ny, nz, params, colv, ktopc, fA, fB, gA, gB, dbg, mode);
}

void orc_init_f32(int nx, int ny, int nz, const void* params, const uint32_t* colv, float* f0, float* f1) {
  init_all<float>(nx, ny, nz, params, colv, f0, f1);
}

void orc_init_f64(int nx, int ny, int nz, const void* params, const uint32_t* colv, double* f0, double* f1) {
  init_all<double>(nx, ny, nz, params, colv, f0, f1);
}

// genSurfWGSL (kernel.js:435-471): pre-collision theta and force-corrected u, v (times conv) in the first fluid cell
// of every column, north-up; zeros where ktop >= nz
void orc_surf_f32(int nx, int ny, int nz, const void* params, const uint32_t* colv, const uint32_t* ktopc,
                  const float* fA, const float* gA, float conv, float* sout) {
  const Grid<float> G = make_grid<float>(nx, ny, nz, params, colv, ktopc);
  const long NXY = G.NXY;
#pragma omp parallel
  {
  const FlushSubnormals ftz;
#pragma omp for schedule(static)
  for (long c = 0; c < NXY; ++c) {
    const int i = (int)(c % nx), j = (int)(c / nx);
    const int kg = (int)colv[4 * c + 1];
    const int k = kg;
    const long o = (long)(ny - 1 - j) * nx + i;
    if (k >= nz) {
      sout[o] = 0.f;
      sout[NXY + o] = 0.f;
      sout[2 * NXY + o] = 0.f;
      continue;
    }
    Streamed<float> S;
    stream_cell(G, fA, gA, i, j, k, S);
    Moments<float> M;
    moments(S, false, M);
    float cdf;
    std::memcpy(&cdf, &colv[4 * c + 2], 4);
    Forces<float> F;
    forces(G, S, M, cdf, k, F);
    sout[o] = M.th;
    sout[NXY + o] = F.ux * conv;
    sout[2 * NXY + o] = F.uy * conv;
  }
  }
}

// genVolWGSL (kernel.js:475-520): theta of the lowest nzv levels, north-up [k][row][col], u8 round(theta*volscale)
// clamped to 0..255, 4 per u32 little-endian; max theta (>= 0) of those cells into *tmax
void orc_vol_f32(int nx, int ny, int nz, const void* params, const uint32_t* ktopc, const float* gA, int nzv,
                 float volscale, uint32_t* vout, float* tmax) {
  const Params P = parse_params(params);
  const long NXY = (long)nx * ny, N = NXY * nz, NVOL = (long)nzv * NXY, NW = (NVOL + 3) / 4;
  float gmax = 0.f;
#pragma omp parallel reduction(max : gmax)
  {
  const FlushSubnormals ftz;
#pragma omp for schedule(static)
  for (long t = 0; t < NW; ++t) {
    uint32_t packed = 0;
    float tm = 0.f;
    for (int e = 0; e < 4; ++e) {
      const long p = 4 * t + e;
      if (p >= NVOL) continue;
      const int k = (int)(p / NXY);
      const long rem = p % NXY;
      const int i = (int)(rem % nx);
      const int j = ny - 1 - (int)(rem / nx);
      const int kg = (int)ktopc[(long)j * nx + i];
      float th = 0.f;
      if (k >= kg) {
        const long n = ((long)k * ny + j) * nx + i;
        float g[7];
        g[0] = gA[n];
        static_for<6>([&](auto Qm1) {
          constexpr int q = Qm1 + 1;
          constexpr int cx = C7[q][0], cy = C7[q][1], cz = C7[q][2];
          const int si = i - cx, sj = j - cy, sk = k - cz;
          float gv;
          if (sk >= nz) {
            gv = gA[(long)q * N + n];
          } else if (si < 0 || si >= nx || sj < 0 || sj >= ny) {
            gv = inflow_cond<cx, cy>(P, si, sj, nx, ny) ? 0.f : gA[(long)q * N + n];
          } else {
            const long s = ((long)sk * ny + sj) * nx + si;
            if (sk < (int)ktopc[(long)sj * nx + si]) gv = gA[(long)OPP7(q) * N + n];
            else gv = gA[(long)q * N + s];
          }
          g[q] = gv;
        });
        th = g[0];
        for (int q = 1; q < 7; ++q) th = th + g[q];
      }
      const float r = std::nearbyint(th * volscale);   // WGSL round(): half to even
      const uint32_t qv = (uint32_t)std::min(std::max(r, 0.f), 255.f);
      packed |= qv << (8u * (uint32_t)e);
      tm = std::max(tm, th);
    }
    vout[t] = packed;
    gmax = std::max(gmax, std::max(tm, 0.f));
  }
  }
  *tmax = gmax;
}

// genReinitWGSL (kernel.js:557-575): cells that turned from solid to fluid get rest equilibrium and theta = 0
void orc_reinit_f32(int nx, int ny, int nz, const uint32_t* ktopc, const uint32_t* oldk, float* f, float* g) {
  const FlushSubnormals ftz;
  const long NXY = (long)nx * ny, N = NXY * nz;
  for (long c = 0; c < NXY; ++c) {
    const int k1 = std::min((int)oldk[c], nz);
    for (int k = (int)ktopc[c]; k < k1; ++k) {
      const long n = (long)k * NXY + c;
      for (int q = 0; q < 19; ++q) f[(long)q * N + n] = float(W19d(q));
      for (int q = 0; q < 7; ++q) g[(long)q * N + n] = 0.f;
    }
  }
}

// genStatsWGSL (kernel.js:580-633) over all fluid cells of the stored state: per-cell f32 values
// (theta, 0.5|j|^2/rho, rho - 1, 1) summed in f64; max theta (>= 0); count of non-finite rho or theta;
// max |j|/rho. out[0..3] sums, out[4] theta max, out[5] non-finite count, out[6] umax (lattice units)
void orc_stats_f32(int nx, int ny, int nz, const uint32_t* ktopc, const float* fA, const float* gA, double* out) {
  const long NXY = (long)nx * ny, N = NXY * nz;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0, nonf = 0;
  float tmax = 0.f, umax = 0.f;
#pragma omp parallel reduction(+ : s0, s1, s2, s3, nonf) reduction(max : tmax, umax)
  {
  const FlushSubnormals ftz;
#pragma omp for schedule(static)
  for (long n = 0; n < N; ++n) {
    const int i = (int)(n % nx), j = (int)((n / nx) % ny), k = (int)(n / NXY);
    if (k < (int)ktopc[(long)j * nx + i]) continue;
    auto fq = [&](int q) { return fA[(long)q * N + n]; };
    float rho = fq(0);
    for (int q = 1; q < 19; ++q) rho = rho + fq(q);
    const float jx = first_moment<float, 0>(fq), jy = first_moment<float, 1>(fq), jz = first_moment<float, 2>(fq);
    float th = gA[n];
    for (int q = 1; q < 7; ++q) th = th + gA[(long)q * N + n];
    if (!std::isfinite(rho) || !std::isfinite(th)) {
      nonf += 1;
      continue;
    }
    s0 += th;
    s1 += 0.5f * (jx * jx + jy * jy + jz * jz) / rho;
    s2 += rho - 1.0f;
    s3 += 1.0;
    tmax = std::max(tmax, std::max(th, 0.f));
    umax = std::max(umax, std::sqrt(jx * jx + jy * jy + jz * jz) / rho);
  }
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  out[3] = s3;
  out[4] = tmax;
  out[5] = nonf;
  out[6] = umax;
}

}  // extern "C"
