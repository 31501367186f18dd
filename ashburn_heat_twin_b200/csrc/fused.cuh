// The fused D3Q19 + D3Q7 stream-collide step of the live solver for sm_100a, and the pre-collision moment
// extraction the near-surface read-back uses.
//
// Algorithm: js/live/kernel.js of the reference, genStepWGSL (kernel.js:395-431) with its sections secProfile
// (:112-120), secNeighbourCache (:102-110), secOutflowPrelude (:122-148), secStreamF (:159-217), secStreamG
// (:219-243), secMoments (:264-277), secForces (:279-306), secRelax (:308-338), secCollision (:340-367),
// secScalarCollision (:369-386). Every floating-point expression keeps the reference's operand order; compiled with
// -fmad=false the result is the reference arithmetic with IEEE-rounded f32 operations.
//
// B200 mapping (not the reference's one-thread-per-cell linear dispatch):
//   * one thread per (i, j) column walking a z-slab [k0, k1): the column record, the 3x3 neighbour ktop cache, the
//     face flags and the outflow-sponge term are loaded / computed once per column instead of once per cell, and
//     solid cells below ktop are skipped without a launch slot;
//   * a warp is 32 consecutive i of one row, rows are 128-byte aligned (pitch px), so each population plane is read
//     and written as full 128-byte lines (the +-1 x shifts of the pull touch one extra sector, served by L1/L2);
//   * the boundary rules of the stream become an index remap: every population is one unconditional load from
//     (source plane, source cell) where bounce-back and the free-slip lid only change the plane and the cell; the
//     in/outflow faces (a thin set of columns) patch the loaded own value afterwards. So all 26 loads of a cell are
//     independent and in flight together;
//   * reads use the non-coherent path (the source buffer is read-only during a step), writes are streaming stores.
#pragma once

#include <type_traits>

#include "lattice.cuh"
#include "lanes.cuh"

namespace ahx {

template <class R, int cx, int cy, int cz>
__device__ __forceinline__ R cdot(R a, R b, R c) {
  // (cx)*a + (cy)*b + (cz)*c over the nonzero components, x y z order; 0 if none (kernel.js:184-199, 342-345)
  R acc = R(0);
  bool first = true;
  if constexpr (cx != 0) { acc = R(cx) * a; first = false; }
  if constexpr (cy != 0) { acc = first ? R(cy) * b : acc + R(cy) * b; first = false; }
  if constexpr (cz != 0) { acc = first ? R(cz) * c : acc + R(cz) * c; first = false; }
  (void)first;
  return acc;
}

// signed sum over q of the values whose c[comp] is +-1, in q order (kernel.js:245-252)
template <class R, int comp, class F>
__device__ __forceinline__ R moment1(const F& fq) {
  R acc = R(0);
  bool first = true;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int c = kC19[q][comp];
    if constexpr (c != 0) {
      const R v = fq(q);
      if (first) acc = (c > 0) ? v : -v;
      else acc = (c > 0) ? acc + v : acc - v;
      first = false;
    }
  });
  return acc;
}

// second moment Pi_pr in q order (kernel.js:254-262)
template <class R, int p, int r>
__device__ __forceinline__ R moment2(const R* f) {
  R acc = R(0);
  bool first = true;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int v = kC19[q][p] * kC19[q][r];
    if constexpr (v != 0) {
      if (first) acc = (v > 0) ? f[q] : -f[q];
      else acc = (v > 0) ? acc + f[q] : acc - f[q];
      first = false;
    }
  });
  return acc;
}

// Everything a column needs that does not depend on k.
template <class R>
struct Column {
  int i, j, ktc, kg;
  float cd, qsrc;
  int kn[3][3];          // ktop of the 3x3 neighbourhood, clamped at the edges (kernel.js:102-110)
  bool latW, latE, latS, latN;   // this column lies on the west / east / south / north face
  bool onb;              // on an outflow face: needs the outflow prelude (kernel.js:125)
  bool face;             // on any lateral face: some sources are outside the domain
  bool spon;             // inside the outflow viscous sponge (kernel.js:322-330)
  R spg;                 // 0.15*rr*rr of the sponge
  int kint;              // first level whose whole 3x3x3 neighbourhood is fluid (interior fast path from here)
};

// The column records and the ktop plane are read by every z-slab block of a column (and again by the single-level
// cells of the 16-bit paired kernels), a few MB against the GBs of populations streaming through L2 each step: their
// loads carry an L2 evict-last policy so they stay resident (a cache hint; no value changes).
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint4 ldg_keep(const uint4* p, uint64_t pol) {
  uint4 v;
  asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ldg_keep(const uint32_t* p, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

template <class R>
__device__ __forceinline__ void load_column(const DomainView& D, const ParamsHead& P, int i, int j, Column<R>& C) {
  const int nx = D.nx, ny = D.ny;
  const uint64_t pol = l2_keep_policy();
  const uint4 cv = ldg_keep(D.colv + (size_t)j * nx + i, pol);
  C.i = i;
  C.j = j;
  C.ktc = (int)cv.x;
  C.kg = (int)cv.y;
  C.cd = __uint_as_float(cv.z);
  C.qsrc = __uint_as_float(cv.w);
  const int im = max(i - 1, 0), ip = min(i + 1, nx - 1), jm = max(j - 1, 0), jp = min(j + 1, ny - 1);
  const int xs[3] = {im, i, ip}, ys[3] = {jm, j, jp};
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
      C.kn[ox][oy] = (ox == 1 && oy == 1) ? C.kg : (int)ldg_keep(D.ktop + (size_t)ys[oy] * nx + xs[ox], pol);
  int km = C.kg;
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy) km = max(km, C.kn[ox][oy]);
  C.kint = km + 1;
  const int jg = j + D.jg0, nyg = D.nyg;   // global row: faces and sponges follow the whole domain
  C.latW = (i == 0);
  C.latE = (i == nx - 1);
  C.latS = (jg == 0);
  C.latN = (jg == nyg - 1);
  C.face = C.latW || C.latE || C.latS || C.latN;
  C.onb = (C.latW && P.inflow_w == 0) || (C.latE && P.inflow_e == 0) || (C.latS && P.inflow_s == 0) ||
          (C.latN && P.inflow_n == 0);
  int dmin = 1000;
  if (P.inflow_w == 0 && i < dmin) dmin = i;
  if (P.inflow_e == 0 && nx - 1 - i < dmin) dmin = nx - 1 - i;
  if (P.inflow_s == 0 && jg < dmin) dmin = jg;
  if (P.inflow_n == 0 && nyg - 1 - jg < dmin) dmin = nyg - 1 - jg;
  C.spon = dmin < P.nsw;
  C.spg = R(0);
  if (C.spon) {
    const R rr = (R(P.nsw) - R(dmin)) / R(P.nsw);
    C.spg = R(0.15) * rr * rr;
  }
}

// is the source of direction (cx, cy) outside the domain for this column (kernel.js:166-167)
template <int cx, int cy, class R>
__device__ __forceinline__ bool lateral_out(const Column<R>& C) {
  bool r = false;
  if constexpr (cx == 1) r = r || C.latW;
  if constexpr (cx == -1) r = r || C.latE;
  if constexpr (cy == 1) r = r || C.latS;
  if constexpr (cy == -1) r = r || C.latN;
  return r;
}

// inflowCond (kernel.js:150-157), given that the source is outside
template <int cx, int cy, class R>
__device__ __forceinline__ bool inflow_cond(const Column<R>& C, const ParamsHead& P) {
  bool r = false;
  if constexpr (cx == 1) r = r || (C.latW && P.inflow_w != 0);
  if constexpr (cx == -1) r = r || (C.latE && P.inflow_e != 0);
  if constexpr (cy == 1) r = r || (C.latS && P.inflow_s != 0);
  if constexpr (cy == -1) r = r || (C.latN && P.inflow_n != 0);
  return r;
}

// Pre-collision state of one cell: the streamed populations plus the profile values used later.
template <class R>
struct Cell {
  R f[19], g[7];
  R uI, vI, kb;
};

// Round-to-nearest operations the compiler cannot contract. The face formulas below use them so the FMA build gives
// the same bits in every kernel variant (its contraction choices may differ between instantiations); in the exact
// build they evaluate exactly as the plain operators in the same order.
__device__ __forceinline__ float nmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float nadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float nsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double nmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double nadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double nsub(double a, double b) { return __dsub_rn(a, b); }

// 1 + 3 cu + 4.5 cu^2 - 1.5 usq, left to right as the reference writes it
template <class R>
__device__ __forceinline__ R feq_poly(R cu, R usq) {
  return nsub(nadd(nadd(R(1.0), nmul(R(3.0), cu)), nmul(nmul(R(4.5), cu), cu)), nmul(R(1.5), usq));
}

// The lateral-face rules of the stream for a cell of a face column (C.face), after its populations were loaded with
// every outside source taken from the own cell: secOutflowPrelude (kernel.js:122-148) and the in/outflow cases of
// secStreamF / secStreamG (kernel.js:187-204, 219-243). f and g are the decoded populations of cell n at level k (top:
// k is the lid level); nf is the cell's own element offset in an f plane (lvl). The formulas use non-contractible
// operations, so every kernel path gives the same bits.
template <class S>
__device__ __forceinline__ void face_patch(const DomainView& D, const ParamsHead& P, const Column<RealOf<S>>& C,
                                           bool top, uint32_t nf, RealOf<S> uI, RealOf<S> vI, RealOf<S> (&f)[19],
                                           RealOf<S> (&g)[7]) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  const StoreF<S>* fA = static_cast<const StoreF<S>*>(D.fA);
  const uint32_t qs = D.qs;
  // secOutflowPrelude (kernel.js:122-148): own-cell density and velocity on outflow faces
  R rn = R(1), uxn = R(0), uyn = R(0), uzn = R(0);
  if (C.onb) {
    R own[19];
    static_for<19>([&](auto Q) {
      constexpr int q = Q;
      own[q] = KF::dec_f(KF::load(fA + (uint32_t)q * qs + nf), R(w19(q)));
    });
    rn = own[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) rn = rn + own[q];
    auto fo = [&](int q) { return own[q]; };
    uxn = moment1<R, 0>(fo) / rn;
    uyn = moment1<R, 1>(fo) / rn;
    uzn = moment1<R, 2>(fo) / rn;
  }
  const R usqn = nadd(nadd(nmul(uxn, uxn), nmul(uyn, uyn)), nmul(uzn, uzn));
  R uxc = uxn, uyc = uyn;
  if (P.oclip != 0) {
    if (C.latW && P.inflow_w == 0 && uxc > R(0)) uxc = R(0);
    if (C.latE && P.inflow_e == 0 && uxc < R(0)) uxc = R(0);
    if (C.latS && P.inflow_s == 0 && uyc > R(0)) uyc = R(0);
    if (C.latN && P.inflow_n == 0 && uyc < R(0)) uyc = R(0);
  }
  const R usqc = nadd(nadd(nmul(uxc, uxc), nmul(uyc, uyc)), nmul(uzn, uzn));
  static_for<18>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    if constexpr (cx != 0 || cy != 0) {
      if (!(cz == -1 && top) && lateral_out<cx, cy>(C)) {
        const R w = R(w19(q));
        if (inflow_cond<cx, cy>(C, P)) {
          const R cu = cdot<R, cx, cy, 0>(uI, vI, R(0));
          f[q] = nmul(w, feq_poly(cu, nadd(nmul(uI, uI), nmul(vI, vI))));
        } else {
          const R cu = cdot<R, cx, cy, cz>(uxn, uyn, uzn);
          if (P.oclip != 0) {
            const R cuc = cdot<R, cx, cy, cz>(uxc, uyc, uzn);
            f[q] = nadd(f[q], nmul(w, nsub(feq_poly(cuc, usqc), nmul(rn, feq_poly(cu, usqn)))));
          } else {
            f[q] = nadd(f[q], nmul(nmul(w, nsub(R(1.0), rn)), feq_poly(cu, usqn)));
          }
        }
      }
    }
  });
  static_for<6>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    if constexpr (cx != 0 || cy != 0) {
      if (!(cz == -1 && top) && lateral_out<cx, cy>(C) && inflow_cond<cx, cy>(C, P)) g[q] = R(0);
    }
  });
}

// secProfile + secOutflowPrelude + secStreamF + secStreamG for cell (C.i, C.j, k); m = j px + i is the cell's
// row-column index in a level (element offsets through lvl).
template <class S>
__device__ __forceinline__ void stream_cell(const DomainView& D, const ParamsHead& P, const float4* prof,
                                            const Column<RealOf<S>>& C, int k, uint32_t m,
                                            Cell<RealOf<S>>& X) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  const StoreF<S>* fA = static_cast<const StoreF<S>*>(D.fA);
  const StoreG<S>* gA = static_cast<const StoreG<S>*>(D.gA);
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  const uint32_t qs = D.qs, ps = D.ps, px = (uint32_t)D.px;
  const uint32_t nf = lvl<TF>(k, m, ps), ng = lvl<TG>(k, m, ps);
  const bool top = (k == D.nz - 1);
  // secProfile
  int zagl = k - C.ktc;
  if (zagl < 0) zagl = 0;
  if (zagl > D.nz - 1) zagl = D.nz - 1;   // unreachable for valid columns (kt >= 1); keeps the index in bounds
  const float4 pr = prof[zagl];
  const R uI = R(pr.x), vI = R(pr.y);
  X.uI = uI;
  X.vI = vI;
  X.kb = R(pr.z);

  // secStreamF / secStreamG as an index remap: one load per population
  X.f[0] = KF::dec_f(KF::load(fA + nf), R(w19(0)));
  static_for<18>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    const int sk = k - cz;
    const bool lat = lateral_out<cx, cy>(C);
    uint32_t off;
    if (cz == -1 && top) {
      // free-slip lid: the z-mirrored population from the same layer, or the own cell's when the lateral source
      // is outside or solid (kernel.js:168-181)
      constexpr int mz = mirz19(q);
      const bool own = lat || (k < C.kn[1 - cx][1 - cy]);
      off = (uint32_t)mz * qs + (own ? nf : lvl_nbr<TF>(k, m, nf, 0, (uint32_t)(cx + cy * (int)px), ps));
    } else if (lat) {
      off = (uint32_t)q * qs + nf;   // in/outflow: patched below from the own value
    } else if (sk < C.kn[1 - cx][1 - cy]) {
      off = (uint32_t)opp19(q) * qs + nf;   // half-way bounce-back (kernel.js:209-210)
    } else {
      off = (uint32_t)q * qs + lvl_nbr<TF>(k, m, nf, cz, (uint32_t)(cx + cy * (int)px), ps);
    }
    X.f[q] = KF::dec_f(KF::load(fA + off), R(w19(q)));
  });
  X.g[0] = KG::dec_g(KG::load(gA + ng));
  static_for<6>([&](auto Qm1) {
    constexpr int q = Qm1 + 1;
    constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    const int sk = k - cz;
    const bool lat = lateral_out<cx, cy>(C);
    uint32_t off;
    if ((cz == -1 && top) || lat) {
      off = (uint32_t)q * qs + ng;   // zero-gradient lid / outflow: own value; inflow patched to 0 below
    } else if (sk < C.kn[1 - cx][1 - cy]) {
      off = (uint32_t)opp7(q) * qs + ng;
    } else {
      off = (uint32_t)q * qs + lvl_nbr<TG>(k, m, ng, cz, (uint32_t)(cx + cy * (int)px), ps);
    }
    X.g[q] = KG::dec_g(KG::load(gA + off));
  });

  if (C.face) face_patch<S>(D, P, C, top, nf, uI, vI, X.f, X.g);
}

// Interior cells (not on a lateral face, below the lid, every source fluid): the stream is a plain gather, one load
// per population at a fixed offset (level-paired planes: the source's lvl offset, which depends on the parity of the
// level); loads exactly the values stream_cell would.
template <class S>
__device__ __forceinline__ void stream_interior(const DomainView& D, const float4* prof,
                                                const Column<RealOf<S>>& C, int k, uint32_t m,
                                                Cell<RealOf<S>>& X) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  int zagl = k - C.ktc;
  if (zagl < 0) zagl = 0;
  if (zagl > D.nz - 1) zagl = D.nz - 1;
  const float4 pr = prof[zagl];
  X.uI = R(pr.x);
  X.vI = R(pr.y);
  X.kb = R(pr.z);
  const uint32_t ps = D.ps, px = (uint32_t)D.px, n = (uint32_t)k * ps + m;
  const uint32_t nf = lvl<TF>(k, m, ps), ng = lvl<TG>(k, m, ps);
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    [[maybe_unused]] constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    if constexpr (kLevelPairs<TF>)
      X.f[q] = KF::dec_f(KF::load(static_cast<const TF*>(D.fA) +
                                  ((uint32_t)q * D.qs + lvl_nbr<TF>(k, m, nf, cz, (uint32_t)(cx + cy * (int)px), ps))),
                         R(w19(q)));
    else
      X.f[q] = KF::dec_f(KF::load(static_cast<const TF*>(D.src_f[q]) + n), R(w19(q)));
  });
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    [[maybe_unused]] constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    if constexpr (kLevelPairs<TG>)
      X.g[q] = KG::dec_g(KG::load(static_cast<const TG*>(D.gA) +
                                  ((uint32_t)q * D.qs + lvl_nbr<TG>(k, m, ng, cz, (uint32_t)(cx + cy * (int)px), ps))));
    else
      X.g[q] = KG::dec_g(KG::load(static_cast<const TG*>(D.src_g[q]) + n));
  });
}

template <class R>
struct Macro {
  R rho, jx, jy, jz, th;
  R Fx, Fy, Fz, sg, ux, uy, uz;
};

// secMoments (first moments only) + secForces (kernel.js:264-306)
template <class R>
__device__ __forceinline__ void moments_forces(const ParamsHead& P, const Column<R>& C, int k, int nz,
                                               const Cell<R>& X, Macro<R>& M) {
  R rho = X.f[0];
#pragma unroll
  for (int q = 1; q < 19; ++q) rho = rho + X.f[q];
  auto fq = [&](int q) { return X.f[q]; };
  const R jx = moment1<R, 0>(fq), jy = moment1<R, 1>(fq), jz = moment1<R, 2>(fq);
  R th = X.g[0];
#pragma unroll
  for (int q = 1; q < 7; ++q) th = th + X.g[q];
  R Fx = R(0), Fy = R(0);
  R Fz = rho * R(P.gbeta) * th;
  if (k == C.kg && C.kg == C.ktc) {
    // log-law drag in the first fluid cell of building-free columns, limited so it never reverses the flow
    const R cd = R(C.cd);
    const R ux0 = jx / rho, uy0 = jy / rho;
    const R sp = sqrt(ux0 * ux0 + uy0 * uy0);
    Fx = -rho * cd * sp * ux0;
    Fy = -rho * cd * sp * uy0;
    const R lim = R(0.5) * rho;
    if (cd * sp > R(0.5)) {
      Fx = -lim * ux0;
      Fy = -lim * uy0;
    }
  }
  R sg = R(0);
  if (k >= nz - P.nsp) {
    // top sponge: relax u toward the inflow profile, damp uz
    const R aa = (R(k - (nz - P.nsp)) + R(1.0)) / R(P.nsp);
    sg = R(P.sigmax) * aa * aa;
    Fx += rho * sg * (X.uI - jx / rho);
    Fy += rho * sg * (X.vI - jy / rho);
    Fz += -rho * sg * (jz / rho);
  }
  M.rho = rho;
  M.jx = jx;
  M.jy = jy;
  M.jz = jz;
  M.th = th;
  M.Fx = Fx;
  M.Fy = Fy;
  M.Fz = Fz;
  M.sg = sg;
  M.ux = (jx + R(0.5) * Fx) / rho;
  M.uy = (jy + R(0.5) * Fy) / rho;
  M.uz = (jz + R(0.5) * Fz) / rho;
}

// secRelax + secCollision + secScalarCollision (kernel.js:308-386); writes the next state of cell n
template <class S>
__device__ __forceinline__ void collide_store(const DomainView& D, const ParamsHead& P,
                                              const Column<RealOf<S>>& C, int k, uint32_t nf, uint32_t ng,
                                              const Cell<RealOf<S>>& X,
                                              const Macro<RealOf<S>>& M, uint32_t rs) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  StoreF<S>* fB = static_cast<StoreF<S>*>(D.fB);
  StoreG<S>* gB = static_cast<StoreG<S>*>(D.gB);
  const R rho = M.rho, ux = M.ux, uy = M.uy, uz = M.uz, Fx = M.Fx, Fy = M.Fy, Fz = M.Fz;
  const R* f = X.f;
  const R Pxx = moment2<R, 0, 0>(f), Pyy = moment2<R, 1, 1>(f), Pzz = moment2<R, 2, 2>(f);
  const R Pxy = moment2<R, 0, 1>(f), Pxz = moment2<R, 0, 2>(f), Pyz = moment2<R, 1, 2>(f);
  const R usq = ux * ux + uy * uy + uz * uz;
  const R r3 = rho * R(1.0 / 3.0);
  const R Nxx = Pxx - r3 - rho * ux * ux;
  const R Nyy = Pyy - r3 - rho * uy * uy;
  const R Nzz = Pzz - r3 - rho * uz * uz;
  const R Nxy = Pxy - rho * ux * uy;
  const R Nxz = Pxz - rho * ux * uz;
  const R Nyz = Pyz - rho * uy * uz;
  const R Pn = sqrt(Nxx * Nxx + Nyy * Nyy + Nzz * Nzz + R(2.0) * (Nxy * Nxy + Nxz * Nxz + Nyz * Nyz));
  const R kb = X.kb;
  R tb = R(P.tau0) + R(3.0) * R(P.momfac) * kb;
  if (C.spon) tb += C.spg;
  const R tau = R(0.5) * (tb + sqrt(tb * tb + R(P.cs2smag) * Pn / rho));
  const R nusgs = (tau - tb) * R(1.0 / 3.0);
  const R kap = nusgs / R(P.prt) + kb + R(P.kfloor);
  const R taug = R(0.5) + R(4.0) * kap;
  const R om = R(1.0) - R(1.0) / tau;
  const R fpre = R(1.0) - R(0.5) / tau;
  const R trN = (Nxx + Nyy + Nzz) * R(1.0 / 3.0);
  const R uF = ux * Fx + uy * Fy + uz * Fz;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    const R w = R(w19(q));
    const R w45 = R(4.5 * w19(q));
    const R cu = cdot<R, cx, cy, cz>(ux, uy, uz);
    const R feq = w * rho * (R(1.0) + R(3.0) * cu + R(4.5) * cu * cu - R(1.5) * usq);
    R qn = R(0);
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
    KF::store(fB + (nf + D.plane[q]), enc_f_d<KF, q>(feq + om * fr + Fq, w, rs));
  });
  R Ssrc = R(0);
  if (k == C.kg) Ssrc = R(C.qsrc) * R(P.srcscale);
  const R omg = R(1.0) / taug;
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    const R w = R(w7(q));
    const R geq = w * M.th * (R(1.0) + R(4.0) * cdot<R, cx, cy, cz>(ux, uy, uz));
    KG::store(gB + (ng + D.plane[q]), enc_g_d<KG, q>((X.g[q] + omg * (geq - X.g[q]) + w * Ssrc) * (R(1.0) - M.sg), rs));
  });
}

// Top-sponge strength at level k (secForces, kernel.js:296-304): sigmax a^2 with a = (k - (nz - nsp) + 1) / nsp in
// the top nsp levels, else 0. One definition for the single-cell and the paired FMA paths.
__device__ __forceinline__ float sponge_sg(const ParamsHead& P, int nz, int k) {
  if (k < nz - P.nsp) return 0.0f;
  const float aa = __fdividef(__fadd_rn((float)(k - (nz - P.nsp)), 1.0f), (float)P.nsp);
  return __fmul_rn(__fmul_rn(P.sigmax, aa), aa);
}
__device__ __forceinline__ double sponge_sg_d(const ParamsHead& P, int nz, int k) {
  if (k < nz - P.nsp) return 0.0;
  const double aa = ((double)(k - (nz - P.nsp)) + 1.0) / (double)P.nsp;
  return (double)P.sigmax * aa * aa;
}

// The relaxation of the FMA build (lanes.cuh) for one cell: each population q is paired with its opposite, the even
// and odd parts of the equilibrium, the regularised non-equilibrium term and the Guo forcing are formed once per
// pair, and 1/rho, 1/tau are taken once. Mathematically identical to moments_forces + collide_store; rounding
// differs (held to the single-step theta rel-L2 <= 1e-5 bar).
template <class S>
__device__ __forceinline__ void fast_update(const DomainView& D, const ParamsHead& P, const RelaxConst& RK,
                                            const Column<RealOf<S>>& C, int k, uint32_t nf, uint32_t ng,
                                            const Cell<RealOf<S>>& X,
                                            Macro<RealOf<S>>& M, uint32_t rs) {
  using R = RealOf<S>;
  using KF = CodecF<S>;
  using KG = CodecG<S>;
  StoreF<S>* fB = static_cast<StoreF<S>*>(D.fB);
  StoreG<S>* gB = static_cast<StoreG<S>*>(D.gB);
  Moments<R> m;
  lane_moments<R>(X.f, X.g, m);
  R Fx0 = R(0), Fy0 = R(0);
  if (k == C.kg && C.kg == C.ktc) {
    // implicit-limited log-law drag on the first fluid cell of a building-free column
    const R ux0 = vmul(m.jx, m.irho), uy0 = vmul(m.jy, m.irho);
    const R csp = vmul(R(C.cd), vsqrt(vfma(uy0, uy0, vmul(ux0, ux0))));
    const R a = csp > R(0.5) ? vmul(R(-0.5), m.rho) : vsub(R(0), vmul(m.rho, csp));
    Fx0 = vmul(a, ux0);
    Fy0 = vmul(a, uy0);
  }
  R sg;
  if constexpr (sizeof(R) == 8) sg = sponge_sg_d(P, D.nz, k);
  else sg = sponge_sg(P, D.nz, k);
  const R Ssrc = (k == C.kg) ? vmul(R(C.qsrc), R(P.srcscale)) : R(0);
  const R tb_add = C.spon ? R(C.spg) : R(0);
  Relaxed<R> o;
  lane_relax<R>(
      P, RK, m, X.g, X.uI, X.vI, X.kb, sg, Fx0, Fy0, Ssrc, tb_add, o,
      [&](auto Q, R x) {
        constexpr int q = Q;
        KF::store(static_cast<StoreF<S>*>(D.dst_f[q]) + nf, enc_f_x<KF, q>(x, R(w19(q)), rs));
      },
      [&](auto Q, R v) {
        constexpr int q = Q;
        KG::store(static_cast<StoreG<S>*>(D.dst_g[q]) + ng, enc_g_d<KG, q>(v, rs));
      });
  M.rho = m.rho;
  M.jx = m.jx;
  M.jy = m.jy;
  M.jz = m.jz;
  M.th = m.th;
  M.Fx = o.Fx;
  M.Fy = o.Fy;
  M.Fz = o.Fz;
  M.sg = sg;
  M.ux = o.ux;
  M.uy = o.uy;
  M.uz = o.uz;
}

// paired load / store of one population of cells n and n + ps, decoded / encoded exactly as the single-cell codec
template <class T>
__device__ __forceinline__ float2 pair_load_f(const T* p, uint32_t ps, float w) {
  using K = Codec<T>;
  if constexpr (K::kBytes == 2)
    return vfma(make_float2(K::raw(K::load(p)), K::raw(K::load(p + ps))), vc<float2>(1.0 / K::kF), vc<float2>(w));
  else
    return make_float2(K::load(p), K::load(p + ps));
}
template <class T>
__device__ __forceinline__ float2 pair_load_g(const T* p, uint32_t ps) {
  using K = Codec<T>;
  if constexpr (K::kBytes == 2)
    return vmul(make_float2(K::raw(K::load(p)), K::raw(K::load(p + ps))), vc<float2>(1.0 / K::kG));
  else
    return make_float2(K::load(p), K::load(p + ps));
}
// population P of cells n and n + ps, given as x = f / w (flow) or g (temperature), encoded exactly as the
// single-cell codec would encode each (enc_f_x / enc_g_d)
template <int P, class T>
__device__ __forceinline__ void pair_store_f(T* p, uint32_t ps, float2 x, float w, uint32_t h0, uint32_t h1) {
  using K = Codec<T>;
  if constexpr (K::kBytes == 2) {
    const float sw = K::kF * w;
    const float2 e = vfma(x, make_float2(sw, sw), make_float2(-sw, -sw));
    if constexpr (K::kDither) {
      const uint32_t d = K::cvt_sr2(e.x, e.y, h0 * kDitherMul<P>, h1 * kDitherMul<P>);
      K::store_bits(p, d);
      K::store_bits(p + ps, d >> 16);
    } else {
      K::store(p, K::cvt(e.x));
      K::store(p + ps, K::cvt(e.y));
    }
  } else {
    const float2 v = vmul(x, make_float2(w, w));
    K::store(p, v.x);
    K::store(p + ps, v.y);
  }
}
template <int P, class T>
__device__ __forceinline__ void pair_store_g(T* p, uint32_t ps, float2 v, uint32_t h0, uint32_t h1) {
  using K = Codec<T>;
  if constexpr (K::kDither) {
    const float2 e = vmul(v, vc<float2>(K::kG));
    const uint32_t d = K::cvt_sr2(e.x, e.y, h0 * kDitherMul<19 + P>, h1 * kDitherMul<19 + P>);
    K::store_bits(p, d);
    K::store_bits(p + ps, d >> 16);
  } else if constexpr (K::kBytes == 2) {
    const float2 e = vmul(v, vc<float2>(K::kG));
    K::store(p, K::cvt(e.x));
    K::store(p + ps, K::cvt(e.y));
  } else {
    K::store(p, v.x);
    K::store(p + ps, v.y);
  }
}

// The same for a level-paired 16-bit plane (lvl): the levels (k, k + 1), k even, of one population of a column are
// one 32-bit word. Loads: the word at p holds both sources when the population has no vertical component (TWO =
// false); else the sources are the high half of the word at p and the low half of the word one level pair up (p +
// 2 ps), joined by one byte permutation. Decoded and encoded exactly as the single-cell codec does each half.
template <bool TWO, class T>
__device__ __forceinline__ uint32_t word_pull(const T* p, uint32_t ps) {
  using K = Codec<T>;
  const uint32_t a = K::load_w(p);
  if constexpr (!TWO) return a;
  else return __byte_perm(a, K::load_w(p + 2u * ps), 0x5432);
}
// both halves of a level-pair word decoded (flow: h / s + w; temperature: h / s)
template <class T>
__device__ __forceinline__ float2 word_dec_f(uint32_t wd, float w) {
  using K = Codec<T>;
  return vfma(K::raw2(wd), vc<float2>(1.0 / K::kF), vc<float2>(w));
}
template <class T>
__device__ __forceinline__ float2 word_dec_g(uint32_t wd) {
  using K = Codec<T>;
  return vmul(K::raw2(wd), vc<float2>(1.0 / K::kG));
}
template <bool TWO, class T>
__device__ __forceinline__ float2 word_load_f(const T* p, uint32_t ps, float w) {
  return word_dec_f<T>(word_pull<TWO>(p, ps), w);
}
template <bool TWO, class T>
__device__ __forceinline__ float2 word_load_g(const T* p, uint32_t ps) {
  return word_dec_g<T>(word_pull<TWO>(p, ps));
}
template <int P, class T>
__device__ __forceinline__ void word_store_f(T* p, float2 x, float w, uint32_t h0, uint32_t h1) {
  using K = Codec<T>;
  const float sw = K::kF * w;
  const float2 e = vfma(x, make_float2(sw, sw), make_float2(-sw, -sw));
  if constexpr (K::kDither) K::store_w(p, K::cvt_sr2(e.x, e.y, h0 * kDitherMul<P>, h1 * kDitherMul<P>));
  else K::store_w(p, K::cvt2(e.x, e.y));
}
template <int P, class T>
__device__ __forceinline__ void word_store_g(T* p, float2 v, uint32_t h0, uint32_t h1) {
  using K = Codec<T>;
  const float2 e = vmul(v, vc<float2>(K::kG));
  if constexpr (K::kDither) K::store_w(p, K::cvt_sr2(e.x, e.y, h0 * kDitherMul<19 + P>, h1 * kDitherMul<19 + P>));
  else K::store_w(p, K::cvt2(e.x, e.y));
}

// The relaxation and the stores of an interior cell pair (k, k + 1) of one column (fast_pair below, and the TMA-staged
// paired step), given the decoded pull sources of both cells as the two lanes of each population (nf, ng: the pair's
// own element offsets).
template <class S>
__device__ __forceinline__ void fast_pair_relax(const DomainView& D, const ParamsHead& P, const RelaxConst& RK,
                                                const float4* prof, const Column<float>& C, int k, uint32_t nf,
                                                uint32_t ng, const float2 (&f)[19], const float2 (&g)[7], uint32_t r0,
                                                uint32_t r1) {
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  const uint32_t ps = D.ps;
  const int z0 = min(max(k - C.ktc, 0), D.nz - 1), z1 = min(max(k + 1 - C.ktc, 0), D.nz - 1);
  const float4 p0 = prof[z0], p1 = prof[z1];
  Moments<float2> m;
  lane_moments<float2>(f, g, m);
  const float2 zero = vc<float2>(0.0);
  const float2 tb_add = C.spon ? vc<float2>(C.spg) : zero;
  Relaxed<float2> o;
  lane_relax<float2>(
      P, RK, m, g, make_float2(p0.x, p1.x), make_float2(p0.y, p1.y), make_float2(p0.z, p1.z),
      make_float2(sponge_sg(P, D.nz, k), sponge_sg(P, D.nz, k + 1)), zero, zero, zero, tb_add, o,
      [&](auto Q, float2 v) {
        constexpr int q = Q;
        TF* dst = static_cast<TF*>(D.dst_f[q]) + nf;
        if constexpr (kLevelPairs<TF>) word_store_f<q>(dst, v, (float)w19(q), r0, r1);
        else pair_store_f<q>(dst, ps, v, (float)w19(q), r0, r1);
      },
      [&](auto Q, float2 v) {
        constexpr int q = Q;
        TG* dst = static_cast<TG*>(D.dst_g[q]) + ng;
        if constexpr (kLevelPairs<TG>) word_store_g<q>(dst, v, r0, r1);
        else pair_store_g<q>(dst, ps, v, r0, r1);
      });
}

// The 38 pull-source words of an interior level pair (k, k + 1), k even, of a storage whose f and g planes are both
// level-paired (FP16, BF16, FP16 with stochastic rounding), t = k / 2: for population slot p (f: q, g: 19 + q) slot
// pair_slot(p) holds the first source word (word t of the source column for cz = 0 and cz = -1, word t - 1 for
// cz = +1) and, when the population moves vertically, the next slot its second word (one pair up: word t for cz = +1,
// word t + 1 for cz = -1). The pair may be the lid pair (k + 1 the
// top level, nz even): the cz = -1 sources of the top cell are then, for f, the free-slip mirror, the cz = +1
// partner's population at the same lateral source and level (kernel.js:168-181), i.e. the high half of the partner's
// second word, which the second slot then holds; for g the own value (zero gradient), the high half of the first word,
// which the second slot then repeats. Every load is issued unconditionally, so all 38 are in flight together.
constexpr int kPairSlots = 38;
constexpr int pair_slot(int p) {   // evaluated at compile time (constant expressions only)
  int s = 0;
  for (int a = 0; a < p; ++a) s += 1 + ((a < 19 ? kC19[a][2] : kC7[a - 19][2]) != 0 ? 1 : 0);
  return s;
}
static_assert(pair_slot(26) == kPairSlots, "38 words per level pair");

template <class S>
__device__ __forceinline__ void pair_words_load(const DomainView& D, int k, uint32_t mc, uint32_t (&w)[kPairSlots]) {
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  const uint32_t ps = D.ps;
  const uint32_t nf = lvl<TF>(k, mc, ps), ng = lvl<TG>(k, mc, ps);
  const bool top = k + 1 == D.nz - 1;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cz = kC19[q][2];
    constexpr int sl = pair_slot(q);
    const TF* src = static_cast<const TF*>(D.src_f[q]) + nf;
    w[sl] = CodecF<S>::load_w(src);
    if constexpr (cz == 1) w[sl + 1] = CodecF<S>::load_w(src + 2u * ps);
    if constexpr (cz == -1) {
      // at the lid: the mirror's second word (its pull source has the same lateral shift)
      const TF* base2 = static_cast<const TF*>(top ? D.src_f[mirz19(q)] : D.src_f[q]);
      w[sl + 1] = CodecF<S>::load_w(base2 + nf + 2u * ps);
    }
  });
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cz = kC7[q][2];
    constexpr int sl = pair_slot(19 + q);
    const TG* src = static_cast<const TG*>(D.src_g[q]) + ng;
    w[sl] = CodecG<S>::load_w(src);
    if constexpr (cz == 1) w[sl + 1] = CodecG<S>::load_w(src + 2u * ps);
    if constexpr (cz == -1) w[sl + 1] = CodecG<S>::load_w(src + (top ? 0u : 2u * ps));
  });
}

// relax the pair (k, k + 1) from its 38 words (pair_words_load): both cells' sources joined per population by one byte
// permutation, decoded and relaxed as fast_pair_relax does
template <class S>
__device__ __forceinline__ void pair_words_relax(const DomainView& D, const ParamsHead& P, const RelaxConst& RK,
                                                 const float4* prof, const Column<float>& C, int k, uint32_t mc,
                                                 const uint32_t (&w)[kPairSlots], uint32_t r0, uint32_t r1) {
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  const uint32_t ps = D.ps;
  const uint32_t nf = lvl<TF>(k, mc, ps), ng = lvl<TG>(k, mc, ps);
  const bool top = k + 1 == D.nz - 1;
  // cz = -1: (high of the first word, low of the second), at the lid (high, high of the second); cz = +1 always
  // (high of the first, low of the second)
  const uint32_t sel = top ? 0x7632u : 0x5432u;
  float2 f[19], g[7];
  static_for<26>([&](auto Pi) {
    constexpr int p = Pi;
    constexpr bool isf = p < 19;
    constexpr int q = isf ? p : p - 19;
    constexpr int cz = isf ? kC19[q][2] : kC7[q][2];
    constexpr int sl = pair_slot(p);
    uint32_t x = w[sl];
    if constexpr (cz == 1) x = __byte_perm(w[sl], w[sl + 1], 0x5432);
    if constexpr (cz == -1) x = __byte_perm(w[sl], w[sl + 1], sel);
    if constexpr (isf) f[q] = word_dec_f<TF>(x, (float)w19(q));
    else g[q] = word_dec_g<TG>(x);
  });
  fast_pair_relax<S>(D, P, RK, prof, C, k, nf, ng, f, g, r0, r1);
}

// Two vertically adjacent interior cells (k, k + 1) of one column, streamed and relaxed as the two lanes of packed
// f32x2 arithmetic (mc = j px + i; k even when a population plane is level-paired: then each population of the two
// cells is one word, and with level-paired f and g the pair may be the lid pair, pair_words_load). Interior cells are
// never the first fluid cell (no drag, no source); the result of each lane is bit-identical to stream_interior or
// stream_cell + fast_update on that cell alone.
template <class S>
__device__ __forceinline__ void fast_pair(const DomainView& D, const ParamsHead& P, const RelaxConst& RK,
                                          const float4* prof, const Column<float>& C, int k, uint32_t mc, uint32_t r0,
                                          uint32_t r1) {
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  if constexpr (kLevelPairs<TF> && kLevelPairs<TG>) {
    uint32_t w[kPairSlots];
    pair_words_load<S>(D, k, mc, w);
    pair_words_relax<S>(D, P, RK, prof, C, k, mc, w, r0, r1);
  } else {
    const uint32_t ps = D.ps;
    // own element offsets: the pair's word in a level-paired f plane (lvl of the even level k), else level k's cell
    const uint32_t nf = lvl<TF>(k, mc, ps), ng = lvl<TG>(k, mc, ps);
    float2 f[19], g[7];
    static_for<19>([&](auto Q) {
      constexpr int q = Q;
      const TF* src = static_cast<const TF*>(D.src_f[q]) + nf;
      if constexpr (kLevelPairs<TF>) f[q] = word_load_f<kC19[q][2] != 0>(src, ps, (float)w19(q));
      else f[q] = pair_load_f(src, ps, (float)w19(q));
    });
    static_for<7>([&](auto Q) {
      constexpr int q = Q;
      const TG* src = static_cast<const TG*>(D.src_g[q]) + ng;
      if constexpr (kLevelPairs<TG>) g[q] = word_load_g<kC7[q][2] != 0>(src, ps);
      else g[q] = pair_load_g(src, ps);
    });
    fast_pair_relax<S>(D, P, RK, prof, C, k, nf, ng, f, g, r0, r1);
  }
}

// Population slot p of a cell update: f population p (p < 19) or g population p - 19 (p < 26). Bit p of these masks
// is set where the slot's velocity has that y / z component (+1 or -1).
constexpr uint32_t slot_mask(int comp, int sign) {
  uint32_t m = 0;
  for (int p = 0; p < 26; ++p) {
    const int c = p < 19 ? kC19[p][comp] : kC7[p - 19][comp];
    if (c == sign) m |= 1u << p;
  }
  return m;
}

// L2 prefetch of the interior pull sources of level k for the warp's 32 columns (row base: the first column's cell
// index in its plane): lane p < 26 touches the 128-byte line of slot p's source row, x-aligned to the warp (the one
// element a +-x shift moves across the line edge is left to the load). The offsets are clamped into the population
// buffers, so edge rows and levels never reach outside them. No state is read or written: a hint that puts the
// next level's rows in flight while this one is relaxed.
template <class S>
__device__ __forceinline__ void prefetch_level(const DomainView& D, int k, uint32_t rowbase) {
  const int lane = threadIdx.x & 31;
  if (lane >= 26) return;
  constexpr uint32_t kYp = slot_mask(1, 1), kYn = slot_mask(1, -1), kZp = slot_mask(2, 1), kZn = slot_mask(2, -1);
  const int cy = (int)((kYp >> lane) & 1u) - (int)((kYn >> lane) & 1u);
  const int cz = (int)((kZp >> lane) & 1u) - (int)((kZn >> lane) & 1u);
  const bool isf = lane < 19;
  const int q = isf ? lane : lane - 19;
  const int64_t mrow = (int64_t)rowbase - (int64_t)cy * D.px;
  const bool lp = isf ? kLevelPairs<StoreF<S>> : kLevelPairs<StoreG<S>>;
  const int64_t n = (int64_t)q * D.qs + (lp ? (int64_t)((k - cz) >> 1) * 2 * D.ps + 2 * mrow
                                            : (int64_t)(k - cz) * D.ps + mrow);
  const int64_t lim = (int64_t)(isf ? 19 : 7) * D.qs - 64;
  const int64_t e = n < 0 ? 0 : (n > lim ? lim : n);
  const char* p = isf ? static_cast<const char*>(D.fA) + e * (int64_t)sizeof(StoreF<S>)
                      : static_cast<const char*>(D.gA) + e * (int64_t)sizeof(StoreG<S>);
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Budget accumulators of one thread (summed over its cells, then reduced per block into FP64).
struct BudgetAcc {
  float theta, src, cells;
  float ftu[4], fu[4];
};

constexpr int kBlockX = 32;

// The fused step over one z-slab of the columns of a block. MODE: 0 none, 1 write dbg, 2 accumulate dbg.
template <class S, int MODE, bool BUDGET, bool FAST, bool PAIRS = false>
// stage = false: the block staged this domain's parameters, profile and step key for an earlier tile (batched step)
__device__ __forceinline__ void step_block(const DomainView& D, int bx, int by, int bz, int zslab, bool stage = true) {
  using R = RealOf<S>;
  extern __shared__ float4 smem_prof[];
  __shared__ ParamsHead sP;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  // stochastic rounding: the step counter keys this step's dithers (read before the block reports done, so every
  // block of a step sees the same value)
  __shared__ uint32_t s_tkey;
  if (stage) {
    if (tid < 16) reinterpret_cast<int*>(&sP)[tid] = reinterpret_cast<const int*>(D.params)[tid];
    const float4* gprof = reinterpret_cast<const float4*>(D.params + 64);
    for (int z = tid; z < D.nz; z += nthr) smem_prof[z] = gprof[z];
    if constexpr (kDitherOf<S>)
      if (tid == 0) s_tkey = mix32(__ldcg(D.tick) * 0x9e3779b9u + 0x632be5abu);
  }
  __syncthreads();
  const ParamsHead& P = sP;
  const RelaxConst RK = relax_const(P);

  // role of the block (step_split): the main blocks cover their rows' main columns as warps of 32 consecutive
  // columns; the strip blocks after them give each thread one strip column
  const StepSplit SP = step_split(D.nx, D.jlo, D.jhi, D.jbase, D.jg0, D.nyg, D.strip);
  const bool strip_block = by >= main_blocks_y(D.jhi, D.jbase, (int)blockDim.y);
  int i, j;
  const bool valid = block_column(SP, D.nx, D.jbase, D.jhi, (int)blockDim.y, bx, by, (int)threadIdx.x,
                                  (int)threadIdx.y, i, j);
  const int k0 = bz * zslab;
  const int k1 = min(D.nz, k0 + zslab);
  BudgetAcc B;
  if constexpr (BUDGET) {
    B.theta = B.src = B.cells = 0.f;
#pragma unroll
    for (int a = 0; a < 4; ++a) B.ftu[a] = B.fu[a] = 0.f;
  }
  // A warp is one row of 32 columns. It walks the levels in lockstep from its lowest first fluid level, so the lanes
  // of one load touch one level (coalesced), and it takes the interior fast path only when every active lane is
  // interior (the general path gives identical values for interior cells, so a mixed level runs one path, not two).
  Column<R> C;
  int kstart = k1;
  if (valid) {
    load_column(D, P, i, j, C);
    kstart = max(k0, C.kg);
  }
  const int kw = __reduce_min_sync(0xffffffffu, kstart);
  const uint32_t base = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
  // dither seed of the cell at level k: its index in the whole domain (so y-slabs draw the dithers of the undivided
  // domain) mixed with the step key
  uint32_t gid0 = 0, gstep = 0;
  if constexpr (kDitherOf<S>) {
    gid0 = (uint32_t)(j + D.jg0) * (uint32_t)D.px + (uint32_t)i;
    gstep = (uint32_t)D.nyg * (uint32_t)D.px;
  }
  auto seed = [&](int kk) -> uint32_t {
    if constexpr (kDitherOf<S>) return mix32((gid0 + (uint32_t)kk * gstep) ^ s_tkey);
    else return 0u;
  };
  // PAIRS (FMA build without output modes): two interior levels at a time on the packed f32x2 lanes when every
  // active lane of the warp has both cells interior (bit-identical to the single-level path; more registers)
  constexpr bool kPairs = PAIRS && FAST && MODE == 0 && !BUDGET && std::is_same_v<R, float>;
  // a level-paired plane pairs the levels (2t, 2t + 1) only: an odd first level runs alone
  constexpr bool kEvenPairs = kLevelPairs<StoreF<S>> || kLevelPairs<StoreG<S>>;
  constexpr bool kLidPairs = kLevelPairs<StoreF<S>> && kLevelPairs<StoreG<S>>;
  // FMA build, plain steps, launch option: the next level's (pair's) source rows are prefetched into L2 one level
  // (pair) ahead
  constexpr bool kPrefetch = FAST && MODE == 0 && !BUDGET;   // (main blocks only: strip lanes are not one row)
  const uint32_t rowbase = (uint32_t)j * (uint32_t)D.px + (uint32_t)(SP.we + bx * kBlockX);
#pragma unroll 1
  for (int k = kw; k < k1; ++k) {
    if constexpr (kPrefetch) {
      if (D.pf && !strip_block) {
        if (k + (kPairs ? 2 : 1) < k1) prefetch_level<S>(D, k + (kPairs ? 2 : 1), rowbase);
        if (kPairs && k + 3 < k1) prefetch_level<S>(D, k + 3, rowbase);
      }
    }
    if constexpr (kPairs) {
      if (k + 1 < k1 && (!kEvenPairs || (k & 1) == 0)) {
        // level-paired f and g also pair the lid level with the one below it (fast_pair)
        const bool in2 = valid && k >= C.kg && !C.face && k >= C.kint && k + 1 < D.nz - (kLidPairs ? 0 : 1);
        const unsigned m2 = __ballot_sync(0xffffffffu, valid && k + 1 >= C.kg);
        if (m2 != 0u && __ballot_sync(0xffffffffu, in2) == m2) {
          if (in2) fast_pair<S>(D, P, RK, smem_prof, C, k, base, seed(k), seed(k + 1));
          ++k;
          continue;
        }
      }
    }
    const bool act = valid && k >= C.kg;
    const unsigned m = __ballot_sync(0xffffffffu, act);
    const bool inter = act && !C.face && k >= C.kint && k < D.nz - 1;
    const bool all_inter = __ballot_sync(0xffffffffu, inter) == m;
    if (act) {
      const uint32_t n = (uint32_t)k * D.ps + base;   // the cell in [k][j][px] order (output modes)
      const uint32_t nf = lvl<StoreF<S>>(k, base, D.ps), ng = lvl<StoreG<S>>(k, base, D.ps);
      Cell<R> X;
      // paired kernels of the 16-bit storages: the single-level cells (a small share) read their column record again
      // (cached), so the column data only they use (the 3x3 neighbour heights, the face flags, drag and source) is
      // not held in registers across the level loop: the paired path then fits 80 registers (6 blocks per SM)
      constexpr bool kReload = kPairs && kLidPairs;
      Column<R> Cr;
      if constexpr (kReload) load_column(D, P, i, j, Cr);
      const Column<R>& Cs = kReload ? Cr : C;
      if (all_inter) stream_interior<S>(D, smem_prof, Cs, k, base, X);
      else stream_cell<S>(D, P, smem_prof, Cs, k, base, X);
      Macro<R> M;
      if constexpr (FAST) {
        fast_update<S>(D, P, RK, Cs, k, nf, ng, X, M, seed(k));
      } else {
        moments_forces<R>(P, Cs, k, D.nz, X, M);
        collide_store<S>(D, P, Cs, k, nf, ng, X, M, seed(k));
      }
      if constexpr (MODE == 1) {
        D.dbg[n] = make_float4((float)M.th, (float)M.ux, (float)M.uy, (float)M.uz);
      } else if constexpr (MODE == 2) {
        float4 a = D.dbg[n];
        a.x = a.x + (float)M.th;
        a.y = a.y + (float)M.ux;
        a.z = a.z + (float)M.uy;
        a.w = a.w + (float)M.uz;
        D.dbg[n] = a;
      }
      if constexpr (BUDGET) {
        const float th = (float)M.th, ux = (float)M.ux, uy = (float)M.uy;
        B.theta += th;
        B.cells += 1.f;
        if (k == C.kg) B.src += C.qsrc * P.srcscale;
        if (C.latW) { B.ftu[0] += th * ux; B.fu[0] += ux; }
        if (C.latE) { B.ftu[1] += th * ux; B.fu[1] += ux; }
        if (C.latS) { B.ftu[2] += th * uy; B.fu[2] += uy; }
        if (C.latN) { B.ftu[3] += th * uy; B.fu[3] += uy; }
        // time accumulators: one thread owns each column and each face cell, so plain read-modify-writes suffice
        if (D.sacc != nullptr && k == C.kg) {
          double* a = D.sacc + 3 * ((size_t)j * D.nx + i);
          a[0] += (double)th;
          a[1] += (double)ux;
          a[2] += (double)uy;
        }
        if (D.facc != nullptr && C.face) {
          const size_t fy = (size_t)D.ny * D.nz, fx = (size_t)D.nx * D.nz;
          const size_t cy = (size_t)k * D.ny + j, cx = (size_t)k * D.nx + i;
          if (C.latW) { D.facc[2 * cy] += (double)th; D.facc[2 * cy + 1] += (double)ux; }
          if (C.latE) { D.facc[2 * (fy + cy)] += (double)th; D.facc[2 * (fy + cy) + 1] += (double)ux; }
          if (C.latS) { D.facc[2 * (2 * fy + cx)] += (double)th; D.facc[2 * (2 * fy + cx) + 1] += (double)uy; }
          if (C.latN) { D.facc[2 * (2 * fy + fx + cx)] += (double)th; D.facc[2 * (2 * fy + fx + cx) + 1] += (double)uy; }
        }
      }
    }
  }
  if constexpr (BUDGET) {
    // warp shuffle in FP64, then shared-memory FP64 atomics per block, then one global FP64 atomic per block and
    // quantity into one of kBudgetSlots replicas of the record (the reader sums the replicas)
    __shared__ double sB[11];
    if (tid < 11) sB[tid] = 0.0;
    __syncthreads();
    const float v[11] = {B.theta, B.src, B.ftu[0], B.ftu[1], B.ftu[2], B.ftu[3],
                         B.fu[0], B.fu[1], B.fu[2], B.fu[3], B.cells};
#pragma unroll
    for (int a = 0; a < 11; ++a) {
      double d = (double)v[a];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
      if ((tid & 31) == 0 && d != 0.0) atomicAdd(&sB[a], d);
    }
    __syncthreads();
    if (tid < 11 && sB[tid] != 0.0) {
      const int slot = (bx + 5 * by + 11 * bz) & (kBudgetSlots - 1);
      atomicAdd(D.budget + slot * kBudgetStride + tid, sB[tid]);
    }
  }
}

}  // namespace ahx
