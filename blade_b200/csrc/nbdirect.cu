// Direct-space pair kernel and force finalisation (sm_100a).
//
// Counterpart of getforce_nbdirect_kernel (src/nbdirect/nbdirect.cu:87-490)
// plus recull_blocks (src/domdec/recull.cu:41-122) and unpack_forces
// (src/domdec/assign_blocks.cu:444-468), redesigned for Blackwell SIMT:
//
//  * Work item = one i-block x up to 32 candidate j-tiles (the list rebuild
//    splits each block's candidates into items, work_split.h).  A warp
//    recull-tests its candidates at rCut with the fresh AABBs (one lane per
//    candidate, ballot), then walks the surviving tiles; the persistent warps
//    pull items from a counter, longest first once a launch has measured
//    their cycles (k_order).
//  * Tiles without exclusion mask and MSLD atom are streamed: their j atoms
//    that can reach the i block are queued per warp and evaluated in rounds
//    in which each lane holds two i atoms and one j atom, the pair math of
//    the two pairs in packed FP32x2 instructions, the j atom (coordinates,
//    charge, LJ parameters, force) rotating through a group of lanes with
//    __shfl_sync, so every j force returns to its lane without a butterfly
//    reduction (the reference spends 15 xor-shuffles per j atom).
//  * Masked and MSLD tiles are evaluated per tile: lane l owns i atom l and
//    the compacted j atoms rotate through groups of 32, 16, 8 or 4 lanes.
//  * Accumulation in int64 fixed point (2^-32 units): i forces once per work
//    item, j forces once per queued atom or tile chunk, energy per pair and
//    dU/dlambda per work item.  The FP32 partial sums inside a work item have
//    a fixed order, so results do not depend on which warp, CTA or launch
//    runs which work item, nor on the order in which the items are taken.
//  * Pair math in FP32: rsqrt, erfc as exp(-x^2)*P6(1/(1+p x)) sharing the
//    Gaussian with the force (erfc_fit.h), branch-free force switching.
//  * Launched with programmatic dependent launch (launch_pdl): each kernel
//    waits for its predecessor in pdl_wait() before touching memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "bnb_internal.h"
#include "erfc_fit.h"
#include "nbdirect.h"

namespace bnb {

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ bool aabb_hit(float4 imin, float4 imax, float4 jmin, float4 jmax,
                                         float3 sh, float c2) {
  float g, acc = 0.f, lo, hi;
  lo = __fadd_rn(jmin.x, sh.x); hi = __fadd_rn(jmax.x, sh.x);
  g = fmaxf(fmaxf(__fsub_rn(lo, imax.x), __fsub_rn(imin.x, hi)), 0.f);
  acc = __fmul_rn(g, g);
  lo = __fadd_rn(jmin.y, sh.y); hi = __fadd_rn(jmax.y, sh.y);
  g = fmaxf(fmaxf(__fsub_rn(lo, imax.y), __fsub_rn(imin.y, hi)), 0.f);
  acc = __fadd_rn(acc, __fmul_rn(g, g));
  lo = __fadd_rn(jmin.z, sh.z); hi = __fadd_rn(jmax.z, sh.z);
  g = fmaxf(fmaxf(__fsub_rn(lo, imax.z), __fsub_rn(imin.z, hi)), 0.f);
  acc = __fadd_rn(acc, __fmul_rn(g, g));
  return acc <= c2;
}

// erfc(x) exp(x^2) as P6(t), t = 1/(1+p x): even/odd split halves the
// dependency chain of a plain Horner evaluation.
__device__ __forceinline__ float erfcx_poly(float t) {
  const float t2 = t * t;
  float pe = fmaf(kErfcC6, t2, kErfcC4);
  pe = fmaf(pe, t2, kErfcC2);
  pe = fmaf(pe, t2, kErfcC0);
  float po = fmaf(kErfcC5, t2, kErfcC3);
  po = fmaf(po, t2, kErfcC1);
  return fmaf(po, t, pe);
}

__device__ __forceinline__ long long to_fix(float v) {
  return __float2ll_rn(v * kFixScaleF);
}

__device__ __forceinline__ void red_add(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// ---------------------------------------------------------------------------
// Pair physics at distance r (rinv = 1/r, r2 = r*r): energy E and dE/dr.
// Electrostatics: nbdirect.cu:281-323; van der Waals: nbdirect.cu:326-396.
// ---------------------------------------------------------------------------
template <int ELEC, int VDW, bool NEEDE>
__device__ __forceinline__ void pair_terms(const PairConst &pc, float r, float r2, float rinv,
                                           float qq, float c12, float c6, float &dEdr,
                                           float &E) {
  float fe, ee = 0.f;
  if (ELEC == 1) {  // PME real space
    float t = rcp_approx(fmaf(pc.pBeta, r, 1.0f));
    float p = erfcx_poly(t);
    float g = ex2_approx(pc.mBeta2Log2e * r2);
    float eel = qq * (p * g) * rinv;
    fe = -fmaf(qq * pc.twoBetaSqrtPi, g, eel) * rinv;
    ee = eel;
  } else if (ELEC == 0) {  // FSWITCH
    if (r <= pc.rswitch) {
      fe = -qq * rinv * rinv;
      if (NEEDE) ee = qq * (rinv + pc.fdvc);
    } else {
      // The reference's expanded polynomial (nbdirect.cu:293-299) cancels to
      // ~0 near rCut; in FP32 that costs ~1e-5 relative force error.  The same
      // functions in factored form:
      //   dE/dr = -qq (rc^2-r^2)^2 (rc^2+2r^2-3rs^2) ginv / r^2
      //   E     =  qq (rc-r)^3 P(r) ginv / (5 r),
      //   P(r)  = 2r^3 + 6 rc r^2 + (7rc^2-5rs^2) r + 5rc^3 - 15 rc rs^2.
      float w = pc.roff2 - r2;
      fe = -qq * (w * w * fmaf(2.f, r2, pc.fsC1) * pc.fsG) * (rinv * rinv);
      if (NEEDE) {
        float t = pc.rcut - r;
        float p = fmaf(fmaf(fmaf(2.f, r, pc.fsP1), r, pc.fsP2), r, pc.fsP3);
        ee = qq * (t * t * t) * p * pc.fsG5 * rinv;
      }
    }
  } else {  // FSHIFT
    float ri2 = pc.rcinv * pc.rcinv;
    fe = -qq * (rinv * rinv - ri2);
    if (NEEDE) ee = qq * (rinv - 2.f * pc.rcinv + r * ri2);
  }
  float rinv2 = rinv * rinv;
  float rinv3 = rinv2 * rinv;
  float rinv6 = rinv3 * rinv3;
  float fl, el = 0.f;
  if (VDW == 0) {  // VFSWITCH, branch free
    bool in = r < pc.rswitch;
    float a = in ? rinv3 : pc.k6 * (rinv3 - pc.rci3);
    float b = in ? rinv6 : pc.k12 * (rinv6 - pc.rci6);
    fl = (6.f * c6 * a * rinv3 - 12.f * c12 * b * rinv6) * rinv;
    if (NEEDE) {
      float pe = in ? fmaf(rinv6, rinv6, -pc.dv12) : b * (rinv6 - pc.rci6);
      float qe = in ? rinv6 - pc.dv6 : a * (rinv3 - pc.rci3);
      el = c12 * pe - c6 * qe;
    }
  } else if (VDW == 1) {  // VSWITCH
    if (r < pc.rswitch) {
      fl = (6.f * c6 - 12.f * c12 * rinv6) * rinv6 * rinv;
      if (NEEDE) el = (c12 * rinv6 - c6) * rinv6;
    } else {
      float rijl = pc.ron2 - r2, riju = pc.roff2 - r2;
      float fsw = riju * riju * (riju - 3.f * rijl) * pc.rul3inv;
      float dfsw = rijl * riju * pc.rul12;
      fl = fsw * (6.f * c6 - 12.f * c12 * rinv6) * rinv6 * rinv + dfsw * (c12 * rinv6 - c6) * rinv6;
      if (NEEDE) el = fsw * (c12 * rinv6 - c6) * rinv6;
    }
  } else {  // VSHIFT
    float r5 = r2 * r2 * r, r6 = r2 * r2 * r2;
    float rinv12 = rinv6 * rinv6;
    fl = 6.f * c6 * (rinv6 * rinv - r5 * pc.vshRc12inv) - 12.f * c12 * (rinv12 * rinv + r5 * pc.vshRc18inv);
    if (NEEDE)
      el = c12 * (rinv12 + 2.f * r6 * pc.vshRc18inv - 3.f * pc.vshRc12inv) -
           c6 * (rinv6 + r6 * pc.vshRc12inv - 2.f * pc.vshRc6inv);
  }
  dEdr = fe + fl;
  E = ee + el;
}

// LJ pair coefficients.  Combination mode stores per type (sqrt(12 eps),
// Rmin/2): e6 = 12 sqrt(eps_i eps_j), c6 = 2 eps Rmin^6 = e6 R6/6,
// c12 = eps Rmin^12 = e6 R6^2/12 (potential.cxx:1393-1403).
template <bool COMBINE>
__device__ __forceinline__ void lj_params(const float2 *sLJ, int rowI, int tj, float2 ljI,
                                          float2 ljJ, float &c12, float &c6) {
  if (COMBINE) {
    float e6 = ljI.x * ljJ.x;
    float R = ljI.y + ljJ.y;
    float R2 = R * R;
    float R6 = R2 * R2 * R2;
    c6 = (e6 * (1.f / 6.f)) * R6;
    c12 = (e6 * (1.f / 12.f)) * R6 * R6;
  } else {  // the shared table holds (12 c12, 6 c6)
    float2 v = sLJ[rowI + tj];
    c12 = v.x * (1.f / 12.f);
    c6 = v.y * (1.f / 6.f);
  }
}


struct KArgs {
  Dev d;
  PairConst pc;
  const float *lambda;     // [lamTotal] or null
  int count;               // count in-cutoff pairs (energy variants only)
};

// One non-alchemical pair at r2 < rCut^2: returns (dE/dr)/r and, with
// ENERGY, the pair energy.  PME + VFSWITCH (the production combination) is
// written out with the switching algebra folded:
//   VFSWITCH dE/dr * r = 6 c6 a r^-3 - 12 c12 b r^-6   (nbdirect.cu:336-346)
// with a, b = (r^-3, r^-6) inside rSwitch and (k6 (r^-3 - rc^-3),
// k12 (r^-6 - rc^-6)) outside; in combination mode this is
// e6 w (a - w b) with w = Rmin^6 r^-3.  Other methods use pair_terms.
template <int ELEC, int VDW, bool ENERGY, bool COMBINE>
__device__ __forceinline__ float plain_pair(const PairConst &pc, float r2, float qq, const float2 *sLJ,
                                            int rowI, int tj, float2 ljI, float2 ljJ, float &E) {
  const float rinv = rsqrt_approx(r2);
  const float r = r2 * rinv;
  if (ELEC == 1 && VDW == 0) {
    const float t = rcp_approx(fmaf(pc.pBeta, r, 1.0f));
    const float g = ex2_approx(pc.mBeta2Log2e * r2);
    const float p = erfcx_poly(t);
    const float qg = qq * g;
    const float rinv2 = rinv * rinv;
    const float rinv3 = rinv2 * rinv;
    const float rinv6 = rinv3 * rinv3;
    const bool in = r < pc.rswitch;
    const float a = in ? rinv3 : fmaf(pc.k6, rinv3, -pc.k6rci3);
    const float b = in ? rinv6 : fmaf(pc.k12, rinv6, -pc.k12rci6);
    float flr, c12 = 0.f, c6 = 0.f;
    if (COMBINE) {
      const float e6 = ljI.x * ljJ.x;
      const float R = ljI.y + ljJ.y;
      const float R2 = R * R;
      const float R6 = R2 * R2 * R2;
      const float w = R6 * rinv3;
      flr = e6 * w * fmaf(-w, b, a);
      if (ENERGY) {
        c6 = (e6 * (1.f / 6.f)) * R6;
        c12 = (e6 * (1.f / 12.f)) * R6 * R6;
      }
    } else {  // the shared table holds (12 c12, 6 c6)
      const float2 v = sLJ[rowI + tj];
      flr = fmaf(v.y * a, rinv3, -(v.x * b) * rinv6);
      if (ENERGY) {
        c12 = v.x * (1.f / 12.f);
        c6 = v.y * (1.f / 6.f);
      }
    }
    if (ENERGY) {
      const float pe = in ? fmaf(rinv6, rinv6, -pc.dv12) : b * (rinv6 - pc.rci6);
      const float qe = in ? rinv6 - pc.dv6 : a * (rinv3 - pc.rci3);
      E = qg * p * rinv + (c12 * pe - c6 * qe);
    }
    // Coulomb part of (dE/dr) r: -qq g (p / r + 2 beta / sqrt(pi))
    return (flr - qg * fmaf(p, rinv, pc.twoBetaSqrtPi)) * rinv2;
  } else {
    float c12, c6;
    lj_params<COMBINE>(sLJ, rowI, tj, ljI, ljJ, c12, c6);
    float dEdr;
    pair_terms<ELEC, VDW, ENERGY>(pc, r, r2, rinv, qq, c12, c6, dEdr, E);
    return dEdr * rinv;
  }
}

// ---------------------------------------------------------------------------
// Packed FP32x2 arithmetic (sm_100): one instruction updates the .x and .y
// halves, which the streamed tile path below uses for two independent pairs
// (A in .x, B in .y) of one lane.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sel2(bool x, bool y, float2 a, float2 b) {
  return make_float2(x ? a.x : b.x, y ? a.y : b.y);
}

// Two PME + VFSWITCH pairs at squared distances r2 (.x for pair A, .y for B):
// returns (dE/dr)/r for both; with ENERGY also their energies.  Same
// algebra as plain_pair<PME, VFSWITCH>: erfc(beta r) = exp(-beta^2 r^2) P6(t),
// VFSWITCH folded outside rSwitch.  Table mode takes (12 c12, 6 c6), combine
// mode (e6, R) = (sqrt(12 eps_i) sqrt(12 eps_j), Rmin/2_i + Rmin/2_j).
template <bool ENERGY, bool COMBINE>
__device__ __forceinline__ float2 pme_vfsw_pair2(const PairConst &pc, float2 r2, float2 qq, float2 lj0, float2 lj1,
                                                 float2 &E) {
  const float2 rinv = make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
  const float2 r = mul2(r2, rinv);
  const float2 targ = fma2(f2(pc.pBeta), r, f2(1.0f));
  const float2 t = make_float2(rcp_approx(targ.x), rcp_approx(targ.y));
  const float2 garg = mul2(f2(pc.mBeta2Log2e), r2);
  const float2 g = make_float2(ex2_approx(garg.x), ex2_approx(garg.y));
  const float2 t2 = mul2(t, t);
  float2 pe = fma2(f2(kErfcC6), t2, f2(kErfcC4));
  pe = fma2(pe, t2, f2(kErfcC2));
  pe = fma2(pe, t2, f2(kErfcC0));
  float2 po = fma2(f2(kErfcC5), t2, f2(kErfcC3));
  po = fma2(po, t2, f2(kErfcC1));
  const float2 p = fma2(po, t, pe);
  const float2 qg = mul2(qq, g);
  const float2 rinv2 = mul2(rinv, rinv);
  const float2 rinv3 = mul2(rinv2, rinv);
  const float2 rinv6 = mul2(rinv3, rinv3);
  const bool inA = r.x < pc.rswitch, inB = r.y < pc.rswitch;
  const float2 a = sel2(inA, inB, rinv3, fma2(f2(pc.k6), rinv3, f2(-pc.k6rci3)));
  const float2 b = sel2(inA, inB, rinv6, fma2(f2(pc.k12), rinv6, f2(-pc.k12rci6)));
  float2 flr, c12, c6;
  if (COMBINE) {  // lj0 = e6, lj1 = R
    const float2 R2 = mul2(lj1, lj1);
    const float2 R6 = mul2(mul2(R2, R2), R2);
    const float2 w = mul2(R6, rinv3);
    flr = mul2(mul2(lj0, w), fma2(mul2(w, f2(-1.f)), b, a));
    if (ENERGY) {
      c6 = mul2(mul2(lj0, f2(1.f / 6.f)), R6);
      c12 = mul2(mul2(mul2(lj0, f2(1.f / 12.f)), R6), R6);
    }
  } else {        // lj0 = 12 c12, lj1 = 6 c6
    flr = fma2(mul2(lj1, a), rinv3, mul2(mul2(mul2(lj0, f2(-1.f)), b), rinv6));
    if (ENERGY) {
      c12 = mul2(lj0, f2(1.f / 12.f));
      c6 = mul2(lj1, f2(1.f / 6.f));
    }
  }
  if (ENERGY) {
    const float2 pe_in = fma2(rinv6, rinv6, f2(-pc.dv12));
    const float2 pe_out = mul2(b, add2(rinv6, f2(-pc.rci6)));
    const float2 qe_in = add2(rinv6, f2(-pc.dv6));
    const float2 qe_out = mul2(a, add2(rinv3, f2(-pc.rci3)));
    const float2 pe2 = sel2(inA, inB, pe_in, pe_out);
    const float2 qe2 = sel2(inA, inB, qe_in, qe_out);
    E = fma2(mul2(qg, p), rinv, fma2(c12, pe2, mul2(mul2(c6, qe2), f2(-1.f))));
  }
  // Coulomb part of (dE/dr) r: -qq g (p / r + 2 beta / sqrt(pi))
  return mul2(fma2(mul2(qg, f2(-1.f)), fma2(p, rinv, f2(pc.twoBetaSqrtPi)), flr), rinv2);
}



// Per-lane loads of one candidate tile (its j slot for this lane).
template <int ALCH>
struct TileFetch {
  int jBlock, code, mIdx, atom, siteBlock;
  float4 xj;
  uint32_t row;
  __device__ __forceinline__ void fetch(const Dev &d, int4 cand, int c, int lane) {
    jBlock = __shfl_sync(kFull, cand.x, c);
    code = __shfl_sync(kFull, cand.y, c);
    mIdx = __shfl_sync(kFull, cand.z, c);
    const int jslot = 32 * jBlock + lane;
    xj = d.xyzq[jslot];
    atom = d.slotAtom[jslot];
    siteBlock = ALCH ? d.slotSiteBlock[jslot] : 0;
    row = mIdx >= 0 ? d.masks[32 * (size_t)mIdx + lane] : kFull;
  }
};

// j-side registers that travel with the rotation.
template <bool COMBINE, int ALCH>
struct JRegs {
  float x, y, z, q;
  int meta;                // original j lane << 16 | LJ type (table) ; original lane (combine)
  float ex, er;            // combine mode: sqrt(2 eps), Rmin/2
  int b;                   // MSLD siteBlock
  float l;                 // lambda of b
  float fx, fy, fz, fl;

  // withAlch: also the MSLD fields (tiles without MSLD atoms never read them)
  __device__ __forceinline__ void move(int src, int width, bool withMeta = true, bool withAlch = true) {
    x = __shfl_sync(kFull, x, src, width);
    y = __shfl_sync(kFull, y, src, width);
    z = __shfl_sync(kFull, z, src, width);
    q = __shfl_sync(kFull, q, src, width);
    if (withMeta) meta = __shfl_sync(kFull, meta, src, width);
    if (COMBINE) {
      ex = __shfl_sync(kFull, ex, src, width);
      er = __shfl_sync(kFull, er, src, width);
    }
    if (ALCH && withAlch) {
      b = __shfl_sync(kFull, b, src, width);
      l = __shfl_sync(kFull, l, src, width);
    }
  }
  __device__ __forceinline__ void move_forces(int src, int width, bool alch) {
    fx = __shfl_sync(kFull, fx, src, width);
    fy = __shfl_sync(kFull, fy, src, width);
    fz = __shfl_sync(kFull, fz, src, width);
    if (ALCH && alch) fl = __shfl_sync(kFull, fl, src, width);
  }
};

// gj rotation steps of a tile without MSLD scaling.  MASKED tiles test the
// exclusion/diagonal row bit of the current j (its original lane travels in
// J.meta); the others rely on far-away sentinels for empty slots.
template <int ELEC, int VDW, bool ENERGY, bool COMBINE, bool MASKED, int ALCH>
__device__ __forceinline__ void plain_loop(JRegs<COMBINE, ALCH> &J, const float4 &xi, uint32_t row, int gj,
                                           int rot, const PairConst &pc, const float2 *sLJ, int rowI,
                                           float2 ljI, float &fix, float &fiy, float &fiz, long long &ei,
                                           unsigned long long &pairs, int count) {
#pragma unroll 4
  for (int k = 0; k < gj; k++) {
    const float dx = xi.x - J.x, dy = xi.y - J.y, dz = xi.z - J.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    bool act = r2 < pc.rc2;
    if (MASKED) act = act && ((row >> (COMBINE ? J.meta : (J.meta >> 16))) & 1u);
    if (!ENERGY) {
      // Branch-free: the warp evaluates the pair math whenever any of its
      // lanes is in range, so every lane computes it and lanes out of range
      // (or excluded) select zero -- no divergent branch to enter and leave.
      float E = 0.f;
      float fs = plain_pair<ELEC, VDW, ENERGY, COMBINE>(pc, r2, xi.w * J.q, sLJ, rowI, J.meta & 0xFFFF, ljI,
                                                        make_float2(J.ex, J.er), E);
      fs = act ? fs : 0.f;
      fix = fmaf(fs, dx, fix); fiy = fmaf(fs, dy, fiy); fiz = fmaf(fs, dz, fiz);
      J.fx = fmaf(-fs, dx, J.fx); J.fy = fmaf(-fs, dy, J.fy); J.fz = fmaf(-fs, dz, J.fz);
    } else if (act) {  // energy steps (1 in 10) keep the branch: fewer live registers
      float E = 0.f;
      const float fs = plain_pair<ELEC, VDW, ENERGY, COMBINE>(pc, r2, xi.w * J.q, sLJ, rowI, J.meta & 0xFFFF,
                                                              ljI, make_float2(J.ex, J.er), E);
      fix = fmaf(fs, dx, fix); fiy = fmaf(fs, dy, fiy); fiz = fmaf(fs, dz, fiz);
      J.fx = fmaf(-fs, dx, J.fx); J.fy = fmaf(-fs, dy, J.fy); J.fz = fmaf(-fs, dz, J.fz);
      ei += to_fix(E);  // energies in fixed point per pair: exact sums of the FP32 pair values
      if (count) pairs++;
    }
    J.move(rot, gj, MASKED || !COMBINE, false);
    J.move_forces(rot, gj, false);
  }
}

// ---------------------------------------------------------------------------
// Streamed tiles.  The compacted j atoms of a work item's tiles that need no
// exclusion mask and no MSLD scaling are queued in shared memory as entries
// (j slot | shift code << 27) and evaluated in rounds of up to 32.  For these
// rounds lane l holds two i atoms of the block, A = l mod 16 and B = A + 16,
// so each half of the warp covers the whole i block, and one queued j atom:
// with rounds of width gw (16, 8 or 4) half h takes entries h gw .. h gw +
// gw - 1, one per lane of each of its 16 / gw groups of gw lanes.  The j atom
// meets its lane's two i atoms in packed FP32x2 instructions and rotates
// through the group with its force accumulator, so a rotation step moves one
// j atom for two pairs.  After gw steps the groups of a half are summed by
// xor shuffles and group 0 adds each entry's force to the fixed-point
// accumulators, one addition per queued j atom.  A round costs gw steps for
// up to 2 gw entries, so a tile contributes exactly its compacted j atoms and
// only the last round of a work item is padded.
// ---------------------------------------------------------------------------
template <bool COMBINE>
__device__ __forceinline__ void stream_load(const Dev &d, int e, const float4 *shifts, float &x, float &y,
                                            float &z, float &q, int &t, float &ex, float &er) {
  if (e < 0) {  // padding: far outside rCut of every i atom
    x = 1.0e18f; y = 0.f; z = 0.f; q = 0.f; t = 0; ex = 0.f; er = 0.f;
    return;
  }
  const int js = e & 0x7FFFFFF;
  const float4 sh = shifts[e >> 27];
  const float4 xj = d.xyzq[js];
  x = xj.x + sh.x;
  y = xj.y + sh.y;
  z = xj.z + sh.z;
  q = xj.w;
  t = d.slotType[js];
  if (COMBINE) {
    const float2 lj = d.ljType[t];
    ex = lj.x;
    er = lj.y;
  }
}

// The two i atoms of a lane in the streamed rounds: position and scaled
// charge of A (.x) and B (.y), LJ parameters (combine mode) or table rows.
struct IPair {
  float2 x, y, z, q;
  float2 e6, R;   // combine mode: (sqrt(12 eps), Rmin/2) of A and B
  int rowA, rowB; // table mode: type * nTypes of A and B
};

template <int ELEC, int VDW, bool ENERGY, bool COMBINE>
__device__ __forceinline__ void stream_round(const Dev &d, const PairConst &pc, const float2 *sLJ, const int *sS,
                                             int C, int lane, const IPair &I, const float4 *shifts,
                                             float2 &fix2, float2 &fiy2, float2 &fiz2, long long &ei,
                                             unsigned long long &pairs, int count) {
  const int gw = C > 16 ? 16 : (C > 8 ? 8 : 4);
  const int cl = lane & (gw - 1);
  const int eIdx = (lane >> 4) * gw + cl;
  const int e = eIdx < C ? sS[eIdx] : -1;
  float jx, jy, jz, jq, jex = 0.f, jer = 0.f;
  int tj;
  stream_load<COMBINE>(d, e, shifts, jx, jy, jz, jq, tj, jex, jer);
  float jfx = 0.f, jfy = 0.f, jfz = 0.f;
#pragma unroll 2
  for (int k = 0; k < gw; k++) {
    // packed operations with the j value replicated into both halves
    const float2 dx = fma2(f2(jx), f2(-1.f), I.x);
    const float2 dy = fma2(f2(jy), f2(-1.f), I.y);
    const float2 dz = fma2(f2(jz), f2(-1.f), I.z);
    const float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
    const bool actA = r2.x < pc.rc2, actB = r2.y < pc.rc2;
    const float2 qq = mul2(I.q, f2(jq));
    float2 fs, E = f2(0.f);
    if (ELEC == 1 && VDW == 0) {
      float2 lj0, lj1;
      if (COMBINE) {
        lj0 = mul2(I.e6, f2(jex));
        lj1 = add2(I.R, f2(jer));
      } else {
        const float2 vA = sLJ[I.rowA + tj], vB = sLJ[I.rowB + tj];
        lj0 = make_float2(vA.x, vB.x);
        lj1 = make_float2(vA.y, vB.y);
      }
      fs = pme_vfsw_pair2<ENERGY, COMBINE>(pc, r2, qq, lj0, lj1, E);
    } else {
      fs.x = plain_pair<ELEC, VDW, ENERGY, COMBINE>(pc, r2.x, qq.x, sLJ, I.rowA, tj,
                                                    make_float2(I.e6.x, I.R.x), make_float2(jex, jer), E.x);
      fs.y = plain_pair<ELEC, VDW, ENERGY, COMBINE>(pc, r2.y, qq.y, sLJ, I.rowB, tj,
                                                    make_float2(I.e6.y, I.R.y), make_float2(jex, jer), E.y);
    }
    fs = sel2(actA, actB, fs, f2(0.f));
    fix2 = fma2(fs, dx, fix2);
    fiy2 = fma2(fs, dy, fiy2);
    fiz2 = fma2(fs, dz, fiz2);
    // the j atom's force with the sign of the i side, negated below
    jfx = fmaf(fs.x, dx.x, fmaf(fs.y, dx.y, jfx));
    jfy = fmaf(fs.x, dy.x, fmaf(fs.y, dy.y, jfy));
    jfz = fmaf(fs.x, dz.x, fmaf(fs.y, dz.y, jfz));
    if (ENERGY) {
      if (actA) ei += to_fix(E.x);
      if (actB) ei += to_fix(E.y);
      if (count) pairs += (unsigned long long)actA + (unsigned long long)actB;
    }
    jx = __shfl_sync(kFull, jx, lane + 1, gw);
    jy = __shfl_sync(kFull, jy, lane + 1, gw);
    jz = __shfl_sync(kFull, jz, lane + 1, gw);
    jq = __shfl_sync(kFull, jq, lane + 1, gw);
    if (COMBINE) {
      jex = __shfl_sync(kFull, jex, lane + 1, gw);
      jer = __shfl_sync(kFull, jer, lane + 1, gw);
    } else {
      tj = __shfl_sync(kFull, tj, lane + 1, gw);
    }
    jfx = __shfl_sync(kFull, jfx, lane + 1, gw);
    jfy = __shfl_sync(kFull, jfy, lane + 1, gw);
    jfz = __shfl_sync(kFull, jfz, lane + 1, gw);
  }
  // the groups of a half hold the same entries: sum them (not across halves)
  for (int o = 8; o >= gw; o >>= 1) {
    jfx += __shfl_xor_sync(kFull, jfx, o);
    jfy += __shfl_xor_sync(kFull, jfy, o);
    jfz += __shfl_xor_sync(kFull, jfz, o);
  }
  if ((lane & 15) < gw && e >= 0 && (jfx != 0.f || jfy != 0.f || jfz != 0.f)) {
    const int S = 32 * d.maxBlocks;
    const int js = e & 0x7FFFFFF;
    red_add(&d.accF[js], to_fix(-jfx));
    red_add(&d.accF[S + js], to_fix(-jfy));
    red_add(&d.accF[2 * S + js], to_fix(-jfz));
    if (!(isfinite(jfx) && isfinite(jfy) && isfinite(jfz))) atomicOr(&d.ctr->status, kStatusNonFinite);
  }
}

// ---------------------------------------------------------------------------
// The pair kernel.
// ALCH: 0 none, 1 MSLD scaling, 2 MSLD scaling + soft core.
//
// Tile processing with j compaction: the nj j atoms of a tile that lie within
// rCut of the i block's AABB are taken in chunks of gj = 32, 16, 8 or 4
// (every chunk but the last full), each replicated in groups of gj lanes.
// Every lane keeps its own i atom and rotates through the gj j atoms of its
// group, so a tile costs nj rounded up to a multiple of 4 steps instead of
// 32; the group partial j forces are summed with xor shuffles and returned to
// the owner lanes, one chunk per j atom.
// ---------------------------------------------------------------------------
template <int ELEC, int VDW, int ALCH, bool ENERGY, bool COMBINE>
__global__ void __launch_bounds__(256, 2) k_pair(KArgs A) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int sIdx[8][32];
  __shared__ int sStream[8][128];  // queued entries of streamed tiles, per warp
  const Dev &d = A.d;
  const PairConst &pc = A.pc;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nT = d.nTypes;
  float2 *sLJ = reinterpret_cast<float2 *>(smem);
  size_t off = COMBINE ? 0 : sizeof(float2) * nT * nT;
  off = (off + 15) & ~size_t(15);
  long long *sAccL = reinterpret_cast<long long *>(smem + off);
  float *sLam = reinterpret_cast<float *>(smem + off + (ALCH ? sizeof(long long) * d.lamTotal : 0));

  if (!COMBINE)  // (12 c12, 6 c6): the factors of the force expressions folded in
    for (int i = threadIdx.x; i < nT * nT; i += blockDim.x) {
      const float2 v = d.ljTable[i];
      sLJ[i] = make_float2(12.f * v.x, 6.f * v.y);
    }
  if (ALCH)
    for (int i = threadIdx.x; i < d.lamTotal; i += blockDim.x) {
      sAccL[i] = 0;
      sLam[i] = A.lambda[i];
    }
  __syncthreads();

  const int status = d.ctr->status;
  const int nWork = (status & kStatusListInvalid) ? 0 : d.ctr->workCount;
  const int S = 32 * d.maxBlocks;
  unsigned long long pairs = 0;

  // after the first launch of a list the items are taken longest first, in
  // the order their measured cycles gave (launch_order)
  const bool ordered = d.ctr->orderValid != 0;
  int w = 0;  // position in this launch's sequence of items
  if (lane == 0) w = atomicAdd(&d.ctr->workNext, 1);
  w = __shfl_sync(kFull, w, 0);
  while (w < nWork) {
    const int item = ordered ? d.order[w] : w;
    const long long tItem = clock64();
    const int2 wk = d.work[item];
    const int iBlock = wk.x & 0x3FFFFF;
    const int c0 = wk.y;
    int c1 = d.candStart[iBlock + 1];
    c1 = c1 < c0 + (wk.x >> 22) ? c1 : c0 + (wk.x >> 22);
    const int islot = 32 * iBlock + lane;
    float4 xi = d.xyzq[islot];
    const bool iValid = d.slotAtom[islot] >= 0;
    if (!iValid) xi.x = -1.0e18f;  // empty i slot: never within rCut of any j
    const int ti = d.slotType[islot];
    const int rowI = ti * nT;
    const float2 ljI = COMBINE ? d.ljType[ti] : make_float2(0.f, 0.f);
    const int bi = ALCH ? d.slotSiteBlock[islot] : 0;
    const float li = (ALCH && bi) ? sLam[bi & 0xFFFF] : 1.f;
    const RepInfo &ri = d.rep[d.blockRep[iBlock]];
    const float4 *shifts = ri.shift;  // image shift vectors by shift code
    const float4 imin = d.bmin[iBlock], imax = d.bmax[iBlock];

    // per-step recull of this work item's candidates (recull.cu:41-122)
    int4 cand = make_int4(0, 0, -1, 0);
    bool hit = false;
    if (c0 + lane < c1) {
      cand = d.cand[c0 + lane];
      const float4 sv = shifts[cand.y];
      const float3 sh = make_float3(sv.x, sv.y, sv.z);
      hit = aabb_hit(imin, imax, d.bmin[cand.x], d.bmax[cand.x], sh, pc.rc2);
    }
    unsigned act = __ballot_sync(kFull, hit);

    float fix = 0.f, fiy = 0.f, fiz = 0.f, fli = 0.f;
    // i atoms A = lane mod 16 and B = A + 16 of the streamed rounds, their forces
    IPair ip;
    {
      const int a = lane & 15;
      ip.x = make_float2(__shfl_sync(kFull, xi.x, a), __shfl_sync(kFull, xi.x, a + 16));
      ip.y = make_float2(__shfl_sync(kFull, xi.y, a), __shfl_sync(kFull, xi.y, a + 16));
      ip.z = make_float2(__shfl_sync(kFull, xi.z, a), __shfl_sync(kFull, xi.z, a + 16));
      ip.q = make_float2(__shfl_sync(kFull, xi.w, a), __shfl_sync(kFull, xi.w, a + 16));
      if (COMBINE) {
        ip.e6 = make_float2(__shfl_sync(kFull, ljI.x, a), __shfl_sync(kFull, ljI.x, a + 16));
        ip.R = make_float2(__shfl_sync(kFull, ljI.y, a), __shfl_sync(kFull, ljI.y, a + 16));
        ip.rowA = ip.rowB = 0;
      } else {
        ip.e6 = ip.R = f2(0.f);
        ip.rowA = __shfl_sync(kFull, rowI, a);
        ip.rowB = __shfl_sync(kFull, rowI, a + 16);
      }
    }
    float2 fix2 = f2(0.f), fiy2 = f2(0.f), fiz2 = f2(0.f);
    int nS = 0;        // entries queued in sStream[warp]
    long long ei = 0;  // fixed-point energy of this lane's pairs
    // The loads of each tile are issued one tile ahead, so their latency
    // overlaps the compaction and chunk work of the tile before.
    TileFetch<ALCH> nxt;
    if (act) nxt.fetch(d, cand, __ffs(act) - 1, lane);
    while (act) {
      act &= act - 1;
      const TileFetch<ALCH> cur = nxt;
      if (act) nxt.fetch(d, cand, __ffs(act) - 1, lane);
      const int jBlock = cur.jBlock;
      const int code = cur.code;
      const int mIdx = cur.mIdx;
      const float4 sv = shifts[code];
      const float shx = sv.x, shy = sv.y, shz = sv.z;
      const int jslot = 32 * jBlock + lane;
      const float jx = cur.xj.x + shx, jy = cur.xj.y + shy, jz = cur.xj.z + shz;
      const int bj0 = ALCH ? cur.siteBlock : 0;
      const bool jValid = cur.atom >= 0;
      uint32_t row = cur.row;
      if (jBlock == iBlock && code == 0) row &= (lane == 31) ? 0u : (kFull << (lane + 1));
      if (!iValid) row = 0u;

      // j atoms that can reach the i block (per-atom AABB test, nbdirect.cu:211)
      float g, gap2;
      g = fmaxf(fmaxf(imin.x - jx, jx - imax.x), 0.f);
      gap2 = g * g;
      g = fmaxf(fmaxf(imin.y - jy, jy - imax.y), 0.f);
      gap2 = fmaf(g, g, gap2);
      g = fmaxf(fmaxf(imin.z - jz, jz - imax.z), 0.f);
      gap2 = fmaf(g, g, gap2);
      const bool jin = jValid && gap2 < pc.rc2;
      const unsigned jm = __ballot_sync(kFull, jin);
      const int nj = __popc(jm);
      if (nj == 0) continue;
      const bool alchTile = ALCH ? __any_sync(kFull, (bi | bj0) != 0) : false;
      // Tiles without an exclusion mask and off the diagonal need no per-step
      // mask test: empty j slots and invalid i lanes sit far outside rCut.
      const bool masked = mIdx >= 0 || (jBlock == iBlock && code == 0);

      const int rank = __popc(jm & ((1u << lane) - 1u));
      if (!masked && !alchTile) {  // streamed: queue the compacted j atoms, evaluate full chunks of 64
        if (jin) sStream[warp][nS + rank] = jslot | (code << 27);
        nS += nj;
        __syncwarp();
        if (nS >= 32) {
          stream_round<ELEC, VDW, ENERGY, COMBINE>(d, pc, sLJ, sStream[warp], 32, lane, ip, shifts, fix2, fiy2,
                                                   fiz2, ei, pairs, A.count);
          const int rest = nS - 32;  // < 32
          const int carry = lane < rest ? sStream[warp][32 + lane] : 0;
          __syncwarp();
          if (lane < rest) sStream[warp][lane] = carry;
          __syncwarp();
          nS = rest;
        }
        continue;
      }
      // compaction order: the p-th surviving j atom is lane sIdx[p]
      if (jin) sIdx[warp][rank] = lane;
      __syncwarp();
      // j force of this lane's own j atom, delivered by the chunk that held it
      float ofx = 0.f, ofy = 0.f, ofz = 0.f, ofl = 0.f;
      // The nj surviving j atoms are processed in chunks of 32, 16, 8 or 4
      // (32 only when more than 28 survive; otherwise 16 while more than 12
      // remain, then 8, then 4), each replicated in groups of gj lanes, so a
      // tile costs nj rounded up to a multiple of 4 rotation steps.
      for (int done = 0; done < nj;) {
        const int rem = nj - done;
        const int gj = rem > 28 ? 32 : (rem > 12 ? 16 : (rem > 4 ? 8 : 4));
        const int cnt = rem < gj ? rem : gj;
        const int cl = lane & (gj - 1);
        const int src = cl < cnt ? sIdx[warp][done + cl] : lane;
        JRegs<COMBINE, ALCH> J;
        {
          const int js = 32 * jBlock + src;
          const float4 xj = d.xyzq[js];
          J.x = xj.x + shx;
          J.y = xj.y + shy;
          J.z = xj.z + shz;
          J.q = xj.w;
          const int tj = d.slotType[js];
          J.meta = COMBINE ? src : ((src << 16) | tj);
          if (COMBINE) {
            const float2 lj2 = d.ljType[tj];
            J.ex = lj2.x;
            J.er = lj2.y;
          }
          if (ALCH && alchTile) {
            J.b = d.slotSiteBlock[js];
            J.l = J.b ? sLam[J.b & 0xFFFF] : 1.f;
          }
        }
        if (cl >= cnt) J.x = 1.0e18f;  // empty compacted slot: never within rCut
        J.fx = J.fy = J.fz = J.fl = 0.f;
        const int rot = lane + 1;

        if (!alchTile) {
          if (masked)
            plain_loop<ELEC, VDW, ENERGY, COMBINE, true>(J, xi, row, gj, rot, pc, sLJ, rowI, ljI, fix, fiy, fiz,
                                                         ei, pairs, A.count);
          else
            plain_loop<ELEC, VDW, ENERGY, COMBINE, false>(J, xi, row, gj, rot, pc, sLJ, rowI, ljI, fix, fiy,
                                                          fiz, ei, pairs, A.count);
        } else if (ALCH) {
          for (int k = 0; k < gj; k++) {
            const float dx = xi.x - J.x, dy = xi.y - J.y, dz = xi.z - J.z;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const int jb = COMBINE ? J.meta : (J.meta >> 16);
            if (((row >> jb) & 1u) && r2 < pc.rc2) {
              float c12, c6;
              lj_params<COMBINE>(sLJ, rowI, J.meta & 0xFFFF, ljI, make_float2(J.ex, J.er), c12, c6);
              const float rinv = rsqrt_approx(r2);
              const float r = r2 * rinv;
              const int bj = J.b;
              const float lj = J.l;
              // MSLD scaling, nbdirect.cu:244-254
              const bool sameSite = (bi & 0xFFFF0000) == (bj & 0xFFFF0000);
              const float s = sameSite ? (bi == bj ? li : 0.f) : li * lj;
              const bool pert = (bi | bj) != 0;
              float rEff = r, rinvE = rinv, r2E = r2, dredr = 1.f, dredll = 0.f;
              if (ALCH == 2 && pert) {  // soft core, nbdirect.cu:257-275
                const float rSoft = pc.softR * (1.f - s);
                if (r < rSoft) {
                  const float q = __fdividef(r, rSoft);
                  const float f = fmaf(q * q * q, fmaf(-0.5f, q, 1.f), 0.5f);
                  dredr = (3.f - 2.f * q) * q * q;
                  dredll = -pc.softR * (f - dredr * q);
                  rEff = f * rSoft;
                  rinvE = rcp_approx(rEff);
                  r2E = rEff * rEff;
                }
              }
              float dEdr, E;
              pair_terms<ELEC, VDW, true>(pc, rEff, r2E, rinvE, xi.w * J.q, c12, c6, dEdr, E);
              dEdr *= s;
              if (pert) {  // dU/dlambda routing, nbdirect.cu:400-415
                const float fl = fmaf(dEdr, dredll, E);
                if (sameSite) {
                  if (bi == bj) fli += fl;
                } else {
                  fli = fmaf(lj, fl, fli);
                  J.fl = fmaf(li, fl, J.fl);
                }
              }
              const float fs = dEdr * dredr * rinv;
              fix = fmaf(fs, dx, fix); fiy = fmaf(fs, dy, fiy); fiz = fmaf(fs, dz, fiz);
              J.fx = fmaf(-fs, dx, J.fx); J.fy = fmaf(-fs, dy, J.fy); J.fz = fmaf(-fs, dz, J.fz);
              if (ENERGY) ei += to_fix(s * E);
              if (ENERGY && A.count) pairs++;
            }
            J.move(rot, gj);
            J.move_forces(rot, gj, true);
          }
        }
        // sum the group partials; group 0 lane p now holds compacted j done+p
        float fx = J.fx, fy = J.fy, fz = J.fz, fl = J.fl;
        for (int o = 16; o >= gj; o >>= 1) {
          fx += __shfl_xor_sync(kFull, fx, o);
          fy += __shfl_xor_sync(kFull, fy, o);
          fz += __shfl_xor_sync(kFull, fz, o);
          if (ALCH && alchTile) fl += __shfl_xor_sync(kFull, fl, o);
        }
        // deliver to the owner lane of each j atom of this chunk
        const int from = (rank - done) & 31;
        fx = __shfl_sync(kFull, fx, from);
        fy = __shfl_sync(kFull, fy, from);
        fz = __shfl_sync(kFull, fz, from);
        if (ALCH && alchTile) fl = __shfl_sync(kFull, fl, from);
        if (rank >= done && rank < done + cnt) {
          ofx = fx; ofy = fy; ofz = fz; ofl = fl;
        }
        done += cnt;
      }
      __syncwarp();  // sIdx is rewritten by the next tile
      if (jin && (ofx != 0.f || ofy != 0.f || ofz != 0.f)) {
        red_add(&d.accF[jslot], to_fix(ofx));
        red_add(&d.accF[S + jslot], to_fix(ofy));
        red_add(&d.accF[2 * S + jslot], to_fix(ofz));
        if (!(isfinite(ofx) && isfinite(ofy) && isfinite(ofz))) atomicOr(&d.ctr->status, kStatusNonFinite);
      }
      if (ALCH && alchTile && jin && bj0 && ofl != 0.f)
        atomicAdd(reinterpret_cast<unsigned long long *>(&sAccL[bj0 & 0xFFFF]),
                  static_cast<unsigned long long>(to_fix(ofl)));
    }
    // the rest of the queue (< 32 entries) in rounds of 32, 16 or 8 entries,
    // whichever pads least: e.g. 20 entries as 16 + 8 (12 steps, not 16)
    for (int off = 0; off < nS;) {
      const int rem = nS - off;
      const int cap = rem > 24 ? 32 : (rem > 12 ? 16 : 8);
      const int cnt = rem < cap ? rem : cap;
      stream_round<ELEC, VDW, ENERGY, COMBINE>(d, pc, sLJ, sStream[warp] + off, cnt, lane, ip, shifts, fix2, fiy2,
                                               fiz2, ei, pairs, A.count);
      off += cnt;
    }
    __syncwarp();  // sStream is rewritten by the next work item
    // the two halves hold the same i atoms: after the sum, lane l < 16 has
    // atom l in .x and lane l >= 16 atom l in .y
    fix2.x += __shfl_xor_sync(kFull, fix2.x, 16); fix2.y += __shfl_xor_sync(kFull, fix2.y, 16);
    fiy2.x += __shfl_xor_sync(kFull, fiy2.x, 16); fiy2.y += __shfl_xor_sync(kFull, fiy2.y, 16);
    fiz2.x += __shfl_xor_sync(kFull, fiz2.x, 16); fiz2.y += __shfl_xor_sync(kFull, fiz2.y, 16);
    fix += lane < 16 ? fix2.x : fix2.y;
    fiy += lane < 16 ? fiy2.x : fiy2.y;
    fiz += lane < 16 ? fiz2.x : fiz2.y;
    if (iValid && (fix != 0.f || fiy != 0.f || fiz != 0.f)) {
      red_add(&d.accF[islot], to_fix(fix));
      red_add(&d.accF[S + islot], to_fix(fiy));
      red_add(&d.accF[2 * S + islot], to_fix(fiz));
      if (!(isfinite(fix) && isfinite(fiy) && isfinite(fiz))) atomicOr(&d.ctr->status, kStatusNonFinite);
    }
    if (ALCH && bi && fli != 0.f)
      atomicAdd(reinterpret_cast<unsigned long long *>(&sAccL[bi & 0xFFFF]),
                static_cast<unsigned long long>(to_fix(fli)));
    if (ENERGY) {
      long long e = ei;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(kFull, e, o);
      if (lane == 0 && e != 0) red_add(&d.accE[d.blockRep[iBlock]], e);
    }
    if (lane == 0) {
      const long long dt = clock64() - tItem;
      d.itemCost[item] = dt < 0xFFFFFFFFll ? (unsigned int)dt : 0xFFFFFFFFu;
      w = atomicAdd(&d.ctr->workNext, 1);
    }
    w = __shfl_sync(kFull, w, 0);
  }
  if (A.count) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(kFull, pairs, o);
    if (lane == 0 && pairs) atomicAdd(&d.ctr->pairCount, pairs);
  }
  if (ALCH) {
    __syncthreads();
    for (int i = threadIdx.x; i < d.lamTotal; i += blockDim.x)
      if (sAccL[i]) red_add(&d.accL[i], sAccL[i]);
  }
}

// Log-scale bucket of a cycle count: 8 buckets per octave, 0..255.
__device__ __forceinline__ int cost_bucket(unsigned int c) {
  c = c ? c : 1u;
  const int e = 31 - __clz(c);
  const int m = e >= 3 ? (int)(c >> (e - 3)) & 7 : (int)(c << (3 - e)) & 7;
  return 8 * e + m;
}

// Work items by decreasing measured cost, one CTA: a histogram of the costs
// in log-scale buckets, bucket offsets from the most expensive bucket down
// (a warp scan over 256 buckets), then every item placed in its bucket.
// Inside a bucket the order follows the shared-memory atomics; the results
// of the pair kernel do not depend on the order of its items.
__global__ void __launch_bounds__(1024) k_order(Dev d) {
  pdl_wait();
  __shared__ int hist[256];
  const int n = (d.ctr->status & kStatusListInvalid) ? 0 : d.ctr->workCount;
  for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&hist[cost_bucket(d.itemCost[i])], 1);
  __syncthreads();
  if (threadIdx.x < 32) {  // lane l owns buckets 255 - 8l .. 248 - 8l (descending)
    const int l = threadIdx.x;
    int c[8], sum = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      c[k] = hist[255 - 8 * l - k];
      sum += c[k];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(kFull, incl, o);
      if (l >= o) incl += v;
    }
    int run = incl - sum;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      hist[255 - 8 * l - k] = run;
      run += c[k];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) d.order[atomicAdd(&hist[cost_bucket(d.itemCost[i])], 1)] = i;
  if (threadIdx.x == 0) d.ctr->orderValid = n > 0;
}

// Converts the fixed-point accumulators to the caller's outputs and clears them.
// One thread per atom, in atom order: the outputs (in the caller's atom
// order) are written coalesced, and the per-slot accumulators, still in L2
// from the pair kernel's atomics, are gathered through atomSlot.
__global__ void k_finalize(Dev d, bnb_outputs o, int mode) {
  pdl_wait();
  const int S = 32 * d.maxBlocks;
  const double inv = 1.0 / kFixScale;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < d.N; a += gridDim.x * blockDim.x) {
    const int t = d.atomSlot[a];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const long long v = d.accF[k * S + t];
      if (v) d.accF[k * S + t] = 0;
      const double f = (double)v * inv;
      if (o.force64) out64(&o.force64[3 * a + k], f, mode);
      if (o.force) out32(&o.force[3 * a + k], (float)f, mode);
    }
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) d.ctr->workNext = 0;  // the pair kernel of the next step starts at item 0
    for (int i = threadIdx.x; i < d.lamTotal; i += blockDim.x) {
      long long v = d.accL[i];
      d.accL[i] = 0;
      double f = (double)v * inv;
      if (o.lambdaForce64) out64(&o.lambdaForce64[i], f, mode);
      if (o.lambdaForce) out32(&o.lambdaForce[i], (float)f, mode);
    }
    for (int r = threadIdx.x; r < d.R; r += blockDim.x) {
      long long v = d.accE[r];
      d.accE[r] = 0;
      double e = (double)v * inv;
      if (o.energy64) out64(&o.energy64[r], e, mode);
      if (o.energy) outE(&o.energy[r], e, mode);
    }
  }
}

// Persistent launch: as many CTAs as fit at once; warps pull work items from
// the device counter, so the grid never leaves a partial last wave.
template <int ELEC, int VDW, int ALCH, bool ENERGY, bool COMBINE>
void launch_t(const KArgs &a, int maxGrid, size_t shmem, cudaStream_t s) {
  auto k = k_pair<ELEC, VDW, ALCH, ENERGY, COMBINE>;
  static int perSM = -1, sms = 0;
  static size_t shmemSeen = ~size_t(0);
  if (shmem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
  if (perSM < 0 || shmemSeen != shmem) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, 256, shmem) != cudaSuccess || perSM < 1)
      perSM = 1;
    shmemSeen = shmem;
  }
  int grid = perSM * sms;
  if (grid > maxGrid) grid = maxGrid;
  if (grid < 1) grid = 1;
  launch_pdl(k, grid, 256, shmem, s, a);
}

template <int ELEC, int VDW>
void launch_ev(const KArgs &a, int alch, bool energy, bool combine, int grid, size_t shmem,
               cudaStream_t s) {
#define BNB_L(AL, EN, CO) \
  if (alch == AL && energy == EN && combine == CO) { launch_t<ELEC, VDW, AL, EN, CO>(a, grid, shmem, s); return; }
  BNB_L(0, false, false) BNB_L(0, false, true) BNB_L(0, true, false) BNB_L(0, true, true)
  BNB_L(1, false, false) BNB_L(1, false, true) BNB_L(1, true, false) BNB_L(1, true, true)
  BNB_L(2, false, false) BNB_L(2, false, true) BNB_L(2, true, false) BNB_L(2, true, true)
#undef BNB_L
}

// ---------------------------------------------------------------------------
// All-pairs variant for one small periodic system (bnb_nbdirect_noalloc): no
// block list; every 32x32 tile of atom blocks (J >= I) is visited by one warp
// with minimum-image distances.  Lane l keeps atom 32I+l; the j data and the
// j-force accumulators rotate one lane per step, so after 32 steps every lane
// holds its own j atom again and adds its total once.  The pair physics is
// pair_terms (the general path of the list kernel), with table LJ
// coefficients read from global memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool excluded_sorted(const int *ex, int lo, int hi, int j) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const int v = ex[mid];
    if (v == j) return true;
    if (v < j) lo = mid + 1;
    else hi = mid;
  }
  return false;
}

template <int ELEC, int VDW, bool ENERGY>
__global__ void __launch_bounds__(128) k_allpairs(AllPairsArgs a) {
  const int lane = threadIdx.x & 31;
  const int I = blockIdx.y;
  const int J = blockIdx.x * 4 + (threadIdx.x >> 5);
  const int nb = (a.N + 31) >> 5;
  if (J < I || J >= nb) return;  // uniform per warp
  const PairConst &pc = a.pc;
  const int i = 32 * I + lane;
  const bool iv = i < a.N;
  float xi = 0.f, yi = 0.f, zi = 0.f, qi = 0.f;
  int ti = 0, e0 = 0, e1 = 0;
  if (iv) {
    xi = a.x[3 * i]; yi = a.x[3 * i + 1]; zi = a.x[3 * i + 2];
    const bnb_nbond n = a.nb[i];
    qi = n.q * a.sqrtK;
    ti = n.typeIdx;
    e0 = a.exclStart[i];
    e1 = a.exclStart[i + 1];
  }
  const int j0 = 32 * J + lane;
  float xj = 0.f, yj = 0.f, zj = 0.f, qj = 0.f;
  int tj = 0;
  if (j0 < a.N) {
    xj = a.x[3 * j0]; yj = a.x[3 * j0 + 1]; zj = a.x[3 * j0 + 2];
    const bnb_nbond n = a.nb[j0];
    qj = n.q * a.sqrtK;
    tj = n.typeIdx;
  }
  float fix = 0.f, fiy = 0.f, fiz = 0.f, fjx = 0.f, fjy = 0.f, fjz = 0.f;
  long long ef = 0;  // energy in fixed point per pair
  const int src = (lane + 1) & 31;
  for (int k = 0; k < 32; ++k) {
    const int jl = (lane + k) & 31;
    const int j = 32 * J + jl;
    if (iv && j < a.N && (J != I || jl > lane)) {
      float dx = xi - xj, dy = yi - yj, dz = zi - zj;
      dx -= a.box.x * rintf(dx * a.boxInv.x);
      dy -= a.box.y * rintf(dy * a.boxInv.y);
      dz -= a.box.z * rintf(dz * a.boxInv.z);
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (r2 < pc.rc2 && !excluded_sorted(a.exclAtom, e0, e1, j)) {
        const float rinv = rsqrt_approx(r2);
        const float r = r2 * rinv;
        const bnb_vdw v = a.vdw[ti * a.nTypes + tj];
        float dEdr = 0.f, E = 0.f;
        pair_terms<ELEC, VDW, ENERGY>(pc, r, r2, rinv, qi * qj, v.c12, v.c6, dEdr, E);
        const float sc = dEdr * rinv;
        fix = fmaf(sc, dx, fix); fiy = fmaf(sc, dy, fiy); fiz = fmaf(sc, dz, fiz);
        fjx = fmaf(-sc, dx, fjx); fjy = fmaf(-sc, dy, fjy); fjz = fmaf(-sc, dz, fjz);
        if (ENERGY) ef += to_fix(E);
      }
    }
    xj = __shfl_sync(0xFFFFFFFFu, xj, src);
    yj = __shfl_sync(0xFFFFFFFFu, yj, src);
    zj = __shfl_sync(0xFFFFFFFFu, zj, src);
    qj = __shfl_sync(0xFFFFFFFFu, qj, src);
    tj = __shfl_sync(0xFFFFFFFFu, tj, src);
    fjx = __shfl_sync(0xFFFFFFFFu, fjx, src);
    fjy = __shfl_sync(0xFFFFFFFFu, fjy, src);
    fjz = __shfl_sync(0xFFFFFFFFu, fjz, src);
  }
  const int S = a.stride;
  if (iv) {
    red_add(&a.accF[i], to_fix(fix));
    red_add(&a.accF[S + i], to_fix(fiy));
    red_add(&a.accF[2 * S + i], to_fix(fiz));
  }
  if (j0 < a.N) {
    red_add(&a.accF[j0], to_fix(fjx));
    red_add(&a.accF[S + j0], to_fix(fjy));
    red_add(&a.accF[2 * S + j0], to_fix(fjz));
  }
  if (ENERGY) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ef += __shfl_xor_sync(0xFFFFFFFFu, ef, o);
    if (lane == 0 && ef != 0) red_add(a.accE, ef);
  }
}

// Converts the all-pairs accumulators to the outputs (bnb_compute's output
// semantics) and writes every entry it read back to zero.
__global__ void k_allpairs_finalize(AllPairsArgs a, bnb_outputs o) {
  const double inv = 1.0 / kFixScale;
  const int S = a.stride;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.N; t += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const long long v = a.accF[k * S + t];
      a.accF[k * S + t] = 0;
      const double f = (double)v * inv;
      if (o.force64) o.force64[3 * t + k] = f;
      if (o.force && v) o.force[3 * t + k] += (float)f;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const long long v = *a.accE;
    *a.accE = 0;
    const double en = (double)v * inv;
    if (o.energy64) *o.energy64 = en;
    if (o.energy) *o.energy += en;
  }
}

template <int ELEC, int VDW>
void launch_allpairs_ev(const AllPairsArgs &a, bool energy, dim3 grid, cudaStream_t s) {
  if (energy) k_allpairs<ELEC, VDW, true><<<grid, 128, 0, s>>>(a);
  else k_allpairs<ELEC, VDW, false><<<grid, 128, 0, s>>>(a);
}

}  // namespace

int launch_pair(const Dev &d, const PairConst &pc, const float *lambda, int elec, int vdw,
                int alch, bool energy, bool count, int grid, cudaStream_t s) {
  if (32LL * d.maxBlocks >= (1LL << 27)) return BNB_ERR_TOO_LARGE;  // streamed entries hold the slot in 27 bits
  KArgs a{d, pc, lambda, count ? 1 : 0};
  size_t shmem = d.ljCombine ? 0 : sizeof(float2) * d.nTypes * d.nTypes;
  shmem = (shmem + 15) & ~size_t(15);
  if (alch) shmem += (sizeof(long long) + sizeof(float)) * d.lamTotal;
  bool combine = d.ljCombine != 0;
  switch (elec * 3 + vdw) {
    case 0: launch_ev<0, 0>(a, alch, energy, combine, grid, shmem, s); break;
    case 1: launch_ev<0, 1>(a, alch, energy, combine, grid, shmem, s); break;
    case 2: launch_ev<0, 2>(a, alch, energy, combine, grid, shmem, s); break;
    case 3: launch_ev<1, 0>(a, alch, energy, combine, grid, shmem, s); break;
    case 4: launch_ev<1, 1>(a, alch, energy, combine, grid, shmem, s); break;
    case 5: launch_ev<1, 2>(a, alch, energy, combine, grid, shmem, s); break;
    case 6: launch_ev<2, 0>(a, alch, energy, combine, grid, shmem, s); break;
    case 7: launch_ev<2, 1>(a, alch, energy, combine, grid, shmem, s); break;
    case 8: launch_ev<2, 2>(a, alch, energy, combine, grid, shmem, s); break;
    default: return BNB_ERR_ARG;
  }
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

void launch_finalize(const Dev &d, const bnb_outputs &o, int mode, cudaStream_t s) {
  int n = d.N;
  int grid = (n + 255) / 256;
  if (grid > 148 * 8) grid = 148 * 8;
  if (grid < 1) grid = 1;
  launch_pdl(k_finalize, grid, 256, 0, s, d, o, mode);
}

void launch_order(const Dev &d, cudaStream_t s) { launch_pdl(k_order, 1, 1024, 0, s, d); }

int launch_allpairs(const AllPairsArgs &a, const bnb_outputs &o, int elec, int vdw, bool energy,
                    cudaStream_t s) {
  const int nb = (a.N + 31) / 32;
  const dim3 grid((nb + 3) / 4, nb);
  if (nb > 0) switch (elec * 3 + vdw) {
    case 0: launch_allpairs_ev<0, 0>(a, energy, grid, s); break;
    case 1: launch_allpairs_ev<0, 1>(a, energy, grid, s); break;
    case 2: launch_allpairs_ev<0, 2>(a, energy, grid, s); break;
    case 3: launch_allpairs_ev<1, 0>(a, energy, grid, s); break;
    case 4: launch_allpairs_ev<1, 1>(a, energy, grid, s); break;
    case 5: launch_allpairs_ev<1, 2>(a, energy, grid, s); break;
    case 6: launch_allpairs_ev<2, 0>(a, energy, grid, s); break;
    case 7: launch_allpairs_ev<2, 1>(a, energy, grid, s); break;
    case 8: launch_allpairs_ev<2, 2>(a, energy, grid, s); break;
    default: return BNB_ERR_ARG;
  }
  if (cudaGetLastError() != cudaSuccess) return BNB_ERR_CUDA;
  k_allpairs_finalize<<<a.N > 0 ? (a.N + 255) / 256 : 1, 256, 0, s>>>(a, o);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

}  // namespace bnb
