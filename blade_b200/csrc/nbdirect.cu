// Direct-space pair kernel and force finalisation (sm_100a).
//
// Counterpart of getforce_nbdirect_kernel (src/nbdirect/nbdirect.cu:87-490)
// plus recull_blocks (src/domdec/recull.cu:41-122) and unpack_forces
// (src/domdec/assign_blocks.cu:444-468), redesigned for Blackwell SIMT:
//
//  * Work item = one i-block x up to kTilesPerWork candidate j-tiles.  A warp
//    recull-tests its candidates at rCut with the fresh AABBs (one lane per
//    candidate, ballot), then walks the surviving tiles.
//  * j-tile rotation: lane l owns i-atom l for the whole work item and holds
//    j-atom (l+k)&31 at step k.  After each step the j coordinates, charge,
//    type and the j-force accumulators move one lane down with __shfl_sync, so
//    after 32 steps every j-force is back in its owner lane and no butterfly
//    reduction is needed (the reference spends 15 xor-shuffles per j atom).
//  * Accumulation in int64 fixed point (2^-32 units): i forces once per work
//    item, j forces once per tile, energy and dU/dlambda per work item.  The
//    FP32 partial sums inside a work item have a fixed order, so results do
//    not depend on which warp, CTA or launch runs which work item.
//  * Pair math in FP32: rsqrt, erfc as exp(-x^2)*P8(1/(1+p x)) sharing the
//    Gaussian with the force (erfc_fit.h), branch-free force switching.
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

__device__ __forceinline__ void shift_of(int code, int &sx, int &sy, int &sz) {
  if (code < 2) { sx = code; sy = 0; sz = 0; }
  else if (code < 5) { sx = code - 3; sy = 1; sz = 0; }
  else { int c = code - 5; sx = c % 3 - 1; sy = c / 3 - 1; sz = 1; }
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
    float t = rcp_approx(fmaf(kErfcP, pc.beta * r, 1.0f));
    float p = kErfcC8;
    p = fmaf(p, t, kErfcC7);
    p = fmaf(p, t, kErfcC6);
    p = fmaf(p, t, kErfcC5);
    p = fmaf(p, t, kErfcC4);
    p = fmaf(p, t, kErfcC3);
    p = fmaf(p, t, kErfcC2);
    p = fmaf(p, t, kErfcC1);
    p = fmaf(p, t, kErfcC0);
    float g = ex2_approx(pc.mBeta2Log2e * r2);
    float eel = qq * (p * g) * rinv;
    fe = -fmaf(qq * pc.twoBetaSqrtPi, g, eel) * rinv;
    ee = eel;
  } else if (ELEC == 0) {  // FSWITCH
    if (r <= pc.rswitch) {
      fe = -qq * rinv * rinv;
      if (NEEDE) ee = qq * (rinv + pc.fdvc);
    } else {
      float r3 = r2 * r, r5 = r3 * r2;
      fe = -qq * rinv * (pc.fA * rinv + pc.fB * r + 3.f * pc.fC * r3 + 5.f * pc.fD * r5);
      if (NEEDE)
        ee = qq * (pc.fA * (rinv - pc.rcinv) + pc.fB * (pc.rcut - r) +
                   pc.fC * (pc.roff2 * pc.rcut - r3) + pc.fD * (pc.roff2 * pc.roff2 * pc.rcut - r5));
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

template <bool COMBINE>
__device__ __forceinline__ void lj_params(const float2 *sLJ, int rowI, int tj, float2 ljI,
                                          float2 ljJ, float &c12, float &c6) {
  if (COMBINE) {
    float e = ljI.x * ljJ.x;
    float R = ljI.y + ljJ.y;
    float R2 = R * R;
    float R6 = R2 * R2 * R2;
    c6 = e * R6;
    c12 = 0.5f * e * R6 * R6;
  } else {
    float2 v = sLJ[rowI + tj];
    c12 = v.x;
    c6 = v.y;
  }
}

struct KArgs {
  Dev d;
  PairConst pc;
  const float *lambda;     // [lamTotal] or null
  int count;               // count in-cutoff pairs
};

// ---------------------------------------------------------------------------
// The pair kernel.
// ALCH: 0 none, 1 MSLD scaling, 2 MSLD scaling + soft core.
// ---------------------------------------------------------------------------
template <int ELEC, int VDW, int ALCH, bool ENERGY, bool COMBINE>
__global__ void __launch_bounds__(256, 2) k_pair(KArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Dev &d = A.d;
  const PairConst &pc = A.pc;
  const int lane = threadIdx.x & 31;
  const int nT = d.nTypes;
  float2 *sLJ = reinterpret_cast<float2 *>(smem);
  size_t off = COMBINE ? 0 : sizeof(float2) * nT * nT;
  off = (off + 15) & ~size_t(15);
  long long *sAccL = reinterpret_cast<long long *>(smem + off);
  float *sLam = reinterpret_cast<float *>(smem + off + (ALCH ? sizeof(long long) * d.lamTotal : 0));

  if (!COMBINE)
    for (int i = threadIdx.x; i < nT * nT; i += blockDim.x) sLJ[i] = d.ljTable[i];
  if (ALCH)
    for (int i = threadIdx.x; i < d.lamTotal; i += blockDim.x) {
      sAccL[i] = 0;
      sLam[i] = A.lambda[i];
    }
  __syncthreads();

  const int status = d.ctr->status;
  const int nWork = (status & kStatusListInvalid) ? 0 : d.ctr->workCount;
  const int S = 32 * d.maxBlocks;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int srcLane = (lane + 1) & 31;
  unsigned long long pairs = 0;

  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nWork; w += nWarps) {
    const int2 wk = d.work[w];
    const int iBlock = wk.x;
    const int c0 = wk.y;
    int c1 = d.candStart[iBlock + 1];
    c1 = c1 < c0 + kTilesPerWork ? c1 : c0 + kTilesPerWork;
    const int islot = 32 * iBlock + lane;
    const float4 xi = d.xyzq[islot];
    const bool iValid = d.slotAtom[islot] >= 0;
    const int ti = d.slotType[islot];
    const int rowI = ti * nT;
    const float2 ljI = COMBINE ? d.ljType[ti] : make_float2(0.f, 0.f);
    const int bi = ALCH ? d.slotSiteBlock[islot] : 0;
    const float li = (ALCH && bi) ? sLam[bi & 0xFFFF] : 1.f;
    const RepInfo &ri = d.rep[d.blockRep[iBlock]];
    const float bx = ri.box[0], by = ri.box[1], bz = ri.box[2];

    // per-step recull of this work item's candidates (recull.cu:41-122)
    int4 cand = make_int4(0, 0, -1, 0);
    bool hit = false;
    if (c0 + lane < c1) {
      cand = d.cand[c0 + lane];
      int sx, sy, sz;
      shift_of(cand.y, sx, sy, sz);
      float3 sh = make_float3(__fmul_rn((float)sx, bx), __fmul_rn((float)sy, by),
                              __fmul_rn((float)sz, bz));
      hit = aabb_hit(d.bmin[iBlock], d.bmax[iBlock], d.bmin[cand.x], d.bmax[cand.x], sh, pc.rc2);
    }
    unsigned act = __ballot_sync(kFull, hit);

    float fix = 0.f, fiy = 0.f, fiz = 0.f, ei = 0.f, fli = 0.f;
    while (act) {
      const int c = __ffs(act) - 1;
      act &= act - 1;
      const int jBlock = __shfl_sync(kFull, cand.x, c);
      const int code = __shfl_sync(kFull, cand.y, c);
      const int mIdx = __shfl_sync(kFull, cand.z, c);
      int sx, sy, sz;
      shift_of(code, sx, sy, sz);
      const int jslot = 32 * jBlock + lane;
      float4 xj = d.xyzq[jslot];
      xj.x += (float)sx * bx;
      xj.y += (float)sy * by;
      xj.z += (float)sz * bz;
      int tj = d.slotType[jslot];
      float2 ljJ = COMBINE ? d.ljType[tj] : make_float2(0.f, 0.f);
      int bj = ALCH ? d.slotSiteBlock[jslot] : 0;
      float lj = (ALCH && bj) ? sLam[bj & 0xFFFF] : 1.f;
      const bool jValid = d.slotAtom[jslot] >= 0;
      uint32_t row = mIdx >= 0 ? d.masks[32 * (size_t)mIdx + lane] : kFull;
      if (jBlock == iBlock && code == 0) row &= (lane == 31) ? 0u : (kFull << (lane + 1));
      row &= __ballot_sync(kFull, jValid);
      if (!iValid) row = 0u;
      uint32_t mr = __funnelshift_r(row, row, lane);  // bit k <-> j = (lane+k)&31

      float fjx = 0.f, fjy = 0.f, fjz = 0.f, flj = 0.f;
      const bool alchTile = ALCH ? __any_sync(kFull, (bi | bj) != 0) : false;

      if (!alchTile) {
#pragma unroll 8
        for (int k = 0; k < 32; k++) {
          const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          if ((mr & 1u) && r2 < pc.rc2) {
            float c12, c6;
            lj_params<COMBINE>(sLJ, rowI, tj, ljI, ljJ, c12, c6);
            const float rinv = rsqrt_approx(r2);
            const float r = r2 * rinv;
            float dEdr, E;
            pair_terms<ELEC, VDW, ENERGY>(pc, r, r2, rinv, xi.w * xj.w, c12, c6, dEdr, E);
            const float fs = dEdr * rinv;
            fix = fmaf(fs, dx, fix); fiy = fmaf(fs, dy, fiy); fiz = fmaf(fs, dz, fiz);
            fjx = fmaf(-fs, dx, fjx); fjy = fmaf(-fs, dy, fjy); fjz = fmaf(-fs, dz, fjz);
            if (ENERGY) ei += E;
            if (A.count) pairs++;
          }
          mr >>= 1;
          xj.x = __shfl_sync(kFull, xj.x, srcLane);
          xj.y = __shfl_sync(kFull, xj.y, srcLane);
          xj.z = __shfl_sync(kFull, xj.z, srcLane);
          xj.w = __shfl_sync(kFull, xj.w, srcLane);
          if (COMBINE) {
            ljJ.x = __shfl_sync(kFull, ljJ.x, srcLane);
            ljJ.y = __shfl_sync(kFull, ljJ.y, srcLane);
          } else {
            tj = __shfl_sync(kFull, tj, srcLane);
          }
          fjx = __shfl_sync(kFull, fjx, srcLane);
          fjy = __shfl_sync(kFull, fjy, srcLane);
          fjz = __shfl_sync(kFull, fjz, srcLane);
        }
      } else if (ALCH) {
#pragma unroll 4
        for (int k = 0; k < 32; k++) {
          const float dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          if ((mr & 1u) && r2 < pc.rc2) {
            float c12, c6;
            lj_params<COMBINE>(sLJ, rowI, tj, ljI, ljJ, c12, c6);
            const float rinv = rsqrt_approx(r2);
            const float r = r2 * rinv;
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
            pair_terms<ELEC, VDW, true>(pc, rEff, r2E, rinvE, xi.w * xj.w, c12, c6, dEdr, E);
            dEdr *= s;
            if (pert) {  // dU/dlambda routing, nbdirect.cu:400-415
              const float fl = fmaf(dEdr, dredll, E);
              if (sameSite) {
                if (bi == bj) fli += fl;
              } else {
                fli = fmaf(lj, fl, fli);
                flj = fmaf(li, fl, flj);
              }
            }
            const float fs = dEdr * dredr * rinv;
            fix = fmaf(fs, dx, fix); fiy = fmaf(fs, dy, fiy); fiz = fmaf(fs, dz, fiz);
            fjx = fmaf(-fs, dx, fjx); fjy = fmaf(-fs, dy, fjy); fjz = fmaf(-fs, dz, fjz);
            if (ENERGY) ei = fmaf(s, E, ei);
            if (A.count) pairs++;
          }
          mr >>= 1;
          xj.x = __shfl_sync(kFull, xj.x, srcLane);
          xj.y = __shfl_sync(kFull, xj.y, srcLane);
          xj.z = __shfl_sync(kFull, xj.z, srcLane);
          xj.w = __shfl_sync(kFull, xj.w, srcLane);
          if (COMBINE) {
            ljJ.x = __shfl_sync(kFull, ljJ.x, srcLane);
            ljJ.y = __shfl_sync(kFull, ljJ.y, srcLane);
          } else {
            tj = __shfl_sync(kFull, tj, srcLane);
          }
          bj = __shfl_sync(kFull, bj, srcLane);
          lj = __shfl_sync(kFull, lj, srcLane);
          fjx = __shfl_sync(kFull, fjx, srcLane);
          fjy = __shfl_sync(kFull, fjy, srcLane);
          fjz = __shfl_sync(kFull, fjz, srcLane);
          flj = __shfl_sync(kFull, flj, srcLane);
        }
      }
      // j force of this tile is back in its owner lane
      if (jValid && (fjx != 0.f || fjy != 0.f || fjz != 0.f)) {
        red_add(&d.accF[jslot], to_fix(fjx));
        red_add(&d.accF[S + jslot], to_fix(fjy));
        red_add(&d.accF[2 * S + jslot], to_fix(fjz));
        if (!(isfinite(fjx) && isfinite(fjy) && isfinite(fjz))) atomicOr(&d.ctr->status, kStatusNonFinite);
      }
      if (ALCH && bj && flj != 0.f) atomicAdd(reinterpret_cast<unsigned long long *>(&sAccL[bj & 0xFFFF]),
                                              static_cast<unsigned long long>(to_fix(flj)));
    }
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
      long long e = to_fix(ei);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(kFull, e, o);
      if (lane == 0 && e != 0) red_add(&d.accE[d.blockRep[iBlock]], e);
    }
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

// Converts the fixed-point accumulators to the caller's outputs and clears them.
__global__ void k_finalize(Dev d, bnb_outputs o) {
  const int S = 32 * d.maxBlocks;
  const int B = d.ctr->blockCount;
  const double inv = 1.0 / kFixScale;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 32 * B; t += gridDim.x * blockDim.x) {
    int a = d.slotAtom[t];
    if (a < 0) continue;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      long long v = d.accF[k * S + t];
      d.accF[k * S + t] = 0;
      double f = (double)v * inv;
      if (o.force64) o.force64[3 * a + k] = f;
      if (o.force && v) atomicAdd(&o.force[3 * a + k], (float)f);
    }
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < d.lamTotal; i += blockDim.x) {
      long long v = d.accL[i];
      d.accL[i] = 0;
      double f = (double)v * inv;
      if (o.lambdaForce64) o.lambdaForce64[i] = f;
      if (o.lambdaForce && v) atomicAdd(&o.lambdaForce[i], (float)f);
    }
    for (int r = threadIdx.x; r < d.R; r += blockDim.x) {
      long long v = d.accE[r];
      d.accE[r] = 0;
      double e = (double)v * inv;
      if (o.energy64) o.energy64[r] = e;
      if (o.energy) o.energy[r] += e;
    }
  }
}

template <int ELEC, int VDW, int ALCH, bool ENERGY, bool COMBINE>
void launch_t(const KArgs &a, int grid, size_t shmem, cudaStream_t s) {
  auto k = k_pair<ELEC, VDW, ALCH, ENERGY, COMBINE>;
  if (shmem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
  k<<<grid, 256, shmem, s>>>(a);
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

}  // namespace

int launch_pair(const Dev &d, const PairConst &pc, const float *lambda, int elec, int vdw,
                int alch, bool energy, bool count, int grid, cudaStream_t s) {
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

void launch_finalize(const Dev &d, const bnb_outputs &o, cudaStream_t s) {
  int n = 32 * d.maxBlocks;
  int grid = (n + 255) / 256;
  if (grid > 148 * 8) grid = 148 * 8;
  if (grid < 1) grid = 1;
  k_finalize<<<grid, 256, 0, s>>>(d, o);
}

}  // namespace bnb
