// nb14 and nbex pair lists (sm_100a): the 1-4 interactions and the PME
// correction of excluded pairs that the direct-space tiles skip.
//
// Counterpart of src/bonded/pair.cu: getforce_pair_kernel (pair.cu:205-283)
// with function_pair for Nb14Potential (pair.cu:63-187) and NbExPotential
// (pair.cu:190-202).  One thread per listed pair, minimum image in the
// pair's replica box; forces, dU/dlambda and energies go to int64 fixed-point
// accumulators (the i and j contributions are exact negatives, totals do not
// depend on the order of the atomics), which a finalize pass converts to the
// caller's outputs in atom order.  The pair math is FP32 like the
// reference's single-precision build; erfc/erf/exp are CUDA's functions.
#include <cuda_runtime.h>
#include <math.h>

#include "bnb.h"
#include "bnb_internal.h"
#include "pairs.h"

namespace bnb {
namespace {

constexpr float kTwoOverSqrtPi = 1.128379167095513f;

__device__ __forceinline__ long long fix(float v) { return __float2ll_rn(v * kFixScaleF); }
__device__ __forceinline__ void radd(long long *p, long long v) {
  if (v) atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// function_pair(Nb14Potential...): dE/dr and E (pair.cu:63-187).
template <int ELEC, int VDW>
__device__ __forceinline__ void nb14_terms(const PairsArgs &a, const bnb_nb14 &pp, float r, float &fpair,
                                           float &E) {
  fpair = 0.f;
  E = 0.f;
  if (!(r < a.rCut)) return;
  const float rinv = 1.f / r, rinv3 = rinv * rinv * rinv, rinv6 = rinv3 * rinv3;
  const float rc = a.rCut, rs = a.rSwitch;
  if (VDW == 0) {  // VFSWITCH, pair.cu:70-93
    const float rc3 = rc * rc * rc, rc6 = rc3 * rc3, rs3 = rs * rs * rs, rs6 = rs3 * rs3;
    const bool in = r < rs;
    const float A6 = in ? 1.f : rc3 / (rc3 - rs3), A12 = in ? 1.f : rc6 / (rc6 - rs6);
    const float B6 = in ? 0.f : 1.f / rc3, B12 = in ? 0.f : 1.f / rc6;
    fpair = 6.f * pp.c6 * A6 * (rinv3 - B6) * rinv3 * rinv - 12.f * pp.c12 * A12 * (rinv6 - B12) * rinv6 * rinv;
    const float CC6 = in ? -1.f / rc6 : 0.f, CC12 = in ? -1.f / (rc6 * rc6) : 0.f;
    E = pp.c12 * (A12 * (rinv6 - B12) * (rinv6 - B12) + CC12) - pp.c6 * (A6 * (rinv3 - B6) * (rinv3 - B6) + CC6);
  } else if (VDW == 1) {  // VSWITCH, pair.cu:94-106
    const float c2of = rc * rc, c2on = rs * rs;
    const float rul3 = (c2of - c2on) * (c2of - c2on) * (c2of - c2on), rul12 = 12.f / rul3;
    const float rijl = c2on - r * r, riju = c2of - r * r;
    const float fsw = r < rs ? 1.f : riju * riju * (riju - 3.f * rijl) / rul3;
    const float dfsw = r < rs ? 0.f : rijl * riju * rul12;
    fpair = fsw * (6.f * pp.c6 - 12.f * pp.c12 * rinv6) * rinv6 * rinv + dfsw * (pp.c12 * rinv6 - pp.c6) * rinv6;
    E = fsw * (pp.c12 * rinv6 - pp.c6) * rinv6;
  } else {  // VSHIFT, pair.cu:107-133
    const float r2 = r * r, r5 = r2 * r2 * r, r6 = r2 * r2 * r2;
    const float rinv12 = rinv6 * rinv6;
    const float rc2 = rc * rc, rc6 = rc2 * rc2 * rc2, rc12 = rc6 * rc6, rc18 = rc12 * rc6;
    fpair = 6.f * pp.c6 * (rinv6 * rinv - r5 / rc12) - 12.f * pp.c12 * (rinv12 * rinv + r5 / rc18);
    E = pp.c12 * (rinv12 + 2.f * r6 / rc18 - 3.f / rc12) - pp.c6 * (rinv6 + r6 / rc12 - 2.f / rc6);
  }
  const float kqq = a.kElectric * pp.qxq;
  if (ELEC == 0) {  // FSWITCH, pair.cu:136-156
    const float k = kqq * pp.e14fac;
    const float roff2 = rc * rc, ron2 = rs * rs;
    const float ginv = 1.f / ((roff2 - ron2) * (roff2 - ron2) * (roff2 - ron2));
    const float Ac = roff2 * roff2 * (roff2 - 3.f * ron2) * ginv, Bc = 6.f * roff2 * ron2 * ginv;
    const float Cc = -(ron2 + roff2) * ginv, Dc = 2.f * ginv / 5.f;
    const float dvc = 8.f * (ron2 * roff2 * (rc - rs) - (roff2 * roff2 * rc - ron2 * ron2 * rs) / 5.f) * ginv;
    const float r2 = r * r, r3 = r2 * r, r5 = r3 * r2;
    fpair += r <= rs ? -k * rinv * rinv : -k * rinv * (Ac * rinv + Bc * r + 3.f * Cc * r3 + 5.f * Dc * r5);
    E += r <= rs ? k * (rinv + dvc)
                 : k * (Ac * (rinv - 1.f / rc) + Bc * (rc - r) + Cc * (roff2 * rc - r3) + Dc * (roff2 * roff2 * rc - r5));
  } else if (ELEC == 1) {  // PME, pair.cu:157-165
    const float br = a.beta * r;
    const float erfcrinv = (erfcf(br) + pp.e14fac - 1.f) * rinv;
    fpair += kqq * (-erfcrinv - kTwoOverSqrtPi * a.beta * expf(-br * br)) * rinv;
    E += kqq * erfcrinv;
  } else {  // FSHIFT, pair.cu:166-174
    const float k = kqq * pp.e14fac, roffinv = 1.f / rc;
    fpair += -k * (rinv * rinv - roffinv * roffinv);
    E += k * (rinv - 2.f * roffinv + r * roffinv * roffinv);
  }
}

__device__ __forceinline__ float3 min_image(const PairsArgs &a, int ii, int jj, float &r) {
  const RepInfo &ri = a.rep[a.atomRep[ii]];
  float3 d = make_float3(a.x[3 * ii] - a.x[3 * jj], a.x[3 * ii + 1] - a.x[3 * jj + 1],
                         a.x[3 * ii + 2] - a.x[3 * jj + 2]);
  if (ri.tric[0] == 0.f && ri.tric[1] == 0.f && ri.tric[2] == 0.f) {
    d.x -= ri.box[0] * rintf(d.x / ri.box[0]);
    d.y -= ri.box[1] * rintf(d.y / ri.box[1]);
    d.z -= ri.box[2] * rintf(d.z / ri.box[2]);
  } else {  // triclinic: by C, then B, then A (real3_subpbc<true>, src/main/real3.h:215-240)
    float i = rintf(d.z / ri.box[2]);
    d.x -= ri.tric[1] * i;
    d.y -= ri.tric[2] * i;
    d.z -= ri.box[2] * i;
    i = rintf(d.y / ri.box[1]);
    d.x -= ri.tric[0] * i;
    d.y -= ri.box[1] * i;
    d.x -= ri.box[0] * rintf(d.x / ri.box[0]);
  }
  r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  return d;
}

// Scaling l0*l1, dU/dlambda routing and force output of getforce_pair_kernel
// (pair.cu:224-283); dredr/dredll are 1/0 without soft core.
__device__ __forceinline__ void apply(const PairsArgs &a, int ii, int jj, const int sb[2], float3 d, float r,
                                      float fpair, float E, float l0, float l1, float dredr, float dredll,
                                      bool energy) {
  const int b0 = 0xFFFF & sb[0], b1 = 0xFFFF & sb[1];
  fpair *= l0 * l1;
  if (b0) {
    const float fl = E + fpair * dredll;
    radd(&a.accL[b0], fix(l1 * fl));
    if (b1) radd(&a.accL[b1], fix(l0 * fl));
  }
  fpair *= dredr;
  const float s = fpair / r;
  const long long fx = fix(s * d.x), fy = fix(s * d.y), fz = fix(s * d.z);
  radd(&a.accF[3 * ii], fx);
  radd(&a.accF[3 * ii + 1], fy);
  radd(&a.accF[3 * ii + 2], fz);
  radd(&a.accF[3 * jj], -fx);
  radd(&a.accF[3 * jj + 1], -fy);
  radd(&a.accF[3 * jj + 2], -fz);
  if (energy) radd(&a.accE[a.atomRep[ii]], fix(E * l0 * l1));
}

template <int ELEC, int VDW, bool SOFT, bool ENERGY>
__global__ void k_nb14(PairsArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n14) return;
  const bnb_nb14 pp = a.nb14[t];
  const int ii = pp.idx[0], jj = pp.idx[1];
  float r;
  const float3 d = min_image(a, ii, jj, r);
  const int b0 = 0xFFFF & pp.siteBlock[0], b1 = 0xFFFF & pp.siteBlock[1];
  float l0 = 1.f, l1 = 1.f;
  if (b0) {
    l0 = a.lambda[b0];
    if (b1) l1 = a.lambda[b1];
  }
  float rEff = r, dredr = 1.f, dredll = 0.f;
  if (SOFT && b0) {  // pair.cu:240-254
    const float rSoft = a.softR * (1.f - l0 * l1);
    if (r < rSoft) {
      const float q = r / rSoft;
      rEff = (1.f - 0.5f * q) * q * q * q + 0.5f;
      dredr = (3.f - 2.f * q) * q * q;
      dredll = -a.softR * (rEff - dredr * q);
      rEff *= rSoft;
    }
  }
  float fpair, E;
  nb14_terms<ELEC, VDW>(a, pp, rEff, fpair, E);
  apply(a, ii, jj, pp.siteBlock, d, r, fpair, E, l0, l1, dredr, dredll, ENERGY);
}

template <bool ENERGY>
__global__ void k_nbex(PairsArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.nex) return;
  const bnb_nbex pp = a.nbex[t];
  const int ii = pp.idx[0], jj = pp.idx[1];
  float r;
  const float3 d = min_image(a, ii, jj, r);
  const int b0 = 0xFFFF & pp.siteBlock[0], b1 = 0xFFFF & pp.siteBlock[1];
  float l0 = 1.f, l1 = 1.f;
  if (b0) {
    l0 = a.lambda[b0];
    if (b1) l1 = a.lambda[b1];
  }
  // function_pair(NbExPotential...), pair.cu:190-202: E = -kqq erf(br)/r
  const float rinv = 1.f / r, br = a.beta * r, kqq = a.kElectric * pp.qxq, ef = erff(br);
  const float fpair = kqq * (ef * rinv - kTwoOverSqrtPi * a.beta * expf(-br * br)) * rinv;
  const float E = -kqq * ef * rinv;
  apply(a, ii, jj, pp.siteBlock, d, r, fpair, E, l0, l1, 1.f, 0.f, ENERGY);
}

__global__ void k_pairs_finalize(PairsArgs a, bnb_outputs o) {
  const double inv = 1.0 / kFixScale;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * a.N; t += gridDim.x * blockDim.x) {
    const long long v = a.accF[t];
    if (v) a.accF[t] = 0;
    const double f = (double)v * inv;
    if (o.force64) out64(&o.force64[t], f, a.mode);
    if (o.force) out32(&o.force[t], (float)f, a.mode);
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < a.lamTotal; i += blockDim.x) {
      const long long v = a.accL[i];
      a.accL[i] = 0;
      const double f = (double)v * inv;
      if (o.lambdaForce64) out64(&o.lambdaForce64[i], f, a.mode);
      if (o.lambdaForce) out32(&o.lambdaForce[i], (float)f, a.mode);
    }
    for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
      const long long v = a.accE[r];
      a.accE[r] = 0;
      const double e = (double)v * inv;
      if (o.energy64) out64(&o.energy64[r], e, a.mode);
      if (o.energy) outE(&o.energy[r], e, a.mode);
    }
  }
}

template <int ELEC, int VDW>
void nb14_ev(const PairsArgs &a, bool soft, bool energy, int grid, cudaStream_t s) {
  if (soft) {
    if (energy) k_nb14<ELEC, VDW, true, true><<<grid, 256, 0, s>>>(a);
    else k_nb14<ELEC, VDW, true, false><<<grid, 256, 0, s>>>(a);
  } else {
    if (energy) k_nb14<ELEC, VDW, false, true><<<grid, 256, 0, s>>>(a);
    else k_nb14<ELEC, VDW, false, false><<<grid, 256, 0, s>>>(a);
  }
}

void finalize(const PairsArgs &a, const bnb_outputs &o, cudaStream_t s) {
  int grid = (3 * a.N + 255) / 256;
  grid = grid < 1 ? 1 : (grid > 148 * 8 ? 148 * 8 : grid);
  k_pairs_finalize<<<grid, 256, 0, s>>>(a, o);
}

}  // namespace

int launch_nb14(const PairsArgs &a, const bnb_outputs &o, int elec, int vdw, bool soft, bool energy,
                cudaStream_t s) {
  if (a.n14 > 0) {
    const int grid = (a.n14 + 255) / 256;
    switch (elec * 3 + vdw) {
      case 0: nb14_ev<0, 0>(a, soft, energy, grid, s); break;
      case 1: nb14_ev<0, 1>(a, soft, energy, grid, s); break;
      case 2: nb14_ev<0, 2>(a, soft, energy, grid, s); break;
      case 3: nb14_ev<1, 0>(a, soft, energy, grid, s); break;
      case 4: nb14_ev<1, 1>(a, soft, energy, grid, s); break;
      case 5: nb14_ev<1, 2>(a, soft, energy, grid, s); break;
      case 6: nb14_ev<2, 0>(a, soft, energy, grid, s); break;
      case 7: nb14_ev<2, 1>(a, soft, energy, grid, s); break;
      case 8: nb14_ev<2, 2>(a, soft, energy, grid, s); break;
      default: return BNB_ERR_ARG;
    }
    if (cudaGetLastError() != cudaSuccess) return BNB_ERR_CUDA;
  }
  finalize(a, o, s);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

int launch_nbex(const PairsArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s) {
  if (a.nex > 0) {
    const int grid = (a.nex + 255) / 256;
    if (energy) k_nbex<true><<<grid, 256, 0, s>>>(a);
    else k_nbex<false><<<grid, 256, 0, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return BNB_ERR_CUDA;
  }
  finalize(a, o, s);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

}  // namespace bnb
