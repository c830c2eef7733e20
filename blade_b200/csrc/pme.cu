// PME reciprocal space and Ewald self term (sm_100a).
//
// Counterpart of getforce_ewald and getforce_ewaldself
// (src/nbrecip/nbrecip.cu:19-555).  The algorithm is the reference's smooth
// PME: lambda-scaled charges are spread with order-n cardinal B-splines
// (grid point (floor(u) + t) mod K takes M_n(u - floor(u) + n - 1 - t),
// u = x K / L; nbrecip.cu:85-213), the unnormalised R2C spectrum is
// multiplied by B(m) exp(-pi^2 k^2 / beta^2) / (2 pi V k^2) (nbrecip.cu:
// 215-256), the C2R result is the potential grid and the gather returns
// dU/dx = 2 lambda q (K / L) sum dM M M phi, dU/dlambda = 2 q phi and
// E = lambda q phi (nbrecip.cu:258-465).  Charges arrive scaled by
// sqrt(kElectric), so the influence function carries no kElectric.
// Differences by design:
//   * the charge grid accumulates in int64 fixed point (2^-32), so the grid,
//     and with it every output, is identical run to run;
//   * u is formed in FP64 and wrapped with floor/mod, so any unwrapped
//     coordinate lands on the right grid point;
//   * lanes of an atom's 8-lane group own z offsets (contiguous grid
//     addresses within one instruction) instead of x/y/z parity classes;
//   * R replicas with their own grids in one launch per phase.
// Triclinic cells (the reference's flagBox branch): the fractional
// coordinates s = H^-1 x of the cell matrix H (columns A, B, C) replace x / L
// (nbrecip.cu:116-178), here by back substitution in FP64; the wave vectors
// are H^-T m (nbrecip.cu:236-242) and dU/dx = H^-T dU/ds (nbrecip.cu:456-462),
// with H^-1 as the reference's State::kTricBox_f (state.cxx:485-491).
// Orthorhombic handles keep the plain per-dimension path.
// The 3-D FFTs are cuFFT plans (one batched plan per run of consecutive
// replicas with equal grids), as in the reference.
#include <cuda_runtime.h>

#include "pme.h"

namespace bnb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ long long to_fix(float v) { return __float2ll_rn(v * kFixScaleF); }

__device__ __forceinline__ void red_add(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

// w[t] = M_n(f + n - 1 - t) and dw[t] = M_n'(f + n - 1 - t), t = 0..n-1, from
// the Cox-de Boor recursion M_k(x) = (x M_{k-1}(x) + (k - x) M_{k-1}(x - 1))
// / (k - 1) on the points x = f + j, and M_n'(x) = M_{n-1}(x) - M_{n-1}(x-1).
template <int ORDER>
__device__ __forceinline__ void bspline(float f, float (&w)[ORDER], float (&dw)[ORDER]) {
  float a[ORDER];
  float prev[ORDER];
  a[0] = 1.f;
#pragma unroll
  for (int j = 1; j < ORDER; j++) a[j] = 0.f;
#pragma unroll
  for (int k = 2; k <= ORDER; k++) {
    if (k == ORDER) {
#pragma unroll
      for (int j = 0; j < ORDER; j++) prev[j] = a[j];
    }
    const float inv = 1.f / (float)(k - 1);
#pragma unroll
    for (int j = k - 1; j >= 0; j--) {
      const float x = f + (float)j;
      const float left = j < k - 1 ? a[j] : 0.f;
      const float right = j >= 1 ? a[j - 1] : 0.f;
      a[j] = fmaf(x, left, ((float)k - x) * right) * inv;
    }
  }
#pragma unroll
  for (int t = 0; t < ORDER; t++) {
    const int j = ORDER - 1 - t;
    w[t] = a[j];
    dw[t] = (j < ORDER - 1 ? prev[j] : 0.f) - (j >= 1 ? prev[j - 1] : 0.f);
  }
}

// Grid coordinate of one dimension: first grid index (mod K) and fraction.
__device__ __forceinline__ void grid_coord(float x, int K, float L, int &i0, float &frac) {
  const double u = (double)x * (double)K / (double)L;
  const double u0 = floor(u);
  frac = (float)(u - u0);
  double m = u0 - (double)K * floor(u0 / (double)K);
  i0 = (int)m;
  if (i0 >= K) i0 -= K;  // m rounds to K only when u0 is a tiny negative multiple
  if (i0 < 0) i0 += K;
}

// Grid index (mod K) and fraction of a coordinate already in grid units.
__device__ __forceinline__ void grid_index(double u, int K, int &i0, float &frac) {
  const double u0 = floor(u);
  frac = (float)(u - u0);
  double m = u0 - (double)K * floor(u0 / (double)K);
  i0 = (int)m;
  if (i0 >= K) i0 -= K;
  if (i0 < 0) i0 += K;
}

// Grid coordinates of an atom in its replica's cell (both box types).
__device__ __forceinline__ void grid_coords(const PmeArgs &a, const float *x, const PmeRep &pr, const RepInfo &ri,
                                            int (&i0)[3], float (&f)[3]) {
  if (!a.tric) {
    for (int d = 0; d < 3; d++) grid_coord(x[d], pr.K[d], ri.box[d], i0[d], f[d]);
    return;
  }
  // box = (A_x, B_y, C_z), tric = (B_x, C_x, C_y)
  const double sz = (double)x[2] / (double)ri.box[2];
  const double sy = ((double)x[1] - (double)ri.tric[2] * sz) / (double)ri.box[1];
  const double sx = ((double)x[0] - (double)ri.tric[0] * sy - (double)ri.tric[1] * sz) / (double)ri.box[0];
  grid_index(sx * pr.K[0], pr.K[0], i0[0], f[0]);
  grid_index(sy * pr.K[1], pr.K[1], i0[1], f[1]);
  grid_index(sz * pr.K[2], pr.K[2], i0[2], f[2]);
}

// H^-1 of a triclinic cell as (xx, xy, xz, yy, yz, zz), FP32 like the
// reference's kTricBox_f.
struct RecipCell {
  float xx, xy, xz, yy, yz, zz;
};
__device__ __forceinline__ RecipCell recip_cell(const RepInfo &ri) {
  const float ax = ri.box[0], by = ri.box[1], cz = ri.box[2];
  const float bx = ri.tric[0], cx = ri.tric[1], cy = ri.tric[2];
  const float vinv = 1.f / (ax * by * cz);
  RecipCell k;
  k.xx = by * cz * vinv;
  k.xy = -bx * cz * vinv;
  k.xz = (bx * cy - by * cx) * vinv;
  k.yy = cz * ax * vinv;
  k.yz = -cy * ax * vinv;
  k.zz = ax * by * vinv;
  return k;
}

__device__ __forceinline__ float atom_scale(const PmeArgs &a, int atom, int &block) {
  block = a.siteBlock[atom] & 0xFFFF;
  return (block && a.lambda) ? a.lambda[block] : 1.f;
}

// ---------------------------------------------------------------------------
// Spread: 8 lanes per atom; lane g < ORDER owns z offset g and visits the
// ORDER x ORDER (x, y) offsets.
// ---------------------------------------------------------------------------
template <int ORDER>
__global__ void __launch_bounds__(256) k_spread(PmeArgs a) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int atom = t >> 3, g = t & 7;
  if (atom >= a.N || g >= ORDER) return;
  const int r = a.atomRep[atom];
  const PmeRep pr = a.prep[r];
  const RepInfo &ri = a.rep[r];
  int block;
  const float qe = a.q[atom] * atom_scale(a, atom, block);
  if (qe == 0.f) return;
  float wx[ORDER], wy[ORDER], wz[ORDER], d[ORDER];
  int i0[3];
  float f[3];
  grid_coords(a, a.x + 3 * atom, pr, ri, i0, f);
  const int ix0 = i0[0], iy0 = i0[1], iz0 = i0[2];
  bspline<ORDER>(f[0], wx, d);
  bspline<ORDER>(f[1], wy, d);
  bspline<ORDER>(f[2], wz, d);
  float wzg = wz[0];
#pragma unroll
  for (int k = 1; k < ORDER; k++) wzg = g == k ? wz[k] : wzg;
  const float qz = qe * wzg;
  int iz = iz0 + g;
  if (iz >= pr.K[2]) iz -= pr.K[2];
  long long *base = a.qfix + pr.gridOff;
#pragma unroll
  for (int tx = 0; tx < ORDER; tx++) {
    int ix = ix0 + tx;
    if (ix >= pr.K[0]) ix -= pr.K[0];
    const float qx = qz * wx[tx];
#pragma unroll
    for (int ty = 0; ty < ORDER; ty++) {
      int iy = iy0 + ty;
      if (iy >= pr.K[1]) iy -= pr.K[1];
      red_add(base + ((size_t)ix * pr.K[1] + iy) * pr.K[2] + iz, to_fix(qx * wy[ty]));
    }
  }
}

// Fixed point -> FP32 grid, clearing the fixed-point grid for the next call.
__global__ void k_fix_to_grid(PmeArgs a) {
  pdl_wait();
  const double inv = 1.0 / kFixScale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.totalGrid; i += gridDim.x * blockDim.x) {
    const long long v = a.qfix[i];
    a.grid[i] = (float)((double)v * inv);
    if (v) a.qfix[i] = 0;
  }
}

// ---------------------------------------------------------------------------
// Convolution: blockIdx.y = replica, threads stride over its half spectrum.
// FP32 like the reference's kernel (nbrecip.cu:215-256).
// ---------------------------------------------------------------------------
__global__ void k_convolve(PmeArgs a) {
  pdl_wait();
  const int r = blockIdx.y;
  const PmeRep pr = a.prep[r];
  const RepInfo &ri = a.rep[r];
  const int K0 = pr.K[0], K1 = pr.K[1], K2h = pr.K[2] / 2 + 1;
  const int n = K0 * K1 * K2h;
  const float ix = 1.f / ri.box[0], iy = 1.f / ri.box[1], iz = 1.f / ri.box[2];
  const RecipCell rc = a.tric ? recip_cell(ri) : RecipCell{};
  const float c = (float)(1.0 / (2.0 * kPi * (double)ri.box[0] * (double)ri.box[1] * (double)ri.box[2]));
  const float g = (float)(kPi * kPi / ((double)a.beta * (double)a.beta));
  const float *m0 = a.mod + pr.modOff, *m1 = m0 + K0, *m2 = m1 + K1;
  float2 *spec = a.cplx + pr.cplxOff;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int k = e % K2h;
    const int row = e / K2h;
    const int j = row % K1;
    const int i = row / K1;
    const float mi = (float)(2 * i <= K0 ? i : i - K0), mj = (float)(2 * j <= K1 ? j : j - K1), mk = (float)k;
    float kx, ky, kz;
    if (!a.tric) {
      kx = mi * ix;
      ky = mj * iy;
      kz = mk * iz;
    } else {  // k = H^-T m
      kx = mi * rc.xx;
      ky = fmaf(mi, rc.xy, mj * rc.yy);
      kz = fmaf(mi, rc.xz, fmaf(mj, rc.yz, mk * rc.zz));
    }
    const float k2 = fmaf(kx, kx, fmaf(ky, ky, kz * kz));
    const float factor = e == 0 ? 0.f : m0[i] * m1[j] * m2[k] * c * expf(-g * k2) / k2;
    float2 v = spec[e];
    v.x *= factor;
    v.y *= factor;
    spec[e] = v;
  }
}

// lambda and energy accumulators -> outputs, by the calling CTA's threads.
__device__ void finalize_outputs(const PmeArgs &a, const bnb_outputs &o, bool energy) {
  const double inv = 1.0 / kFixScale;
  for (int i = threadIdx.x; i < a.lamTotal; i += blockDim.x) {
    const long long v = __ldcg(&a.accL[i]);
    a.accL[i] = 0;
    const double f = (double)v * inv;
    if (o.lambdaForce64) out64(&o.lambdaForce64[i], f, a.mode);
    if (o.lambdaForce) out32(&o.lambdaForce[i], (float)f, a.mode);
  }
  if (energy)
    for (int r = threadIdx.x; r < a.R; r += blockDim.x) {
      const long long v = __ldcg(&a.accE[r]);
      a.accE[r] = 0;
      const double e = (double)v * inv;
      if (o.energy64) out64(&o.energy64[r], e, a.mode);
      if (o.energy) outE(&o.energy[r], e, a.mode);
    }
}

// The last CTA of a launch to finish writes the lambda and energy outputs
// (every CTA's reductions are fenced before it takes its ticket), so no
// separate finalize launch follows the gather.
__device__ void finalize_if_last(const PmeArgs &a, const bnb_outputs &o, bool energy) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_outputs(a, o, energy);
  if (threadIdx.x == 0) *a.done = 0;  // ready for the next launch
}

// ---------------------------------------------------------------------------
// Gather: same lane layout as the spread; the 8 lanes of an atom reduce with
// xor shuffles, lane 0 of the group writes the atom's outputs.
// ---------------------------------------------------------------------------
template <int ORDER, bool ENERGY>
__global__ void __launch_bounds__(256) k_gather(PmeArgs a, bnb_outputs o) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int atom = t >> 3, g = t & 7;
  const bool valid = atom < a.N;
  float phi = 0.f, gx = 0.f, gy = 0.f, gz = 0.f, qe = 0.f, qraw = 0.f;
  int r = 0, block = 0;
  PmeRep pr{};
  if (valid) {
    r = a.atomRep[atom];
    pr = a.prep[r];
    const RepInfo &ri = a.rep[r];
    qraw = a.q[atom];
    qe = qraw * atom_scale(a, atom, block);
    if (g < ORDER) {
      float wx[ORDER], wy[ORDER], wz[ORDER], dx[ORDER], dy[ORDER], dz[ORDER];
      int i0[3];
      float f[3];
      grid_coords(a, a.x + 3 * atom, pr, ri, i0, f);
      const int ix0 = i0[0], iy0 = i0[1], iz0 = i0[2];
      bspline<ORDER>(f[0], wx, dx);
      bspline<ORDER>(f[1], wy, dy);
      bspline<ORDER>(f[2], wz, dz);
      float wzg = wz[0], dzg = dz[0];
#pragma unroll
      for (int k = 1; k < ORDER; k++) {
        wzg = g == k ? wz[k] : wzg;
        dzg = g == k ? dz[k] : dzg;
      }
      int iz = iz0 + g;
      if (iz >= pr.K[2]) iz -= pr.K[2];
      const float *base = a.grid + pr.gridOff;
#pragma unroll
      for (int tx = 0; tx < ORDER; tx++) {
        int ix = ix0 + tx;
        if (ix >= pr.K[0]) ix -= pr.K[0];
        float p = 0.f, py = 0.f;  // sum over y of P wy, P dy
#pragma unroll
        for (int ty = 0; ty < ORDER; ty++) {
          int iy = iy0 + ty;
          if (iy >= pr.K[1]) iy -= pr.K[1];
          const float P = __ldg(base + ((size_t)ix * pr.K[1] + iy) * pr.K[2] + iz);
          p = fmaf(P, wy[ty], p);
          py = fmaf(P, dy[ty], py);
        }
        phi = fmaf(wx[tx], p, phi);
        gx = fmaf(dx[tx], p, gx);
        gy = fmaf(wx[tx], py, gy);
      }
      gz = phi * dzg;
      phi *= wzg;
      gx *= wzg;
      gy *= wzg;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    phi += __shfl_xor_sync(kFull, phi, o);
    gx += __shfl_xor_sync(kFull, gx, o);
    gy += __shfl_xor_sync(kFull, gy, o);
    gz += __shfl_xor_sync(kFull, gz, o);
  }
  float e = 0.f;
  if (valid && g == 0) {
    const RepInfo &ri = a.rep[r];
    const float c = 2.f * qe;
    float fx, fy, fz;
    if (!a.tric) {
      fx = c * gx * ((float)pr.K[0] / ri.box[0]);
      fy = c * gy * ((float)pr.K[1] / ri.box[1]);
      fz = c * gz * ((float)pr.K[2] / ri.box[2]);
    } else {  // dU/dx = H^-T dU/ds
      const RecipCell k = recip_cell(ri);
      const float hx = c * gx * (float)pr.K[0], hy = c * gy * (float)pr.K[1], hz = c * gz * (float)pr.K[2];
      fx = hx * k.xx;
      fy = fmaf(hx, k.xy, hy * k.yy);
      fz = fmaf(hx, k.xz, fmaf(hy, k.yz, hz * k.zz));
    }
    if (o.force64) {
      out64(&o.force64[3 * atom], fx, a.mode);
      out64(&o.force64[3 * atom + 1], fy, a.mode);
      out64(&o.force64[3 * atom + 2], fz, a.mode);
    }
    if (o.force) {
      out32(&o.force[3 * atom], fx, a.mode);
      out32(&o.force[3 * atom + 1], fy, a.mode);
      out32(&o.force[3 * atom + 2], fz, a.mode);
    }
    if (block) red_add(&a.accL[block], to_fix(2.f * qraw * phi));
    if (ENERGY) e = qe * phi;
  }
  if (ENERGY) {
    // one atomic per warp when its 4 atoms share a replica
    const int r0 = __shfl_sync(kFull, r, 0);
    const bool same = __all_sync(kFull, !valid || r == r0);
    long long ef = to_fix(e);
    if (same) {
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) ef += __shfl_xor_sync(kFull, ef, o2);
      if (lane == 0 && ef) red_add(&a.accE[r0], ef);
    } else if (ef) {
      red_add(&a.accE[r], ef);
    }
  }
  finalize_if_last(a, o, ENERGY);
}

// ---------------------------------------------------------------------------
// Ewald self term: one thread per atom.
// ---------------------------------------------------------------------------
template <bool ENERGY>
__global__ void k_self(PmeArgs a, float pre, bnb_outputs o) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int atom = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = atom < a.N;
  float e = 0.f;
  int r = 0;
  if (valid) {
    r = a.atomRep[atom];
    int block;
    const float l = atom_scale(a, atom, block);
    const float q = a.q[atom];
    const float es = pre * q * q;
    if (block) red_add(&a.accL[block], to_fix(2.f * l * es));
    e = l * l * es;
  }
  if (ENERGY) {
    const int r0 = __shfl_sync(kFull, r, 0);
    const bool same = __all_sync(kFull, !valid || r == r0);
    long long ef = to_fix(e);
    if (same) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ef += __shfl_xor_sync(kFull, ef, o);
      if (lane == 0 && ef) red_add(&a.accE[r0], ef);
    } else if (ef) {
      red_add(&a.accE[r], ef);
    }
  }
  finalize_if_last(a, o, ENERGY);
}

// lambda and energy accumulators -> outputs when there are no atoms (one CTA).
__global__ void k_pme_finalize(PmeArgs a, bnb_outputs o, bool energy) {
  pdl_wait();
  finalize_outputs(a, o, energy);
}

inline int grid_of(long long threads, int block) {
  long long g = (threads + block - 1) / block;
  return (int)(g < 1 ? 1 : (g > 148LL * 64 ? 148LL * 64 : g));
}

}  // namespace

int pme_spread(const PmeArgs &a, cudaStream_t s) {
  if (a.N > 0) {
    const int grid = (int)((8LL * a.N + 255) / 256);
    switch (a.order) {
      case 4: launch_pdl(k_spread<4>, grid, 256, 0, s, a); break;
      case 6: launch_pdl(k_spread<6>, grid, 256, 0, s, a); break;
      case 8: launch_pdl(k_spread<8>, grid, 256, 0, s, a); break;
      default: return BNB_ERR_ARG;
    }
  }
  launch_pdl(k_fix_to_grid, grid_of(a.totalGrid, 256), 256, 0, s, a);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

int pme_convolve(const PmeArgs &a, cudaStream_t s) {
  int gx = (a.maxCplx + 1023) / 1024;  // about 4 elements per thread
  gx = gx < 1 ? 1 : gx;
  launch_pdl(k_convolve, dim3(gx, a.R), 256, 0, s, a);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

int pme_gather(const PmeArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s) {
  if (a.N > 0) {
    const int grid = (int)((8LL * a.N + 255) / 256);
    switch (a.order * 2 + (energy ? 1 : 0)) {
      case 8: launch_pdl(k_gather<4, false>, grid, 256, 0, s, a, o); break;
      case 9: launch_pdl(k_gather<4, true>, grid, 256, 0, s, a, o); break;
      case 12: launch_pdl(k_gather<6, false>, grid, 256, 0, s, a, o); break;
      case 13: launch_pdl(k_gather<6, true>, grid, 256, 0, s, a, o); break;
      case 16: launch_pdl(k_gather<8, false>, grid, 256, 0, s, a, o); break;
      case 17: launch_pdl(k_gather<8, true>, grid, 256, 0, s, a, o); break;
      default: return BNB_ERR_ARG;
    }
  } else {
    launch_pdl(k_pme_finalize, 1, 256, 0, s, a, o, energy);
  }
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

int pme_self(const PmeArgs &a, const bnb_outputs &o, bool energy, cudaStream_t s) {
  // -beta / sqrt(pi) (kElectric is inside the scaled charges)
  const float pre = (float)(-(double)a.beta / sqrt(kPi));
  if (a.N > 0) {
    const int grid = (a.N + 255) / 256;
    if (energy) launch_pdl(k_self<true>, grid, 256, 0, s, a, pre, o);
    else launch_pdl(k_self<false>, grid, 256, 0, s, a, pre, o);
  } else {
    launch_pdl(k_pme_finalize, 1, 256, 0, s, a, o, energy);
  }
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

}  // namespace bnb
