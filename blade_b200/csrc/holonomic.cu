// Holonomic bond constraints of the batched step (sm_100a), FP64 state.
//
// Counterpart of holonomic_position / holonomic_velocity
// (src/holonomic/holonomic.cu:238-758) over the reference's constraint
// clusters (src/system/potential.h:120-138): rigid triangles (water) and a
// heavy atom with 1, 2 or 3 bonded hydrogens.  Position constraints follow
// each half drift of the leapfrog step (src/update/update.cu:276-303): the
// drifted positions x are corrected along the bond vectors of the positions
// before the drift, xPrev, and the velocities become (x - xPrev) / (dt/2).
// Velocity constraints project the bond-direction relative velocities out.
//
// Every cluster type is solved the same way here: SHAKE with the full
// linearised constraint matrix (Ryckaert, Ciccotti & Berendsen 1977), one
// thread per cluster, iterated until |b0^2 - r^2| < 2 b0^2 tol for every
// bond (the reference's convergence test) or maxIter iterations.  The
// reference solves triangles analytically (SETTLE, Miyamoto & Kollman 1992)
// and one-bond clusters in closed form; both are the exact solutions of the
// same constraint problem, which the iteration reaches to the tolerance.
// Coordinates must be unwrapped (a cluster is never split across images),
// which the batched integrator guarantees.
#include <cuda_runtime.h>
#include <math.h>

#include "bnb.h"

namespace {

constexpr int kStatusNotConverged = 1;

// NA atoms, NC bonds (pa[c], pb[c]) of one cluster.
template <int NA, int NC>
struct Cluster {
  int idx[NA];
  int pa[NC], pb[NC];
  double b02[NC];
};

template <int NA, int NC>
__device__ __forceinline__ double coupling(const Cluster<NA, NC> &cl, const double *im, int c, int cp) {
  // d(x_pa(c) - x_pb(c)) per unit lambda_cp applied as x_pa(cp) += im d, x_pb(cp) -= im d
  double s = 0.0;
  if (cl.pa[c] == cl.pa[cp]) s += im[cl.pa[c]];
  if (cl.pa[c] == cl.pb[cp]) s -= im[cl.pa[c]];
  if (cl.pb[c] == cl.pa[cp]) s -= im[cl.pb[c]];
  if (cl.pb[c] == cl.pb[cp]) s += im[cl.pb[c]];
  return s;
}

// Solves A y = r for NC <= 3 (Gaussian elimination without pivoting: A is
// diagonally dominant for bond constraints near their lengths).
template <int NC>
__device__ __forceinline__ void solve(double (&A)[NC][NC], double (&r)[NC]) {
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const double inv = 1.0 / A[k][k];
#pragma unroll
    for (int i = k + 1; i < NC; i++) {
      const double f = A[i][k] * inv;
#pragma unroll
      for (int j = k; j < NC; j++) A[i][j] -= f * A[k][j];
      r[i] -= f * r[k];
    }
  }
#pragma unroll
  for (int k = NC - 1; k >= 0; k--) {
    double s = r[k];
#pragma unroll
    for (int j = k + 1; j < NC; j++) s -= A[k][j] * r[j];
    r[k] = s / A[k][k];
  }
}

template <int NA, int NC>
__device__ void constrain_position(const Cluster<NA, NC> &cl, const double *xPrev, double *x, double *v,
                                   const double *ism, double halfdt, double tol, int maxIter, float *x_f,
                                   int *status) {
  double xp[NA][3], xc[NA][3], im[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) {
    const int i = cl.idx[a];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      xp[a][k] = xPrev[3 * i + k];
      xc[a][k] = x[3 * i + k];
    }
    im[a] = ism[3 * i] * ism[3 * i];
  }
  double dp[NC][3];
#pragma unroll
  for (int c = 0; c < NC; c++)
#pragma unroll
    for (int k = 0; k < 3; k++) dp[c][k] = xp[cl.pa[c]][k] - xp[cl.pb[c]][k];
  bool done = false;
  for (int it = 0; it <= maxIter; it++) {
    double d[NC][3], r[NC];
    done = true;
#pragma unroll
    for (int c = 0; c < NC; c++) {
#pragma unroll
      for (int k = 0; k < 3; k++) d[c][k] = xc[cl.pa[c]][k] - xc[cl.pb[c]][k];
      r[c] = cl.b02[c] - (d[c][0] * d[c][0] + d[c][1] * d[c][1] + d[c][2] * d[c][2]);
      if (fabs(r[c]) >= 2.0 * cl.b02[c] * tol) done = false;
    }
    if (done || it == maxIter) break;
    double A[NC][NC];
#pragma unroll
    for (int c = 0; c < NC; c++)
#pragma unroll
      for (int cp = 0; cp < NC; cp++)
        A[c][cp] = 2.0 * (d[c][0] * dp[cp][0] + d[c][1] * dp[cp][1] + d[c][2] * dp[cp][2]) *
                   coupling(cl, im, c, cp);
    solve<NC>(A, r);
#pragma unroll
    for (int c = 0; c < NC; c++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        xc[cl.pa[c]][k] += r[c] * im[cl.pa[c]] * dp[c][k];
        xc[cl.pb[c]][k] -= r[c] * im[cl.pb[c]] * dp[c][k];
      }
  }
  if (!done && status) atomicOr(status, kStatusNotConverged);
  const double inv = 1.0 / halfdt;
#pragma unroll
  for (int a = 0; a < NA; a++) {
    const int i = cl.idx[a];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (v) v[3 * i + k] = (xc[a][k] - xp[a][k]) * inv;
      x[3 * i + k] = xc[a][k];
      if (x_f) x_f[3 * i + k] = (float)xc[a][k];
    }
  }
}

template <int NA, int NC>
__device__ void constrain_velocity(const Cluster<NA, NC> &cl, const double *x, double *v, const double *ism) {
  double xc[NA][3], vc[NA][3], im[NA];
#pragma unroll
  for (int a = 0; a < NA; a++) {
    const int i = cl.idx[a];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      xc[a][k] = x[3 * i + k];
      vc[a][k] = v[3 * i + k];
    }
    im[a] = ism[3 * i] * ism[3 * i];
  }
  double d[NC][3], r[NC], A[NC][NC];
#pragma unroll
  for (int c = 0; c < NC; c++) {
#pragma unroll
    for (int k = 0; k < 3; k++) d[c][k] = xc[cl.pa[c]][k] - xc[cl.pb[c]][k];
    r[c] = -((vc[cl.pa[c]][0] - vc[cl.pb[c]][0]) * d[c][0] + (vc[cl.pa[c]][1] - vc[cl.pb[c]][1]) * d[c][1] +
             (vc[cl.pa[c]][2] - vc[cl.pb[c]][2]) * d[c][2]);
  }
#pragma unroll
  for (int c = 0; c < NC; c++)
#pragma unroll
    for (int cp = 0; cp < NC; cp++)
      A[c][cp] = (d[c][0] * d[cp][0] + d[c][1] * d[cp][1] + d[c][2] * d[cp][2]) * coupling(cl, im, c, cp);
  solve<NC>(A, r);
#pragma unroll
  for (int c = 0; c < NC; c++)
#pragma unroll
    for (int k = 0; k < 3; k++) {
      vc[cl.pa[c]][k] += r[c] * im[cl.pa[c]] * d[c][k];
      vc[cl.pb[c]][k] -= r[c] * im[cl.pb[c]] * d[c][k];
    }
#pragma unroll
  for (int a = 0; a < NA; a++)
#pragma unroll
    for (int k = 0; k < 3; k++) v[3 * cl.idx[a] + k] = vc[a][k];
}

__device__ __forceinline__ Cluster<3, 3> triangle(const bnb_triangle_cons &t) {
  Cluster<3, 3> c;
  for (int a = 0; a < 3; a++) c.idx[a] = t.idx[a];
  // bonds 01, 02, 12 (the order of TriangleCons::b0)
  c.pa[0] = 0; c.pb[0] = 1;
  c.pa[1] = 0; c.pb[1] = 2;
  c.pa[2] = 1; c.pb[2] = 2;
  for (int k = 0; k < 3; k++) c.b02[k] = (double)t.b0[k] * (double)t.b0[k];
  return c;
}

template <int NH, typename T>
__device__ __forceinline__ Cluster<NH + 1, NH> branch(const T &t) {
  Cluster<NH + 1, NH> c;
  for (int a = 0; a < NH + 1; a++) c.idx[a] = t.idx[a];
  for (int k = 0; k < NH; k++) {
    c.pa[k] = 0;  // heavy atom first
    c.pb[k] = k + 1;
    c.b02[k] = (double)t.b0[k] * (double)t.b0[k];
  }
  return c;
}

__global__ void k_holonomic_position(bnb_constraints cs, const double *xPrev, double *x, double *v,
                                     const double *ism, double halfdt, double tol, int maxIter, float *x_f,
                                     int *status) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < cs.nTriangle) {
    constrain_position(triangle(cs.triangle[t]), xPrev, x, v, ism, halfdt, tol, maxIter, x_f, status);
    return;
  }
  t -= cs.nTriangle;
  if (t < cs.nBranch1) {
    constrain_position(branch<1>(cs.branch1[t]), xPrev, x, v, ism, halfdt, tol, maxIter, x_f, status);
    return;
  }
  t -= cs.nBranch1;
  if (t < cs.nBranch2) {
    constrain_position(branch<2>(cs.branch2[t]), xPrev, x, v, ism, halfdt, tol, maxIter, x_f, status);
    return;
  }
  t -= cs.nBranch2;
  if (t < cs.nBranch3)
    constrain_position(branch<3>(cs.branch3[t]), xPrev, x, v, ism, halfdt, tol, maxIter, x_f, status);
}

__global__ void k_holonomic_velocity(bnb_constraints cs, const double *x, double *v, const double *ism) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < cs.nTriangle) {
    constrain_velocity(triangle(cs.triangle[t]), x, v, ism);
    return;
  }
  t -= cs.nTriangle;
  if (t < cs.nBranch1) {
    constrain_velocity(branch<1>(cs.branch1[t]), x, v, ism);
    return;
  }
  t -= cs.nBranch1;
  if (t < cs.nBranch2) {
    constrain_velocity(branch<2>(cs.branch2[t]), x, v, ism);
    return;
  }
  t -= cs.nBranch2;
  if (t < cs.nBranch3) constrain_velocity(branch<3>(cs.branch3[t]), x, v, ism);
}

bool valid(const bnb_constraints *cs) {
  if (!cs || cs->nTriangle < 0 || cs->nBranch1 < 0 || cs->nBranch2 < 0 || cs->nBranch3 < 0) return false;
  return (!cs->nTriangle || cs->triangle) && (!cs->nBranch1 || cs->branch1) && (!cs->nBranch2 || cs->branch2) &&
         (!cs->nBranch3 || cs->branch3);
}

}  // namespace

extern "C" int bnb_holonomic_position(const bnb_constraints *cs, const double *xPrev, double *x, double *v,
                                      const double *ism, double halfdt, double tolerance, int maxIter,
                                      float *x_f, int *status, void *stream) {
  if (!valid(cs) || !xPrev || !x || !ism || !(halfdt > 0.0) || !(tolerance > 0.0) || maxIter < 1)
    return BNB_ERR_ARG;
  const long long n = (long long)cs->nTriangle + cs->nBranch1 + cs->nBranch2 + cs->nBranch3;
  if (n == 0) return BNB_OK;
  k_holonomic_position<<<(int)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(*cs, xPrev, x, v, ism, halfdt,
                                                                                tolerance, maxIter, x_f, status);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_holonomic_velocity(const bnb_constraints *cs, const double *x, double *v, const double *ism,
                                      void *stream) {
  if (!valid(cs) || !x || !v || !ism) return BNB_ERR_ARG;
  const long long n = (long long)cs->nTriangle + cs->nBranch1 + cs->nBranch2 + cs->nBranch3;
  if (n == 0) return BNB_OK;
  k_holonomic_velocity<<<(int)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(*cs, x, v, ism);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}
