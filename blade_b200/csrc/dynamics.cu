// Langevin VRORV update of coordinates and MSLD theta (sm_100a), FP64 state.
//
// The batched MSLD step needs an integrator after the force call.  This is
// the reference's leapfrog Langevin scheme (src/update/update.cu:233-305,
// "VRORV": update_VVhbpR then update_OOhbpR, after Leimkuhler & Matthews,
// dx.doi.org/10.1098/rspa.2016.0138) restated as one kernel over all degrees
// of freedom of all replicas:
//   v -= dt * ism^2 * dU/dx;  x += dt/2 v;  v = a v + b ism xi;  x += dt/2 v
// with a = exp(-gamma dt), b = sqrt((1 - a^2) kT) and ism = 1/sqrt(m).
// Degrees of freedom with non-finite ism are frozen, as in the reference.
// Gaussian numbers come from a counter-based generator (SplitMix64 mixing of
// seed, step and index, Steele/Lea/Flood 2014; Box-Muller transform), so a
// step has no RNG state and can be captured in a CUDA graph; the reference
// draws them from cuRAND MTGP32 instead (same distribution, different stream).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "bnb.h"

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double gaussian(uint64_t seed, uint64_t step, uint64_t i) {
  uint64_t a = splitmix64(seed ^ splitmix64(step * 0x2545F4914F6CDD1Dull + i));
  uint64_t b = splitmix64(a);
  double u1 = ((a >> 11) + 1) * (1.0 / 9007199254740993.0);  // (0, 1]
  double u2 = (b >> 11) * (1.0 / 9007199254740992.0);        // [0, 1)
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

__global__ void k_vrorv(int nx, int nt, double *x, double *v, const double *fx, const double *ismx,
                        double *th, double *vt, const double *ft, const double *ismt, double dt,
                        double ax, double bx, double at, double bt, uint64_t seed, uint64_t step,
                        unsigned long long *stepCounter, float *x_f, int *nanFlag) {
  __shared__ bool lastBlock;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (stepCounter) step += stepCounter[0];
  if (i < nx + nt) {
  const bool spatial = i < nx;
  const int k = spatial ? i : i - nx;
  double *X = spatial ? x : th;
  double *V = spatial ? v : vt;
  const double f = spatial ? fx[k] : ft[k];
  const double ism = spatial ? ismx[k] : ismt[k];
  const double a = spatial ? ax : at, b = spatial ? bx : bt;
  double xv = X[k];
  if (isfinite(ism)) {
    double vv = V[k] - dt * ism * ism * f;
    xv += 0.5 * dt * vv;
    vv = a * vv + b * ism * gaussian(seed, step, (uint64_t)i);
    xv += 0.5 * dt * vv;
    V[k] = vv;
    X[k] = xv;
    if (!isfinite(vv) && nanFlag) atomicMax(nanFlag, 1);
  }
  if (spatial && x_f) x_f[k] = (float)xv;
  }
  // Advance the device step counter once every block has read it: the last
  // block to finish increments it (graph replays then draw fresh noise).
  if (stepCounter) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      unsigned long long done = atomicAdd(&stepCounter[1], 1ull);
      lastBlock = done == gridDim.x - 1;
    }
    __syncthreads();
    if (lastBlock && threadIdx.x == 0) {
      stepCounter[1] = 0;
      __threadfence();
      atomicAdd(&stepCounter[0], 1ull);
    }
  }
}

// The same step split at the middle for holonomic constraints, which act
// after each half drift (update_VVhbpR / update_OOhbpR, update.cu:276-303):
//   phase 0:  v -= dt ism^2 dU/dx;  xPrev = x;  x += dt/2 v
//   phase 1:  v = a v + b ism xi;   xPrev = x;  x += dt/2 v
// Without constraints the two phases give the bits of k_vrorv (same
// operations in the same order, same noise index); phase 1 advances the
// device step counter.
__global__ void k_langevin_half(int phase, int nx, int nt, double *x, double *v, double *xPrev, const double *fx,
                                const double *ismx, double *th, double *vt, const double *ft, const double *ismt,
                                double dt, double ax, double bx, double at, double bt, uint64_t seed, uint64_t step,
                                unsigned long long *stepCounter, float *x_f, int *nanFlag) {
  __shared__ bool lastBlock;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (stepCounter) step += stepCounter[0];
  if (i < nx + nt) {
    const bool spatial = i < nx;
    const int k = spatial ? i : i - nx;
    double *X = spatial ? x : th;
    double *V = spatial ? v : vt;
    const double ism = spatial ? ismx[k] : ismt[k];
    double xv = X[k];
    if (spatial && xPrev) xPrev[k] = xv;
    if (isfinite(ism)) {
      double vv = V[k];
      if (phase == 0) {
        vv -= dt * ism * ism * (spatial ? fx[k] : ft[k]);
      } else {
        const double a = spatial ? ax : at, b = spatial ? bx : bt;
        vv = a * vv + b * ism * gaussian(seed, step, (uint64_t)i);
      }
      xv += 0.5 * dt * vv;
      V[k] = vv;
      X[k] = xv;
      if (!isfinite(vv) && nanFlag) atomicMax(nanFlag, 1);
    }
    if (spatial && x_f && phase == 1) x_f[k] = (float)xv;
  }
  if (stepCounter && phase == 1) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      unsigned long long done = atomicAdd(&stepCounter[1], 1ull);
      lastBlock = done == gridDim.x - 1;
    }
    __syncthreads();
    if (lastBlock && threadIdx.x == 0) {
      stepCounter[1] = 0;
      __threadfence();
      atomicAdd(&stepCounter[0], 1ull);
    }
  }
}

// Harmonic bonds, gathered per atom: thread a walks its own CSR row of bond
// partners in stored order and adds sum_b kb (r - b0) (x_a - x_b) / r to
// grad[a] -- each bond is evaluated from both ends, which keeps the sum
// order fixed (no atomics) and the result reproducible bit for bit.
__global__ void k_bonds(int n, const int *start, const int *partner, const float2 *kb_b0, const double *x,
                        double *grad) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const double xa = x[3 * a], ya = x[3 * a + 1], za = x[3 * a + 2];
  double gx = 0, gy = 0, gz = 0;
  for (int e = start[a]; e < start[a + 1]; ++e) {
    const int b = partner[e];
    const float2 p = kb_b0[e];
    const double dx = xa - x[3 * b], dy = ya - x[3 * b + 1], dz = za - x[3 * b + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double s = r > 0 ? (double)p.x * (r - (double)p.y) / r : 0.0;
    gx += s * dx;
    gy += s * dy;
    gz += s * dz;
  }
  grad[3 * a] += gx;
  grad[3 * a + 1] += gy;
  grad[3 * a + 2] += gz;
}

}  // namespace

extern "C" int bnb_bond_gradient(int n, const int *start, const int *partner, const float *kbB0,
                                 const double *x, double *grad, void *stream) {
  if (n < 0 || (n > 0 && (!start || !partner || !kbB0 || !x || !grad))) return BNB_ERR_ARG;
  if (n == 0) return BNB_OK;
  k_bonds<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, start, partner, (const float2 *)kbB0, x, grad);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_langevin_vrorv(int nx, int nt, double *x, double *v, const double *fx,
                                  const double *ismx, double *theta, double *vtheta, const double *ftheta,
                                  const double *ismtheta, double dt, double frictionX, double noiseX,
                                  double frictionTheta, double noiseTheta, unsigned long long seed,
                                  unsigned long long step, unsigned long long *stepCounter, float *x_f,
                                  int *nanFlag, void *stream) {
  if (nx < 0 || nt < 0 || (nx > 0 && (!x || !v || !fx || !ismx)) ||
      (nt > 0 && (!theta || !vtheta || !ftheta || !ismtheta)))
    return BNB_ERR_ARG;
  int n = nx + nt;
  if (n == 0) return BNB_OK;
  k_vrorv<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(nx, nt, x, v, fx, ismx, theta, vtheta, ftheta,
                                                             ismtheta, dt, frictionX, noiseX, frictionTheta,
                                                             noiseTheta, seed, step, stepCounter, x_f, nanFlag);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_langevin_half(int phase, int nx, int nt, double *x, double *v, double *xPrev, const double *fx,
                                 const double *ismx, double *theta, double *vtheta, const double *ftheta,
                                 const double *ismtheta, double dt, double frictionX, double noiseX,
                                 double frictionTheta, double noiseTheta, unsigned long long seed,
                                 unsigned long long step, unsigned long long *stepCounter, float *x_f,
                                 int *nanFlag, void *stream) {
  if ((phase != 0 && phase != 1) || nx < 0 || nt < 0 || (nx > 0 && (!x || !v || !ismx || (phase == 0 && !fx))) ||
      (nt > 0 && (!theta || !vtheta || !ismtheta || (phase == 0 && !ftheta))))
    return BNB_ERR_ARG;
  int n = nx + nt;
  if (n == 0) return BNB_OK;
  k_langevin_half<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(phase, nx, nt, x, v, xPrev, fx, ismx, theta,
                                                                     vtheta, ftheta, ismtheta, dt, frictionX, noiseX,
                                                                     frictionTheta, noiseTheta, seed, step,
                                                                     stepCounter, x_f, nanFlag);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}
