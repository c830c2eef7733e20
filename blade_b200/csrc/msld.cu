// MSLD lambda maps and lambda biases (sm_100a), computed in FP64.
//
// Counterparts of Msld::calc_lambda_from_theta (src/msld/msld.cu:863-921),
// Msld::calc_thetaForce_from_lambdaForce (msld.cu:937-998) and the fixed and
// variable lambda biases (msld.cu:1000-1153).  These are tiny per-site /
// per-block / per-bias loops: one thread each.  Entry points come in the
// FP64 form and, for the buffers BLaDE's State keeps in FP32 (lambda_fd,
// theta_fd, lambdaForce_d, thetaForce_d, lambdaBias_d), an FP32-buffer form
// that still computes in FP64.  Block-fixed flags are byte arrays, the
// layout of the reference's bool blockFixed_d.  Energies are reduced in a
// fixed order per warp and added with one FP64 atomic per warp.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "bnb.h"

namespace {

__global__ void k_lambda_from_theta(int siteCount, const int *siteBound, double fnex,
                                    const double *theta, const uint8_t *fixed, double *lambda,
                                    float *lambda_f) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= siteCount) return;
  int j0 = siteBound[i], j1 = siteBound[i + 1];
  double fixsum = 0, norm = 0;
  for (int j = j0; j < j1; j++) {
    if (fixed && fixed[j]) {
      fixsum += theta[j];
    } else {
      double l = exp(fnex * sin(theta[j]));
      lambda[j] = l;
      norm += l;
    }
  }
  double rfrac = 1.0 - fixsum;
  if (norm > 0) norm = rfrac / norm;
  for (int j = j0; j < j1; j++) {
    double l = (fixed && fixed[j]) ? theta[j] : lambda[j] * norm;
    lambda[j] = l;
    if (lambda_f) lambda_f[j] = (float)l;
  }
}

template <typename L, typename F>
__global__ void k_theta_force(int blockCount, const int *lambdaSite, const int *siteBound, double fnex,
                              const L *lambda, const L *theta, const F *lambdaForce, const uint8_t *fixed,
                              F *thetaForce) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= blockCount) return;
  if (fixed && fixed[i]) return;
  int j0 = siteBound[lambdaSite[i]], j1 = siteBound[lambdaSite[i] + 1];
  double fixsum = 0, dyn = 0;
  for (int j = j0; j < j1; j++) {
    if (fixed && fixed[j]) fixsum += (double)lambda[j];
    else dyn += (double)lambda[j] * (double)lambdaForce[j];
  }
  double fi = lambdaForce[i];
  double rfrac = 1.0 - fixsum;
  if (rfrac > 0) fi -= dyn / rfrac;
  thetaForce[i] += (F)(fi * (double)lambda[i] * fnex * cos((double)theta[i]));
}

__device__ void warp_energy(double e, double *energy) {
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0 && e != 0.0) atomicAdd(energy, e);
}

template <typename L, typename F>
__global__ void k_bias(int blockCount, const L *lambda, const L *fixedBias, int nVar,
                       const bnb_varbias *vb, F *lambdaForce, double *energy) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0;
  if (fixedBias && t < blockCount) {
    atomicAdd(&lambdaForce[t], (F)fixedBias[t]);
    e += (double)fixedBias[t] * (double)lambda[t];
  }
  if (t < nVar) {
    bnb_varbias v = vb[t];
    double li = lambda[v.i], lj = lambda[v.j], k = v.k, l0 = v.l0, n = v.n;
    double E = 0, fi = 0, fj = 0;
    switch (v.type) {
      case 6: E = k * li * lj; fi = k * lj; fj = k * li; break;
      case 8: E = k * li * lj / (li + l0); fi = k * l0 * lj / ((li + l0) * (li + l0));
              fj = k * li / (li + l0); break;
      case 10: E = k * lj * (1 - exp(l0 * li)); fi = k * lj * (-l0 * exp(l0 * li));
               fj = k * (1 - exp(l0 * li)); break;
      case 1: if (li < l0) { E = k * pow(li - l0, n); fi = n * k * pow(li - l0, n - 1); } break;
      case 2: if (li > l0) { E = k * pow(li - l0, n); fi = n * k * pow(li - l0, n - 1); } break;
      case 3: E = k * pow(li - lj, n); fi = n * k * pow(li - lj, n - 1); fj = -fi; break;
      case 4: E = li > l0 ? -k : -k * (1 - (li - l0) * (li - l0) / (l0 * l0));
              fi = li > l0 ? 0 : 2 * k * (li - l0) / (l0 * l0); break;
      case 5: E = -k * li; fi = -k; break;
      case 7: E = k * li * (1 - li) / (li + l0); fi = k * (l0 * (1 + l0) / ((li + l0) * (li + l0)) - 1); break;
      case 9: E = k * lj * (1 - pow((li + l0) / l0, n)); fi = -k * lj * pow((li + l0) / l0, n - 1) / l0;
              fj = k * (1 - pow((li + l0) / l0, n)); break;
      case 11: E = k * pow(li, l0) * pow(lj, n); fi = k * l0 * pow(li, l0 - 1) * pow(lj, n);
               fj = k * n * pow(li, l0) * pow(lj, n - 1); break;
      case 12: E = k * li * pow(lj, n) / (li + l0); fi = k * l0 * pow(lj, n) / ((li + l0) * (li + l0));
               fj = k * n * li * pow(lj, n - 1) / (li + l0); break;
      default: break;
    }
    if (fi != 0.0) atomicAdd(&lambdaForce[v.i], (F)fi);
    if (fj != 0.0) atomicAdd(&lambdaForce[v.j], (F)fj);
    e += E;
  }
  if (energy) warp_energy(e, energy);
}

// Lambda histograms of one sampling step (the data ALF builds from the .lmd
// lambda trajectory that Msld writes every freqLMD steps, src/io/io.cxx:347-371):
// per block a 32-bin histogram of lambda on [0,1] and a count of lambda > 0.99
// (the block's end state); per listed block pair an 8x8 histogram of
// (lambda_i, lambda_j).  Fixed blocks are skipped.
__global__ void k_lambda_histogram(int blockCount, const double *lambda, const uint8_t *fixed, int pairCount,
                                   const int *pairs, unsigned int *hist1, unsigned int *hist2,
                                   unsigned int *endCount) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < blockCount && !(fixed && fixed[t])) {
    const double l = lambda[t];
    int b = (int)(l * 32.0);
    b = b < 0 ? 0 : (b > 31 ? 31 : b);
    if (hist1) atomicAdd(&hist1[32 * t + b], 1u);
    if (endCount && l > 0.99) atomicAdd(&endCount[t], 1u);
  }
  if (t < pairCount && hist2) {
    const double li = lambda[pairs[2 * t]], lj = lambda[pairs[2 * t + 1]];
    int a = (int)(li * 8.0), b = (int)(lj * 8.0);
    a = a < 0 ? 0 : (a > 7 ? 7 : a);
    b = b < 0 ? 0 : (b > 7 ? 7 : b);
    atomicAdd(&hist2[64 * t + 8 * a + b], 1u);
  }
}

inline int blocks_for(int n) { return n > 0 ? (n + 255) / 256 : 1; }

template <typename L, typename F>
int theta_force(int blockCount, const int *lambdaSite, const int *siteBound, double fnex, const L *lambda,
                const L *theta, const F *lambdaForce, const uint8_t *blockFixed, F *thetaForce, void *stream) {
  if (blockCount < 0 || (blockCount > 0 && (!lambdaSite || !siteBound || !lambda || !theta ||
                                            !lambdaForce || !thetaForce)))
    return BNB_ERR_ARG;
  if (blockCount == 0) return BNB_OK;
  k_theta_force<L, F><<<blocks_for(blockCount), 256, 0, (cudaStream_t)stream>>>(
      blockCount, lambdaSite, siteBound, fnex, lambda, theta, lambdaForce, blockFixed, thetaForce);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

template <typename L, typename F>
int bias(int blockCount, const L *lambda, const L *fixedBias, int varCount, const bnb_varbias *varBias,
         F *lambdaForce, double *energy, void *stream) {
  if (blockCount < 0 || varCount < 0 || !lambda || !lambdaForce || (varCount > 0 && !varBias))
    return BNB_ERR_ARG;
  int n = blockCount > varCount ? blockCount : varCount;
  if (n == 0) return BNB_OK;
  k_bias<L, F><<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(blockCount, lambda, fixedBias, varCount,
                                                                varBias, lambdaForce, energy);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

}  // namespace

extern "C" int bnb_lambda_from_theta(int siteCount, const int *siteBound, double fnex,
                                     const double *theta, const uint8_t *blockFixed, double *lambda,
                                     float *lambda_f, void *stream) {
  if (siteCount < 0 || (siteCount > 0 && (!siteBound || !theta || !lambda))) return BNB_ERR_ARG;
  if (siteCount == 0) return BNB_OK;
  k_lambda_from_theta<<<blocks_for(siteCount), 256, 0, (cudaStream_t)stream>>>(
      siteCount, siteBound, fnex, theta, blockFixed, lambda, lambda_f);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_theta_force(int blockCount, const int *lambdaSite, const int *siteBound, double fnex,
                               const double *lambda, const double *theta, const double *lambdaForce,
                               const uint8_t *blockFixed, double *thetaForce, void *stream) {
  return theta_force<double, double>(blockCount, lambdaSite, siteBound, fnex, lambda, theta, lambdaForce,
                                     blockFixed, thetaForce, stream);
}

extern "C" int bnb_theta_force_f32(int blockCount, const int *lambdaSite, const int *siteBound,
                                   double fnex, const float *lambda, const float *theta,
                                   const float *lambdaForce, const uint8_t *blockFixed, float *thetaForce,
                                   void *stream) {
  return theta_force<float, float>(blockCount, lambdaSite, siteBound, fnex, lambda, theta, lambdaForce,
                                   blockFixed, thetaForce, stream);
}

extern "C" int bnb_bias(int blockCount, const double *lambda, const double *fixedBias, int varCount,
                        const bnb_varbias *varBias, double *lambdaForce, double *energy, void *stream) {
  return bias<double, double>(blockCount, lambda, fixedBias, varCount, varBias, lambdaForce, energy, stream);
}

extern "C" int bnb_bias_f32(int blockCount, const float *lambda, const float *fixedBias, int varCount,
                            const bnb_varbias *varBias, float *lambdaForce, double *energy, void *stream) {
  return bias<float, float>(blockCount, lambda, fixedBias, varCount, varBias, lambdaForce, energy, stream);
}

extern "C" int bnb_lambda_histogram(int blockCount, const double *lambda, const uint8_t *blockFixed,
                                    int pairCount, const int *pairs, unsigned int *hist1, unsigned int *hist2,
                                    unsigned int *endCount, void *stream) {
  if (blockCount < 0 || pairCount < 0 || (blockCount > 0 && !lambda) || (pairCount > 0 && !pairs))
    return BNB_ERR_ARG;
  const int n = blockCount > pairCount ? blockCount : pairCount;
  if (n == 0) return BNB_OK;
  k_lambda_histogram<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(blockCount, lambda, blockFixed, pairCount,
                                                                      pairs, hist1, hist2, endCount);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}
