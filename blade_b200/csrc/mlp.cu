// BF16 multilayer perceptron kernels for learned landscape flattening (sm_100a).
//
// No reference counterpart: BLaDE's src/mlp is TorchANI inference through
// LibTorch, unrelated to lambda biases.  The network maps lambda histograms
// and the current bias parameters to corrections of those parameters; it is
// trained and run with these kernels only:
//   linear forward   Z = X W^T + b, Y = act(Z)  (X, W, Y in BF16; Z FP32)
//   linear backward  dZ = dY act'(Z); dX = dZ W; dW = dZ^T X; db = sum_m dZ
//   MSE loss         L = (1/M) sum_m sum_n w_n w_mn (Y - T)^2, dY = dL/dY
//   Adam             FP32 master weights, BF16 working copy
// Every product takes BF16 operands (round to nearest even) and accumulates
// in FP32 in a fixed order, so results are reproducible run to run.  act is
// 0 (identity) or 1 (SiLU, z * sigmoid(z)).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bnb.h"

namespace {

__device__ __forceinline__ float bf2f(uint16_t v) { return __uint_as_float((uint32_t)v << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) {
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  return *reinterpret_cast<uint16_t *>(&h);
}
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

// C[i,j] (+)= sum_l A(i,l) B(l,j) over BF16 operands given by strides:
// A(i,l) = A[i*sai + l*sal], B(l,j) = B[l*sbl + j*sbj]; C row-major [I,J].
// 64x64 output tile per 256-thread CTA, 4x4 per thread, K staged in 16s.
constexpr int kT = 64, kK = 16;

__global__ void __launch_bounds__(256) k_gemm_bf16(int I, int J, int Lk, const uint16_t *A, long long sai,
                                                   long long sal, const uint16_t *B, long long sbl,
                                                   long long sbj, float *C) {
  __shared__ float sA[kK][kT + 1];
  __shared__ float sB[kK][kT + 1];
  const int i0 = blockIdx.y * kT, j0 = blockIdx.x * kT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4] = {};
  for (int l0 = 0; l0 < Lk; l0 += kK) {
    for (int e = threadIdx.x; e < kK * kT; e += 256) {
      const int r = e % kT, l = e / kT;  // r: row of the tile, l: k index
      const int gi = i0 + r, gl = l0 + l, gj = j0 + r;
      sA[l][r] = (gi < I && gl < Lk) ? bf2f(A[gi * sai + gl * sal]) : 0.f;
      sB[l][r] = (gj < J && gl < Lk) ? bf2f(B[gl * sbl + gj * sbj]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < kK; l++) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        a[u] = sA[l][ty + 16 * u];
        b[u] = sB[l][tx + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int gi = i0 + ty + 16 * u, gj = j0 + tx + 16 * v;
      if (gi < I && gj < J) C[(size_t)gi * J + gj] = acc[u][v];
    }
}

// Z = C + bias (in place), Y = act(Z) in BF16 and optionally FP32.
__global__ void k_bias_act(int M, int N, float *Z, const float *bias, int act, uint16_t *Y, float *Yf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M * N) return;
  const float z = Z[t] + (bias ? bias[t % N] : 0.f);
  Z[t] = z;
  const float y = act ? z * sigmoid(z) : z;
  if (Y) Y[t] = f2bf(y);
  if (Yf) Yf[t] = y;
}

// dZ = dY act'(Z): FP32 copy (for db) and BF16 copy (for the products).
__global__ void k_act_grad(int M, int N, const float *dY, const float *Z, int act, float *dZ, uint16_t *dZb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M * N) return;
  float g = dY[t];
  if (act) {
    const float z = Z[t], s = sigmoid(z);
    g *= s * (1.f + z * (1.f - s));
  }
  dZ[t] = g;
  dZb[t] = f2bf(g);
}

// db[n] = sum_m dZ[m,n], rows added in order.
__global__ void k_colsum(int M, int N, const float *dZ, float *db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; m++) s += dZ[(size_t)m * N + n];
  db[n] = s;
}

// One CTA: loss and dY of the weighted mean squared error, summed in a fixed order.
__global__ void k_mse(int M, int N, const float *Y, const float *T, const float *w, const float *we, float *dY,
                      double *loss) {
  __shared__ double red[1024];
  double s = 0.0;
  const float inv = 1.f / (float)M;
  for (int t = threadIdx.x; t < M * N; t += blockDim.x) {
    const float wn = (w ? w[t % N] : 1.f) * (we ? we[t] : 1.f);
    const float d = Y[t] - T[t];
    dY[t] = 2.f * wn * d * inv;
    s += (double)wn * d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss) *loss = red[0] / M;
}

__global__ void k_adam(int n, float *master, uint16_t *wb, const float *g, float *m, float *v, float lr, float b1,
                       float b2, float eps, float wd, float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt;
  const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  float w = master[t];
  w -= lr * ((mt / c1) / (sqrtf(vt / c2) + eps) + wd * w);
  master[t] = w;
  if (wb) wb[t] = f2bf(w);
}

__global__ void k_to_bf16(int n, const float *x, uint16_t *y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] = f2bf(x[t]);
}

inline int grid1(long long n) { return (int)((n + 255) / 256); }

int gemm(int I, int J, int Lk, const uint16_t *A, long long sai, long long sal, const uint16_t *B, long long sbl,
         long long sbj, float *C, cudaStream_t s) {
  dim3 grid((J + kT - 1) / kT, (I + kT - 1) / kT);
  k_gemm_bf16<<<grid, 256, 0, s>>>(I, J, Lk, A, sai, sal, B, sbl, sbj, C);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

}  // namespace

extern "C" int bnb_mlp_linear_forward(int M, int N, int K, const uint16_t *X, const uint16_t *W, const float *bias,
                                      int act, float *Z, uint16_t *Y, float *Yf, void *stream) {
  if (M < 0 || N < 0 || K < 0 || !X || !W || !Z || (act != 0 && act != 1)) return BNB_ERR_ARG;
  if ((long long)M * N >= (1ll << 31)) return BNB_ERR_ARG;
  if (M == 0 || N == 0) return BNB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = gemm(M, N, K, X, K, 1, W, 1, K, Z, s);  // Z[m,n] = sum_k X[m,k] W[n,k]
  if (rc) return rc;
  k_bias_act<<<grid1((long long)M * N), 256, 0, s>>>(M, N, Z, bias, act, Y, Yf);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_mlp_linear_backward(int M, int N, int K, const float *dY, const float *Z, int act,
                                       const uint16_t *X, const uint16_t *W, float *dZ, uint16_t *dZb, float *dX,
                                       float *dW, float *db, void *stream) {
  if (M < 0 || N < 0 || K < 0 || !dY || !Z || !X || !W || !dZ || !dZb || !dW || !db || (act != 0 && act != 1))
    return BNB_ERR_ARG;
  if ((long long)M * N >= (1ll << 31) || (long long)M * K >= (1ll << 31)) return BNB_ERR_ARG;
  if (M == 0 || N == 0) return BNB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  k_act_grad<<<grid1((long long)M * N), 256, 0, s>>>(M, N, dY, Z, act, dZ, dZb);
  k_colsum<<<grid1(N), 256, 0, s>>>(M, N, dZ, db);
  int rc = gemm(N, K, M, dZb, 1, N, X, K, 1, dW, s);  // dW[n,k] = sum_m dZ[m,n] X[m,k]
  if (rc) return rc;
  if (dX) {
    rc = gemm(M, K, N, dZb, N, 1, W, K, 1, dX, s);  // dX[m,k] = sum_n dZ[m,n] W[n,k]
    if (rc) return rc;
  }
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_mlp_mse(int M, int N, const float *Y, const float *T, const float *weight,
                           const float *elemWeight, float *dY, double *loss, void *stream) {
  if (M <= 0 || N <= 0 || !Y || !T || !dY) return BNB_ERR_ARG;
  k_mse<<<1, 1024, 0, (cudaStream_t)stream>>>(M, N, Y, T, weight, elemWeight, dY, loss);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_mlp_adam(int n, float *master, uint16_t *weightBf16, const float *grad, float *m, float *v,
                            float lr, float beta1, float beta2, float eps, float weightDecay, int step,
                            void *stream) {
  if (n < 0 || step < 1 || (n > 0 && (!master || !grad || !m || !v))) return BNB_ERR_ARG;
  if (n == 0) return BNB_OK;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_adam<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(n, master, weightBf16, grad, m, v, lr, beta1, beta2, eps,
                                                     weightDecay, c1, c2);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}

extern "C" int bnb_to_bf16(int n, const float *x, uint16_t *y, void *stream) {
  if (n < 0 || (n > 0 && (!x || !y))) return BNB_ERR_ARG;
  if (n == 0) return BNB_OK;
  k_to_bf16<<<grid1(n), 256, 0, (cudaStream_t)stream>>>(n, x, y);
  return cudaGetLastError() == cudaSuccess ? BNB_OK : BNB_ERR_CUDA;
}
