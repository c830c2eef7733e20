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
// in FP32 in a fixed order on the tensor pipe (mma.sync m16n8k16), so results
// are reproducible run to run.  act is
// 0 (identity) or 1 (SiLU, z * sigmoid(z)).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bnb.h"

namespace {

__device__ __forceinline__ uint16_t f2bf(float f) {
  __nv_bfloat16 h = __float2bfloat16_rn(f);
  return *reinterpret_cast<uint16_t *>(&h);
}
__device__ __forceinline__ float sigmoid(float z) { return 1.f / (1.f + expf(-z)); }

// C[i,j] = sum_l A(i,l) B(l,j) over BF16 operands given by strides:
// A(i,l) = A[i*sai + l*sal], B(l,j) = B[l*sbl + j*sbj]; C row-major [I,J].
// On the tensor pipe: a 64x64 output tile per 256-thread CTA, K staged in
// 64s through shared memory (A as [row][k], B as [column][k]), each of the
// 8 warps (2 x 4) computing 32x16 of the tile as 2 x 2 mma.m16n8k16 with
// BF16 operands and FP32 accumulators, k steps of 16 in increasing order.
constexpr int kT = 64, kK = 64, kPad = 8;

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(256) k_gemm_bf16(int I, int J, int Lk, const uint16_t *A, long long sai,
                                                   long long sal, const uint16_t *B, long long sbl,
                                                   long long sbj, float *C) {
  __shared__ __align__(16) uint16_t sA[kT][kK + kPad];  // [tile row][k]
  __shared__ __align__(16) uint16_t sB[kT][kK + kPad];  // [tile column][k]
  const int i0 = blockIdx.y * kT, j0 = blockIdx.x * kT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp >> 2, wn = warp & 3;  // warp tile: rows wm*32.., columns wn*16..
  const int g = lane >> 2, t = lane & 3;    // mma fragment coordinates
  float acc[2][2][4] = {};
  for (int l0 = 0; l0 < Lk; l0 += kK) {
    for (int e = threadIdx.x; e < kK * kT; e += 256) {
      const int r = e / kK, l = e % kK;  // r: tile row (A) or column (B), l: k index
      const int gi = i0 + r, gj = j0 + r, gl = l0 + l;
      sA[r][l] = (gi < I && gl < Lk) ? A[gi * sai + gl * sal] : (uint16_t)0;
      sB[r][l] = (gj < J && gl < Lk) ? B[gl * sbl + gj * sbj] : (uint16_t)0;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kK; ks += 16) {
      uint32_t af[2][4], bfr[2][2];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const int rb = wm * 32 + mt * 16;
        af[mt][0] = *reinterpret_cast<const uint32_t *>(&sA[rb + g][ks + 2 * t]);
        af[mt][1] = *reinterpret_cast<const uint32_t *>(&sA[rb + g + 8][ks + 2 * t]);
        af[mt][2] = *reinterpret_cast<const uint32_t *>(&sA[rb + g][ks + 2 * t + 8]);
        af[mt][3] = *reinterpret_cast<const uint32_t *>(&sA[rb + g + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 2; nt++) {
        const int cb = wn * 16 + nt * 8;
        bfr[nt][0] = *reinterpret_cast<const uint32_t *>(&sB[cb + g][ks + 2 * t]);
        bfr[nt][1] = *reinterpret_cast<const uint32_t *>(&sB[cb + g][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++) mma_bf16_16816(acc[mt][nt], af[mt], bfr[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int nt = 0; nt < 2; nt++) {
      const int row = i0 + wm * 32 + mt * 16 + g, col = j0 + wn * 16 + nt * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; h++) {  // h = 0: row g, h = 1: row g + 8
        const int r = row + 8 * h;
        if (r < I && col < J) C[(size_t)r * J + col] = acc[mt][nt][2 * h];
        if (r < I && col + 1 < J) C[(size_t)r * J + col + 1] = acc[mt][nt][2 * h + 1];
      }
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

// db[n] = sum_m dZ[m,n]: 32 columns per 256-thread CTA, 8 row slices per
// column (slice r sums rows r, r+8, ... in order), the slices then added in a
// fixed tree order -- parallel and reproducible.
__global__ void __launch_bounds__(256) k_colsum(int M, int N, const float *dZ, float *db) {
  __shared__ float part[8][33];
  const int c = threadIdx.x & 31, r = threadIdx.x >> 5;
  const int n = blockIdx.x * 32 + c;
  float s = 0.f;
  if (n < N)
    for (int m = r; m < M; m += 8) s += dZ[(size_t)m * N + n];
  part[r][c] = s;
  __syncthreads();
  if (r == 0 && n < N)
    db[n] = ((part[0][c] + part[1][c]) + (part[2][c] + part[3][c])) +
            ((part[4][c] + part[5][c]) + (part[6][c] + part[7][c]));
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
  k_colsum<<<(N + 31) / 32, 256, 0, s>>>(M, N, dZ, db);
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
