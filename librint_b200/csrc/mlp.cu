// Small-MLP training and inference kernels for the learned initial guess
// (FP32 storage and arithmetic).  A layer is Y = act(X W^T + b) with X (M x K),
// W (N x K), b (N); act is identity or SiLU.  Backward gives dX, dW, db.
// Shapes here are small (K, N <= 512), so plain 32x32 shared-memory tiles are
// enough; the work is launch- and latency-bound, not FLOP-bound.
#include <cuda_runtime.h>

#include "engine.h"

namespace lrb {
namespace {

constexpr int TS = 32;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// C[m][n] = sum_k A[m][k] * B[n][k] (+ bias[n]); optional pre-activation copy
__global__ void k_gemm_nt(int M, int N, int K, const float *__restrict__ A,
                          const float *__restrict__ B, const float *__restrict__ bias, int act,
                          float *__restrict__ Z, float *__restrict__ Y) {
  __shared__ float sa[TS][TS + 1], sb[TS][TS + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8 threads, 4 rows each
  const int m0 = blockIdx.y * TS, n0 = blockIdx.x * TS;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += TS) {
    for (int r = ty; r < TS; r += 8) {
      const int m = m0 + r, k = k0 + tx, n = n0 + r;
      sa[r][tx] = (m < M && k < K) ? A[(long long)m * K + k] : 0.f;
      sb[r][tx] = (n < N && k < K) ? B[(long long)n * K + k] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TS; ++kk) {
      const float bv = sb[tx][kk];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(sa[ty + 8 * i][kk], bv, acc[i]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i, n = n0 + tx;
    if (m < M && n < N) {
      float z = acc[i] + (bias ? bias[n] : 0.f);
      if (Z) Z[(long long)m * N + n] = z;
      Y[(long long)m * N + n] = act == 1 ? silu(z) : z;
    }
  }
}

// C[m][n] = sum_k A[m][k] * B[k][n]   (dX = dZ W)
__global__ void k_gemm_nn(int M, int N, int K, const float *__restrict__ A,
                          const float *__restrict__ B, float *__restrict__ C) {
  __shared__ float sa[TS][TS + 1], sb[TS][TS + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m0 = blockIdx.y * TS, n0 = blockIdx.x * TS;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += TS) {
    for (int r = ty; r < TS; r += 8) {
      const int m = m0 + r, k = k0 + tx;
      sa[r][tx] = (m < M && k < K) ? A[(long long)m * K + k] : 0.f;
      const int kb = k0 + r, n = n0 + tx;
      sb[r][tx] = (kb < K && n < N) ? B[(long long)kb * N + n] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TS; ++kk) {
      const float bv = sb[kk][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(sa[ty + 8 * i][kk], bv, acc[i]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i, n = n0 + tx;
    if (m < M && n < N) C[(long long)m * N + n] = acc[i];
  }
}

// C[n][k] = sum_m A[m][n] * B[m][k]   (dW = dZ^T X), accumulated over m
__global__ void k_gemm_tn(int M, int N, int K, const float *__restrict__ A,
                          const float *__restrict__ B, float *__restrict__ C) {
  __shared__ float sa[TS][TS + 1], sb[TS][TS + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int n0 = blockIdx.y * TS, k0 = blockIdx.x * TS;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int m0 = 0; m0 < M; m0 += TS) {
    for (int r = ty; r < TS; r += 8) {
      const int m = m0 + r;
      sa[r][tx] = (m < M && n0 + tx < N) ? A[(long long)m * N + n0 + tx] : 0.f;
      sb[r][tx] = (m < M && k0 + tx < K) ? B[(long long)m * K + k0 + tx] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int mm = 0; mm < TS; ++mm) {
      const float bv = sb[mm][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(sa[mm][ty + 8 * i], bv, acc[i]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int n = n0 + ty + 8 * i, k = k0 + tx;
    if (n < N && k < K) C[(long long)n * K + k] = acc[i];
  }
}

// dZ = dY * act'(Z) and column sums db (db zeroed by the caller).  Block
// 32 x 8 covers 32 columns and ACT_ROWS rows; partial sums meet in shared
// memory, then one atomic per column.
constexpr int ACT_ROWS = 256;
__global__ void k_act_back(int M, int N, int act, const float *__restrict__ Z,
                           const float *__restrict__ dY, float *__restrict__ dZ,
                           float *__restrict__ db) {
  __shared__ float red[8][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int n = blockIdx.x * 32 + tx;
  const int m0 = blockIdx.y * ACT_ROWS;
  float s = 0.f;
  if (n < N) {
    const int m1 = min(M, m0 + ACT_ROWS);
    for (int m = m0 + ty; m < m1; m += 8) {
      const long long t = (long long)m * N + n;
      const float g = act == 1 ? dY[t] * dsilu(Z[t]) : dY[t];
      dZ[t] = g;
      s += g;
    }
  }
  red[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && n < N) {
    float t = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) t += red[i][tx];
    atomicAdd(&db[n], t);
  }
}

// loss += sum w (y - t)^2 / count ; dY = 2 w (y - t) / count
__global__ void k_mse(long long n, const float *__restrict__ Y, const float *__restrict__ T,
                      const float *__restrict__ W, float inv_count, float *__restrict__ dY,
                      float *__restrict__ loss) {
  __shared__ float sm[256];
  float s = 0.f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const float w = W ? W[t] : 1.f;
    const float d = Y[t] - T[t];
    dY[t] = 2.f * w * d * inv_count;
    s += w * d * d * inv_count;
  }
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, sm[0]);
}

__global__ void k_adam(long long n, float *__restrict__ p, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gi = g[t];
  const float mi = b1 * m[t] + (1.f - b1) * gi;
  const float vi = b2 * v[t] + (1.f - b2) * gi * gi;
  m[t] = mi;
  v[t] = vi;
  p[t] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

}  // namespace
}  // namespace lrb

using namespace lrb;

extern "C" {

// Y = act(X W^T + b); Z (pre-activation) may be NULL.  act: 0 identity, 1 SiLU.
LRB_API int lrb_mlp_forward(const float *X, int M, int K, const float *W, const float *b, int N,
                            int act, float *Z, float *Y, void *stream) {
  if (M <= 0 || N <= 0 || K <= 0) return LRB_OK;
  const dim3 blk(32, 8), grd((N + TS - 1) / TS, (M + TS - 1) / TS);
  k_gemm_nt<<<grd, blk, 0, (cudaStream_t)stream>>>(M, N, K, X, W, b, act, Z, Y);
  engine().launches++;
  return cudaGetLastError() == cudaSuccess ? LRB_OK : LRB_ERR_CUDA;
}

// From dY (M x N), Z, X, W: dZ (scratch M x N), dW (N x K), db (N), dX (M x K,
// may be NULL for the first layer).
LRB_API int lrb_mlp_backward(const float *X, int M, int K, const float *W, int N, int act,
                             const float *Z, const float *dY, float *dZ, float *dW, float *db,
                             float *dX, void *stream) {
  if (M <= 0 || N <= 0 || K <= 0) return LRB_ERR_INPUT;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 blk(32, 8);
  if (cudaMemsetAsync(db, 0, sizeof(float) * N, st) != cudaSuccess) return LRB_ERR_CUDA;
  k_act_back<<<dim3((N + 31) / 32, (M + ACT_ROWS - 1) / ACT_ROWS), blk, 0, st>>>(M, N, act, Z, dY,
                                                                               dZ, db);
  k_gemm_tn<<<dim3((K + TS - 1) / TS, (N + TS - 1) / TS), blk, 0, st>>>(M, N, K, dZ, X, dW);
  engine().launches += 2;
  if (dX) {
    k_gemm_nn<<<dim3((K + TS - 1) / TS, (M + TS - 1) / TS), blk, 0, st>>>(M, K, N, dZ, W, dX);
    engine().launches++;
  }
  return cudaGetLastError() == cudaSuccess ? LRB_OK : LRB_ERR_CUDA;
}

// Weighted mean-squared error: loss (device scalar, accumulated) and dY.
LRB_API int lrb_mse(const float *Y, const float *T, const float *Wt, long long n, float inv_count,
                    float *dY, float *loss, void *stream) {
  if (n <= 0) return LRB_ERR_INPUT;
  k_mse<<<256, 256, 0, (cudaStream_t)stream>>>(n, Y, T, Wt, inv_count, dY, loss);
  engine().launches++;
  return cudaGetLastError() == cudaSuccess ? LRB_OK : LRB_ERR_CUDA;
}

LRB_API int lrb_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float b1,
                     float b2, float eps, int step, void *stream) {
  if (n <= 0 || step <= 0) return LRB_ERR_INPUT;
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  k_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2,
                                                                        eps, c1, c2);
  engine().launches++;
  return cudaGetLastError() == cudaSuccess ? LRB_OK : LRB_ERR_CUDA;
}

}  // extern "C"
