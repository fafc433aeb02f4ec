// Kernels of the learned Newton warm start: a small MLP over nodal features
// (BF16 weights and activations, FP32 accumulation and master weights).
//
//  * k_gemm_bf16: C[M x N] (FP32) = op(A)[M x K] * op(B)[K x N] (+ beta * C)
//    on the tensor cores with mma.sync m16n8k16 (BF16 in, FP32 accumulate).
//    Operands are addressed through (row, col) strides, so one kernel covers
//    the forward product H W^T, the weight gradient dZ^T H and the input
//    gradient dZ W without explicit transposes.  64x64 CTA tile, four warps
//    of 32x32, K step 32 staged in shared memory (zero-filled at the edges).
//  * k_bias_silu_fwd, k_silu_bwd, k_colsum, k_adam, k_cast: elementwise work
//    of the forward / backward pass and the optimiser.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "fne_internal.h"

namespace fne {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;

__device__ __forceinline__ unsigned pack_bf16x2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  const unsigned short l = *reinterpret_cast<unsigned short*>(&lo);
  const unsigned short h = *reinterpret_cast<unsigned short*>(&hi);
  return (unsigned)l | ((unsigned)h << 16);
}

__device__ __forceinline__ void mma_bf16_16816(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A(m, k) = A[m * sam + k * sak]; B(k, n) = B[k * sbk + n * sbn];
// C(m, n) = C[m * ldc + n] (FP32).
__global__ void __launch_bounds__(128) k_gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                   long long sam, long long sak, const __nv_bfloat16* __restrict__ B,
                                                   long long sbk, long long sbn, float* __restrict__ C, long long ldc,
                                                   float beta) {
  __shared__ __nv_bfloat16 As[kBM][kBK + kPad];  // [m][k]
  __shared__ __nv_bfloat16 Bs[kBN][kBK + kPad];  // [n][k]
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // warp tile origin
  const int grp = lane >> 2, tig = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += kBK) {
    // stage the tiles (any operand layout; out-of-range elements are zero)
    for (int idx = threadIdx.x; idx < kBM * kBK; idx += blockDim.x) {
      int r, c;
      if (sak == 1) {  // k contiguous: walk k fastest
        r = idx / kBK; c = idx - r * kBK;
      } else {         // m contiguous: walk m fastest
        c = idx / kBM; r = idx - c * kBM;
      }
      const int m = m0 + r, k = k0 + c;
      As[r][c] = (m < M && k < K) ? A[(long long)m * sam + (long long)k * sak] : zero;
    }
    for (int idx = threadIdx.x; idx < kBN * kBK; idx += blockDim.x) {
      int r, c;
      if (sbk == 1) {
        r = idx / kBK; c = idx - r * kBK;
      } else {
        c = idx / kBN; r = idx - c * kBN;
      }
      const int n = n0 + r, k = k0 + c;
      Bs[r][c] = (n < N && k < K) ? B[(long long)k * sbk + (long long)n * sbn] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      unsigned af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + 16 * i + grp;
        af[i][0] = pack_bf16x2(As[r][kk + 2 * tig], As[r][kk + 2 * tig + 1]);
        af[i][1] = pack_bf16x2(As[r + 8][kk + 2 * tig], As[r + 8][kk + 2 * tig + 1]);
        af[i][2] = pack_bf16x2(As[r][kk + 2 * tig + 8], As[r][kk + 2 * tig + 9]);
        af[i][3] = pack_bf16x2(As[r + 8][kk + 2 * tig + 8], As[r + 8][kk + 2 * tig + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = wn + 8 * j + grp;
        bfr[j][0] = pack_bf16x2(Bs[n][kk + 2 * tig], Bs[n][kk + 2 * tig + 1]);
        bfr[j][1] = pack_bf16x2(Bs[n][kk + 2 * tig + 8], Bs[n][kk + 2 * tig + 9]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16_16816(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm + 16 * i + grp + (r >= 2 ? 8 : 0);
        const int n = n0 + wn + 8 * j + 2 * tig + (r & 1);
        if (m < M && n < N) {
          float* cp = C + (long long)m * ldc + n;
          *cp = acc[i][j][r] + (beta != 0.f ? beta * *cp : 0.f);
        }
      }
}

// Z[n, m] += b[m]; H = silu(Z) (FP32 and BF16 copies); act = 0 leaves H = Z.
__global__ void k_bias_act_fwd(long long rows, int cols, float* __restrict__ Z, const float* __restrict__ b, int act,
                               float* __restrict__ H32, __nv_bfloat16* __restrict__ H16) {
  const long long n = rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float z = Z[i] + (b ? b[i % cols] : 0.f);
    Z[i] = z;
    const float h = act ? z / (1.f + expf(-z)) : z;
    if (H32) H32[i] = h;
    if (H16) H16[i] = __float2bfloat16(h);
  }
}

// dZ = dH * silu'(Z) (act = 1) or dH (act = 0); FP32 and BF16 copies.
__global__ void k_act_bwd(long long n, const float* __restrict__ Z, const float* __restrict__ dH, int act,
                          float* __restrict__ dZ32, __nv_bfloat16* __restrict__ dZ16) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float d = dH[i];
    if (act) {
      const float z = Z[i];
      const float s = 1.f / (1.f + expf(-z));
      d *= s * (1.f + z * (1.f - s));
    }
    if (dZ32) dZ32[i] = d;
    if (dZ16) dZ16[i] = __float2bfloat16(d);
  }
}

// out[m] = sum_n X[n, m] (bias gradient), one thread per column, fixed order.
__global__ void k_colsum(long long rows, int cols, const float* __restrict__ X, float* __restrict__ out) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= cols) return;
  double acc = 0.0;
  for (long long n = 0; n < rows; ++n) acc += X[n * cols + m];
  out[m] = (float)acc;
}

// Adam on FP32 master weights; refreshes the BF16 copy used by the GEMMs.
__global__ void k_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ p16) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (p16) p16[i] = __float2bfloat16(pi);
  }
}

__global__ void k_cast_bf16(long long n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>(148 * 16, (n + 255) / 256)); }

int launch_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FNE_OK;
}

}  // namespace
}  // namespace fne

using namespace fne;

extern "C" int fne_gemm_bf16(int M, int N, int K, const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbk,
                             int64_t sbn, float* C, int64_t ldc, float beta, void* stream) {
  if (M < 0 || N < 0 || K < 0 || (M * (int64_t)N > 0 && !C) || (M * (int64_t)K > 0 && !A) ||
      (K * (int64_t)N > 0 && !B))
    return set_error(FNE_EINVAL, "fne_gemm_bf16: bad arguments");
  if (M == 0 || N == 0) return FNE_OK;
  const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  if (grid.y > 65535) return set_error(FNE_EBOUNDS, "fne_gemm_bf16: M too large");
  k_gemm_bf16<<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, (const __nv_bfloat16*)A, sam, sak,
                                                        (const __nv_bfloat16*)B, sbk, sbn, C, ldc, beta);
  return launch_status("fne_gemm_bf16");
}

extern "C" int fne_mlp_bias_act(int64_t rows, int cols, float* Z, const float* bias, int act, float* H32, void* H16,
                                void* stream) {
  if (rows < 0 || cols <= 0 || !Z) return set_error(FNE_EINVAL, "fne_mlp_bias_act: bad arguments");
  const long long n = rows * (long long)cols;
  if (n == 0) return FNE_OK;
  k_bias_act_fwd<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(rows, cols, Z, bias, act, H32,
                                                                  (__nv_bfloat16*)H16);
  return launch_status("fne_mlp_bias_act");
}

extern "C" int fne_mlp_act_bwd(int64_t n, const float* Z, const float* dH, int act, float* dZ32, void* dZ16,
                               void* stream) {
  if (n < 0 || (n > 0 && (!dH || (act && !Z)))) return set_error(FNE_EINVAL, "fne_mlp_act_bwd: bad arguments");
  if (n == 0) return FNE_OK;
  k_act_bwd<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, Z, dH, act, dZ32, (__nv_bfloat16*)dZ16);
  return launch_status("fne_mlp_act_bwd");
}

extern "C" int fne_mlp_colsum(int64_t rows, int cols, const float* X, float* out, void* stream) {
  if (rows < 0 || cols <= 0 || !X || !out) return set_error(FNE_EINVAL, "fne_mlp_colsum: bad arguments");
  k_colsum<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(rows, cols, X, out);
  return launch_status("fne_mlp_colsum");
}

extern "C" int fne_mlp_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2,
                            float eps, int step, void* p16, void* stream) {
  if (n < 0 || step < 1 || (n > 0 && (!p || !g || !m || !v))) return set_error(FNE_EINVAL, "fne_mlp_adam: bad arguments");
  if (n == 0) return FNE_OK;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, p, g, m, v, lr, b1, b2, eps, c1, c2,
                                                          (__nv_bfloat16*)p16);
  return launch_status("fne_mlp_adam");
}

extern "C" int fne_mlp_cast_bf16(int64_t n, const float* x, void* y, void* stream) {
  if (n < 0 || (n > 0 && (!x || !y))) return set_error(FNE_EINVAL, "fne_mlp_cast_bf16: bad arguments");
  if (n == 0) return FNE_OK;
  k_cast_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(n, x, (__nv_bfloat16*)y);
  return launch_status("fne_mlp_cast_bf16");
}
