// Kernels of the learned Newton warm start: a small MLP over nodal features
// (BF16 weights and activations, FP32 accumulation and master weights).
//
//  * k_gemm_tc: C[M x N] (FP32) = op(A)[M x K] * op(B)[K x N] (+ beta * C) on
//    the 5th-generation tensor cores: tcgen05.mma kind::f16 with BF16
//    operands and an FP32 accumulator in tensor memory (TMEM).  One CTA per
//    128 x BN tile of C (BN = 32 or 128); the 128 threads stage each 64-deep K
//    slice of A and B into shared memory in the no-swizzle K-major
//    core-matrix layout (8 rows x 16 bytes; zero-filled at the edges; eight
//    values per load where an operand's K direction is contiguous), one
//    thread issues the four K = 16 MMAs of the slice and commits them to an
//    mbarrier (bounded wait), and the epilogue reads the accumulator back
//    with tcgen05.ld (each warp its 32-lane quadrant).  Operands are
//    addressed through (row, col) strides, so one kernel covers the forward
//    product H W^T, the weight gradient dZ^T H and the input gradient dZ W
//    without explicit transposes.
//  * k_bias_silu_fwd, k_silu_bwd, k_colsum, k_adam, k_cast: elementwise work
//    of the forward / backward pass and the optimiser.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "fne_internal.h"

namespace fne {
namespace {

constexpr int kTcBM = 128, kTcBK = 64;  // C rows per CTA, K depth per staged slice
constexpr long long kTcWaitLimit = 1LL << 22;

// status of the tensor-core GEMM: 1 once an MMA-completion wait gave up
__device__ int g_gemm_err = 0;

namespace tcg {

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// shared-memory matrix descriptor, no swizzle, K-major core matrices:
// lbo = bytes between the two 16-byte K halves of one K = 16 step,
// sbo = bytes between consecutive groups of 8 rows
__device__ __forceinline__ uint64_t mat_desc(uint32_t a, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((a >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;
}
// instruction descriptor: D f32, A / B bf16, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit) {
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace tcg

// A(m, k) = A[m * sam + k * sak]; B(k, n) = B[k * sbk + n * sbn];
// C(m, n) = C[m * ldc + n] (FP32).
template <int BN>
__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                 long long sam, long long sak, const __nv_bfloat16* __restrict__ B,
                                                 long long sbk, long long sbn, float* __restrict__ C, long long ldc,
                                                 float beta, long long wait_limit) {
  // core-matrix layout: element (row r, k) of a slice at [k / 8][r][k % 8]
  __shared__ __align__(128) __nv_bfloat16 sA[kTcBK / 8][kTcBM][8];
  __shared__ __align__(128) __nv_bfloat16 sB[kTcBK / 8][BN][8];
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTcBM, n0 = blockIdx.x * BN;
  constexpr int TCOLS = BN < 32 ? 32 : BN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tcg::saddr(&s_tmem)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    tcg::mbar_init(tcg::saddr(&s_bar));
    s_fail = 0;
  }
  tcg::fence_before();
  __syncthreads();
  tcg::fence_after();
  const uint32_t tmem = s_tmem, bar = tcg::saddr(&s_bar);
  constexpr uint32_t idesc = tcg::idesc_bf16(kTcBM, BN);
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  uint32_t phase = 0;
  // operands whose K direction is contiguous and 16-byte aligned are staged
  // eight values (one core-matrix row of 16 bytes) per load
  const bool a_vec = sak == 1 && (K & 7) == 0 && (sam & 7) == 0 && ((uintptr_t)A & 15) == 0;
  const bool b_vec = sbk == 1 && (K & 7) == 0 && (sbn & 7) == 0 && ((uintptr_t)B & 15) == 0;
  for (int k0 = 0; k0 < K; k0 += kTcBK) {
    // stage the slices (walking the operand's contiguous direction fastest)
    if (a_vec) {
      for (int idx = tid; idx < kTcBM * (kTcBK / 8); idx += 128) {
        const int r = idx / (kTcBK / 8), c8 = idx - r * (kTcBK / 8);
        const int m = m0 + r, k = k0 + 8 * c8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (m < M && k < K) v = __ldg(reinterpret_cast<const uint4*>(A + (long long)m * sam + k));
        *reinterpret_cast<uint4*>(&sA[c8][r][0]) = v;
      }
    } else
    for (int idx = tid; idx < kTcBM * kTcBK; idx += 128) {
      int r, c;
      if (sak == 1) {
        r = idx / kTcBK; c = idx - r * kTcBK;
      } else {
        c = idx / kTcBM; r = idx - c * kTcBM;
      }
      const int m = m0 + r, k = k0 + c;
      sA[c >> 3][r][c & 7] = (m < M && k < K) ? A[(long long)m * sam + (long long)k * sak] : zero;
    }
    if (b_vec) {
      for (int idx = tid; idx < BN * (kTcBK / 8); idx += 128) {
        const int r = idx / (kTcBK / 8), c8 = idx - r * (kTcBK / 8);
        const int n = n0 + r, k = k0 + 8 * c8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (n < N && k < K) v = __ldg(reinterpret_cast<const uint4*>(B + (long long)n * sbn + k));
        *reinterpret_cast<uint4*>(&sB[c8][r][0]) = v;
      }
    } else
    for (int idx = tid; idx < BN * kTcBK; idx += 128) {
      int r, c;
      if (sbk == 1) {
        r = idx / kTcBK; c = idx - r * kTcBK;
      } else {
        c = idx / BN; r = idx - c * BN;
      }
      const int n = n0 + r, k = k0 + c;
      sB[c >> 3][r][c & 7] = (n < N && k < K) ? B[(long long)k * sbk + (long long)n * sbn] : zero;
    }
    tcg::fence_proxy_async();  // the generic-proxy stores, visible to the tensor core
    __syncthreads();
    if (tid == 0) {
      tcg::fence_after();
#pragma unroll
      for (int kk = 0; kk < kTcBK / 16; ++kk) {
        const uint64_t ad = tcg::mat_desc(tcg::saddr(&sA[2 * kk][0][0]), kTcBM * 16, 128);
        const uint64_t bd = tcg::mat_desc(tcg::saddr(&sB[2 * kk][0][0]), BN * 16, 128);
        tcg::mma(tmem, ad, bd, idesc, (k0 > 0 || kk > 0) ? 1u : 0u);
      }
      tcg::commit(bar);
      if (!tcg::mbar_wait(bar, phase, wait_limit)) s_fail = 1;
    }
    phase ^= 1u;
    __syncthreads();  // the slices stay until their MMAs completed
    if (s_fail) break;
  }
  if (s_fail) {
    if (tid == 0) {
      tcg::mbar_wait(bar, phase ^ 1u, kTcWaitLimit);  // no MMA in flight when TMEM is released
      atomicExch(&g_gemm_err, 1);
    }
  } else if (K > 0) {
    tcg::fence_after();
    const int m = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 8) {
      uint32_t r[8];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                   : "r"(ta)
                   : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < M)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = n0 + c0 + j;
          if (n < N) {
            float* cp = C + (long long)m * ldc + n;
            *cp = __uint_as_float(r[j]) + (beta != 0.f ? beta * *cp : 0.f);
          }
        }
    }
  } else {  // K = 0: C = beta C
    for (int idx = tid; idx < kTcBM * BN; idx += 128) {
      const int m = m0 + idx / BN, n = n0 + idx % BN;
      if (m < M && n < N) C[(long long)m * ldc + n] *= beta;
    }
  }
  tcg::fence_before();
  __syncthreads();
  tcg::fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
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

namespace {
long long g_gemm_wait_limit = kTcWaitLimit;  // polls of the GEMM's MMA-completion waits
}  // namespace

extern "C" int fne_gemm_set_wait_limit(int64_t polls) {
  g_gemm_wait_limit = polls < 0 ? kTcWaitLimit : (long long)polls;
  return FNE_OK;
}

extern "C" int fne_gemm_check_status(void) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_gemm_err, sizeof(int));
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_gemm_check_status: ") + cudaGetErrorString(e));
  if (v == 0) return FNE_OK;
  const int zero = 0;
  cudaMemcpyToSymbol(g_gemm_err, &zero, sizeof(int));
  return set_error(FNE_ETIMEOUT, "fne_gemm_bf16: an MMA-completion wait gave up");
}

extern "C" int fne_gemm_bf16(int M, int N, int K, const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbk,
                             int64_t sbn, float* C, int64_t ldc, float beta, void* stream) {
  if (M < 0 || N < 0 || K < 0 || (M * (int64_t)N > 0 && !C) || (M * (int64_t)K > 0 && !A) ||
      (K * (int64_t)N > 0 && !B))
    return set_error(FNE_EINVAL, "fne_gemm_bf16: bad arguments");
  if (M == 0 || N == 0) return FNE_OK;
  const int bn = N <= 32 ? 32 : 128;
  const dim3 grid((N + bn - 1) / bn, (M + kTcBM - 1) / kTcBM);
  if (grid.y > 65535) return set_error(FNE_EBOUNDS, "fne_gemm_bf16: M too large");
  const long long lim = g_gemm_wait_limit;
  if (bn == 32)
    k_gemm_tc<32><<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, (const __nv_bfloat16*)A, sam, sak,
                                                          (const __nv_bfloat16*)B, sbk, sbn, C, ldc, beta, lim);
  else
    k_gemm_tc<128><<<grid, 128, 0, (cudaStream_t)stream>>>(M, N, K, (const __nv_bfloat16*)A, sam, sak,
                                                           (const __nv_bfloat16*)B, sbk, sbn, C, ldc, beta, lim);
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
