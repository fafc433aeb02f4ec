// 3-D Mohr-Coulomb slope family (P1 / P2 tetrahedra, 3 DOFs per node):
// element energy, gradient and constitutive Hessian on the GPU, scattered
// into the owned gradient and COO values.
//
// Replaces the element kernels of SlopeStability3DReorderedElementAssembler
// (src/problems/slope_stability_3d/jax_petsc/reordered_element_assembler.py:
// 189-206, 377-560): the density of src/problems/slope_stability_3d/jax/
// jax_energy_3d.py:38-191, its stress, and the element Hessian
// K_e = sum_q w_q B_q^T D_q B_q of constitutive_element_hessian_3d
// (jax_energy_3d.py:262-357), where the reference differentiates through
// eigvalsh with JAX and here the hand-written spectral derivatives of
// fne_mc3d_point.cuh are used.  Inputs are the reference's per-element,
// per-quadrature-point arrays: dphix / dphiy / dphiz (E, nq, n_p),
// quad_weight and the material fields c_bar_q, sin_phi_q, shear_q, bulk_q,
// lame_q (E, nq).
//
// k_mc3d_elem: a CTA of 128 threads takes a tile of 128 / nq elements.  One
// thread per (element, quadrature point) forms the strain and runs the
// constitutive point function (FP64: eigen-decomposition by cyclic
// Jacobi, branch potentials, spectral tangent) and stores w sigma and the
// upper triangle of w D in shared memory.  Then one warp per element: lanes
// over (node, component) form the element gradient; per quadrature point,
// lanes over nodes form (w D) B(b) from the three nonzeros of each column of
// B and lanes over node pairs a <= b add B(a)^T (w D) B(b) to their 3 x 3
// blocks.  Blocks and gradients go to per-element buffers that the
// node-block gather (fne_gather.cuh: per output block, contributions in
// element order, no atomics) sums into the COO values and the gradient.  FP32 mode keeps the point function in FP64 and runs the
// contraction, the buffers and the Hessian output in FP32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "fne_gather.cuh"
#include "fne_internal.h"
#include "fne_mc3d_point.cuh"

namespace fne {

namespace {

constexpr int kM3Warps = 4;      // warps per CTA
constexpr int kM3MaxQ = 16;      // quadrature points per element (kernel limit)
constexpr int kM3Pt = 6;         // per-point inputs: w, c_bar, sin_phi, shear, bulk, lame

struct Mc3dArgs {
  int n_el;                        // local elements
  int nq;
  const int* __restrict__ codes;   // [n_el][3 NP] gather codes
  const double* __restrict__ grad; // [n_el][3][nq][NP] physical basis gradients
  const double* __restrict__ pt;   // [n_el][nq][6] per-point inputs
  const unsigned char* __restrict__ wflag;
  const double* __restrict__ u;
  const double* __restrict__ dir;
  const double* __restrict__ rhs;  // [n_owned] or null
  int n_owned;
  long long lo;
  double tiny;
  int elastic;
  double* partials;
  unsigned* counter;
  double* energy;
};

__device__ __forceinline__ double m3_block_sum(double v, double* ws) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// per-CTA partial, then the last CTA to finish sums the partials in index
// order (deterministic, no spin-waits)
__device__ void m3_energy_finalize(double v, const Mc3dArgs& A) {
  __shared__ double ws[32];
  __shared__ int is_last;
  v = m3_block_sum(v, ws);
  if (threadIdx.x == 0) {
    A.partials[blockIdx.x] = v;
    __threadfence();
    is_last = atomicAdd(A.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s = 0.0;
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) s += __ldcg(A.partials + j);
  s = m3_block_sum(s, ws);
  if (threadIdx.x == 0) {
    A.energy[0] = s;
    *A.counter = 0u;
  }
}

// linear elastic point: psi = lame/2 I1^2 + mu Q (the reference's elastic mode)
__device__ __forceinline__ void m3_elastic(const double e[6], double mu, double lame, double& psi, double sig[6],
                                           double D[6][6]) {
  const double I1 = e[0] + e[1] + e[2];
  psi = 0.5 * lame * I1 * I1 + mu * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] +
                                     0.5 * (e[3] * e[3] + e[4] * e[4] + e[5] * e[5]));
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) D[i][j] = 0.0;
  for (int i = 0; i < 3; ++i) {
    sig[i] = lame * I1 + 2.0 * mu * e[i];
    sig[3 + i] = mu * e[3 + i];
    for (int j = 0; j < 3; ++j) D[i][j] = lame + (i == j ? 2.0 * mu : 0.0);
    D[3 + i][3 + i] = mu;
  }
}

// strain-vector component of DOF (node a, component c): the gradient entry
// on each of the six strain rows (xx, yy, zz, xy, yz, xz)
template <typename Real>
__device__ __forceinline__ void m3_bcol(Real gx, Real gy, Real gz, int c, Real b[6]) {
  b[0] = c == 0 ? gx : Real(0);
  b[1] = c == 1 ? gy : Real(0);
  b[2] = c == 2 ? gz : Real(0);
  b[3] = c == 0 ? gy : (c == 1 ? gx : Real(0));
  b[4] = c == 1 ? gz : (c == 2 ? gy : Real(0));
  b[5] = c == 0 ? gz : (c == 2 ? gx : Real(0));
}

// One quadrature point (FP64): strain from the nodal values, the point
// function, w sigma and the upper triangle of w D to shared memory; returns
// w psi.  Not inlined, so every instantiation of the element kernel runs the
// same machine code here and the separate energy / gradient / Hessian passes
// reproduce the fused pass bit for bit.
template <typename Real, int NP>
__device__ __noinline__ double m3_point_update(const double* __restrict__ grad, const int* __restrict__ codes,
                                               const double* __restrict__ u, const double* __restrict__ dir,
                                               const double* __restrict__ pt, int el, int q, int nq, double tiny,
                                               int elastic, Real* sig_out, Real* D_out) {
  const double* gq = grad + (long long)el * 3 * nq * NP + q * NP;
  const int* cd = codes + (long long)el * 3 * NP;
  double e[6] = {0, 0, 0, 0, 0, 0};
  for (int a = 0; a < NP; ++a) {
    double uc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int code = __ldg(cd + 3 * a + c);
      uc[c] = code >= 0 ? __ldg(u + code) : __ldg(dir + (-1 - code));
    }
    const double gx = __ldg(gq + a), gy = __ldg(gq + nq * NP + a), gz = __ldg(gq + 2 * nq * NP + a);
    e[0] += gx * uc[0];
    e[1] += gy * uc[1];
    e[2] += gz * uc[2];
    e[3] += gy * uc[0] + gx * uc[1];
    e[4] += gz * uc[1] + gy * uc[2];
    e[5] += gz * uc[0] + gx * uc[2];
  }
  const double* m = pt + ((long long)el * nq + q) * kM3Pt;
  const double w = __ldg(m);
  double psi, sig[6], D[6][6];
  if (elastic)
    m3_elastic(e, __ldg(m + 3), __ldg(m + 5), psi, sig, D);
  else
    mc3d::point(e, __ldg(m + 1), __ldg(m + 2), __ldg(m + 3), __ldg(m + 4), __ldg(m + 5), tiny, psi, sig, D);
#pragma unroll
  for (int i = 0; i < 6; ++i) sig_out[i] = (Real)(w * sig[i]);
  int t = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) D_out[t++] = (Real)(w * D[i][j]);
  return w * psi;
}

template <typename Real, int NP, int WANT>
__global__ void __launch_bounds__(32 * kM3Warps, 3) k_mc3d_elem(Mc3dArgs A, Real* __restrict__ kbuf,
                                                             Real* __restrict__ gbuf) {
  constexpr int N = 3 * NP, NPAIR = NP * (NP + 1) / 2, NT = 32 * kM3Warps;
  __shared__ Real s_sig[NT][6];                      // w sigma per point of the tile
  __shared__ Real s_D[NT][21];                       // w D, upper triangle row-major
  __shared__ Real s_g[kM3Warps][3][kM3MaxQ * NP];    // gx, gy, gz of the warp's element
  __shared__ Real s_T[kM3Warps][NP][18];             // (w D) B(b) of one point, per node
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nq = A.nq, epc = NT / nq;                // elements per tile: all their points in one pass
  double eacc = 0.0;
  for (int el0 = blockIdx.x * epc; el0 < A.n_el; el0 += gridDim.x * epc) {
    const int ne = min(epc, A.n_el - el0);
    // constitutive update, one thread per (element, quadrature point) of the
    // tile (FP64): strain from the nodal values, then the point function
    if ((int)threadIdx.x < ne * nq) {
      const int j = threadIdx.x / nq, q = threadIdx.x - j * nq, el = el0 + j;
      const double wpsi = m3_point_update<Real, NP>(A.grad, A.codes, A.u, A.dir, A.pt, el, q, nq, A.tiny,
                                                    A.elastic, s_sig[threadIdx.x], s_D[threadIdx.x]);
      if ((WANT & 1) && __ldg(A.wflag + el)) eacc += wpsi;
    }
    __syncthreads();
    // contraction: one warp per element of the tile
    for (int j = warp; (WANT & 6) && j < ne; j += kM3Warps) {
      const int el = el0 + j;
      const Real(*sg)[6] = s_sig + j * nq;
      const Real(*sD)[21] = s_D + j * nq;
      const double* gsrc = A.grad + (long long)el * 3 * nq * NP;
      for (int i = lane; i < 3 * nq * NP; i += 32) {
        const int k = i / (nq * NP), r = i - k * nq * NP;
        s_g[warp][k][r] = (Real)__ldg(gsrc + i);
      }
      __syncwarp();
      // element gradient: lanes over (node, component)
      if (WANT & 2) {
        for (int i = lane; i < N; i += 32) {
          const int a = i / 3, c = i - 3 * a;
          Real s = Real(0);
          for (int q = 0; q < nq; ++q) {
            Real b[6];
            m3_bcol<Real>(s_g[warp][0][q * NP + a], s_g[warp][1][q * NP + a], s_g[warp][2][q * NP + a], c, b);
#pragma unroll
            for (int k = 0; k < 6; ++k) s += b[k] * sg[q][k];
          }
          gbuf[(long long)el * N + i] = s;
        }
      }
      // Hessian blocks B(a)^T (w D) B(b) over the node pairs a <= b.  Each
      // column of B has three nonzeros (DOF (b, d) feeds three strain rows), so
      // per quadrature point the lanes first form T_b = (w D) B(b) (6 x 3, 18
      // products of three terms) and the lanes over pairs then add B(a)^T T_b
      // (9 sums of three terms)
      if (WANT & 4) {
        constexpr int PPL = (NPAIR + 31) / 32;  // pairs per lane
        Real K[PPL][3][3];
        int pa[PPL], pb[PPL];
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
          int a = 0, rem = lane + 32 * k;
          while (a < NP && rem >= NP - a) {
            rem -= NP - a;
            ++a;
          }
          pa[k] = a;
          pb[k] = a + rem;
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) K[k][c][d] = Real(0);
        }
        // (w D) B(b): lanes over (node b, strain row i), each forming row i
        // of T_b from row i of w D (upper-triangle positions precomputed)
        constexpr int NTI = NP * 6, TPL = (NTI + 31) / 32;
        int tb[TPL], ti[TPL], didx[TPL][6];
#pragma unroll
        for (int k = 0; k < TPL; ++k) {
          const int it = min(lane + 32 * k, NTI - 1);
          tb[k] = it / 6;
          ti[k] = it - 6 * tb[k];
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            const int lo = min(ti[k], j), hi = max(ti[k], j);
            didx[k][j] = lo * 6 - lo * (lo - 1) / 2 + (hi - lo);
          }
        }
        for (int q = 0; q < nq; ++q) {
#pragma unroll
          for (int k = 0; k < TPL; ++k) {
            if (lane + 32 * k >= NTI) continue;
            const Real* Dq = sD[q];
            const Real d0 = Dq[didx[k][0]], d1 = Dq[didx[k][1]], d2 = Dq[didx[k][2]], d3 = Dq[didx[k][3]],
                       d4 = Dq[didx[k][4]], d5 = Dq[didx[k][5]];
            const Real gx = s_g[warp][0][q * NP + tb[k]], gy = s_g[warp][1][q * NP + tb[k]],
                       gz = s_g[warp][2][q * NP + tb[k]];
            Real* T = s_T[warp][tb[k]] + 3 * ti[k];
            T[0] = d0 * gx + d3 * gy + d5 * gz;
            T[1] = d1 * gy + d3 * gx + d4 * gz;
            T[2] = d2 * gz + d4 * gy + d5 * gx;
          }
          __syncwarp();
#pragma unroll
          for (int k = 0; k < PPL; ++k) {
            if (lane + 32 * k >= NPAIR) continue;
            const Real ax = s_g[warp][0][q * NP + pa[k]], ay = s_g[warp][1][q * NP + pa[k]],
                       az = s_g[warp][2][q * NP + pa[k]];
            const Real* T = s_T[warp][pb[k]];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              K[k][0][d] += ax * T[0 * 3 + d] + ay * T[3 * 3 + d] + az * T[5 * 3 + d];
              K[k][1][d] += ay * T[1 * 3 + d] + ax * T[3 * 3 + d] + az * T[4 * 3 + d];
              K[k][2][d] += az * T[2 * 3 + d] + ay * T[4 * 3 + d] + ax * T[5 * 3 + d];
            }
          }
          __syncwarp();
        }
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
          const int p = lane + 32 * k;
          if (p >= NPAIR) continue;
          Real* o = kbuf + ((long long)el * NPAIR + p) * 9;
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) o[c * 3 + d] = K[k][c][d];
        }
      }
      __syncwarp();
    }
    __syncthreads();
  }
  if (WANT & 1) {
    if (A.rhs)  // load term -f.u of the owned DOFs
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_owned; i += gridDim.x * blockDim.x)
        eacc -= A.rhs[i] * A.u[A.lo + i];
    m3_energy_finalize(eacc, A);
  }
}

// P4 tetrahedra (35 nodes, up to kM3MaxQHi points): the same point tiles;
// the contraction keeps one node b at a time, (w D) B(b) at every point of
// the element in shared memory, and lanes over the nodes a <= b accumulate
// B(a)^T (w D) B(b) over the points, reading the basis gradients of a from
// global memory (the 3 x nq x 35 gradient table of one element does not fit
// beside the point tiles).
constexpr int kM3MaxQHi = 32;

template <typename Real, int NP, int WANT>
__global__ void __launch_bounds__(32 * kM3Warps) k_mc3d_elem_hi(Mc3dArgs A, Real* __restrict__ kbuf,
                                                                Real* __restrict__ gbuf) {
  constexpr int N = 3 * NP, NPAIR = NP * (NP + 1) / 2, NT = 32 * kM3Warps;
  __shared__ Real s_sig[NT][6];
  __shared__ Real s_D[NT][21];
  __shared__ Real s_T[kM3Warps][kM3MaxQHi][18];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nq = A.nq, epc = NT / nq;
  double eacc = 0.0;
  for (int el0 = blockIdx.x * epc; el0 < A.n_el; el0 += gridDim.x * epc) {
    const int ne = min(epc, A.n_el - el0);
    if ((int)threadIdx.x < ne * nq) {
      const int j = threadIdx.x / nq, q = threadIdx.x - j * nq, el = el0 + j;
      const double wpsi = m3_point_update<Real, NP>(A.grad, A.codes, A.u, A.dir, A.pt, el, q, nq, A.tiny,
                                                    A.elastic, s_sig[threadIdx.x], s_D[threadIdx.x]);
      if ((WANT & 1) && __ldg(A.wflag + el)) eacc += wpsi;
    }
    __syncthreads();
    for (int j = warp; (WANT & 6) && j < ne; j += kM3Warps) {
      const int el = el0 + j;
      const Real(*sg)[6] = s_sig + j * nq;
      const Real(*sD)[21] = s_D + j * nq;
      const double* gx_ = A.grad + (long long)el * 3 * nq * NP;
      const double* gy_ = gx_ + nq * NP;
      const double* gz_ = gy_ + nq * NP;
      if (WANT & 2) {
        for (int i = lane; i < N; i += 32) {
          const int a = i / 3, c = i - 3 * a;
          Real s = Real(0);
          for (int q = 0; q < nq; ++q) {
            Real b[6];
            m3_bcol<Real>((Real)__ldg(gx_ + q * NP + a), (Real)__ldg(gy_ + q * NP + a), (Real)__ldg(gz_ + q * NP + a),
                          c, b);
#pragma unroll
            for (int k = 0; k < 6; ++k) s += b[k] * sg[q][k];
          }
          gbuf[(long long)el * N + i] = s;
        }
      }
      if (WANT & 4) {
        for (int b = 0; b < NP; ++b) {
          for (int q = lane; q < nq; q += 32) {
            const Real* Dq = sD[q];
            Real D[6][6];
            int t = 0;
#pragma unroll
            for (int i = 0; i < 6; ++i)
#pragma unroll
              for (int k = i; k < 6; ++k) {
                D[i][k] = Dq[t];
                D[k][i] = Dq[t];
                ++t;
              }
            const Real gx = (Real)__ldg(gx_ + q * NP + b), gy = (Real)__ldg(gy_ + q * NP + b),
                       gz = (Real)__ldg(gz_ + q * NP + b);
            Real* T = s_T[warp][q];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
              T[i * 3 + 0] = D[i][0] * gx + D[i][3] * gy + D[i][5] * gz;
              T[i * 3 + 1] = D[i][1] * gy + D[i][3] * gx + D[i][4] * gz;
              T[i * 3 + 2] = D[i][2] * gz + D[i][4] * gy + D[i][5] * gx;
            }
          }
          __syncwarp();
          for (int a = lane; a <= b; a += 32) {
            Real K[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int d = 0; d < 3; ++d) K[c][d] = Real(0);
            for (int q = 0; q < nq; ++q) {
              const Real ax = (Real)__ldg(gx_ + q * NP + a), ay = (Real)__ldg(gy_ + q * NP + a),
                         az = (Real)__ldg(gz_ + q * NP + a);
              const Real* T = s_T[warp][q];
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                K[0][d] += ax * T[0 * 3 + d] + ay * T[3 * 3 + d] + az * T[5 * 3 + d];
                K[1][d] += ay * T[1 * 3 + d] + ax * T[3 * 3 + d] + az * T[4 * 3 + d];
                K[2][d] += az * T[2 * 3 + d] + ay * T[4 * 3 + d] + ax * T[5 * 3 + d];
              }
            }
            // pair (a, b), a <= b, in row-major upper-triangle order
            const int p = a * NP - a * (a - 1) / 2 + (b - a);
            Real* o = kbuf + ((long long)el * NPAIR + p) * 9;
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int d = 0; d < 3; ++d) o[c * 3 + d] = K[c][d];
          }
          __syncwarp();
        }
      }
    }
    __syncthreads();
  }
  if (WANT & 1) {
    if (A.rhs)  // load term -f.u of the owned DOFs
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_owned; i += gridDim.x * blockDim.x)
        eacc -= A.rhs[i] * A.u[A.lo + i];
    m3_energy_finalize(eacc, A);
  }
}

}  // namespace

struct Mc3dHandle {
  int precision = 0, hess_fp32 = 0, np = 0, nq = 0, n_local = 0, num_sms = 148;
  int64_t nnz = 0, lo = 0, hi = 0, n_free = 0, n_total = 0;
  double tiny = 1.0e-15;
  int elastic = 0;
  int *codes = nullptr;
  double *grad = nullptr, *pt = nullptr, *dir = nullptr, *rhs = nullptr, *partials = nullptr;
  unsigned char* wflag = nullptr;
  unsigned* counter = nullptr;
  void *kbuf = nullptr, *gbuf = nullptr;
  int grid_elem = 1, n_rnodes = 0;
  int *bp_rn_blk = nullptr, *bp_rn_con = nullptr, *bp_rn_row = nullptr, *bp_rn_gpos = nullptr,
      *bp_rn_inc = nullptr, *bp_con = nullptr, *bp_inc = nullptr;
  unsigned* bp_blk = nullptr;
  int64_t device_bytes = 0, n_contrib = 0;
};

namespace {

template <typename T>
int m3_upload(Mc3dHandle* h, T** p, const T* src, size_t count) {
  *p = nullptr;
  if (count == 0) return FNE_OK;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return set_error(FNE_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->device_bytes += (int64_t)(count * sizeof(T));
  if (src) {
    e = cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
  }
  return FNE_OK;
}

// resident CTAs per SM of the fused pass (registers and shared memory)
template <typename Real>
int m3_ctas_per_sm(int np) {
  int n = 0;
  const cudaError_t e =
      np == 35   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_mc3d_elem_hi<Real, 35, 7>, 32 * kM3Warps, 0)
      : np == 10 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_mc3d_elem<Real, 10, 7>, 32 * kM3Warps, 0)
                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_mc3d_elem<Real, 4, 7>, 32 * kM3Warps, 0);
  return e == cudaSuccess && n > 0 ? n : 2;
}

template <typename Real, typename HOut, int NP>
cudaError_t m3_launch(Mc3dHandle* h, int flags, const double* u, double* energy, double* grad, void* hess,
                      cudaStream_t st) {
  Mc3dArgs A{h->n_local, h->nq,    h->codes, h->grad,    h->pt,  h->wflag, u,
             h->dir,     h->rhs,   (int)(h->hi - h->lo), h->lo,  h->tiny,  h->elastic,
             h->partials, h->counter, energy};
  Real* kb = static_cast<Real*>(h->kbuf);
  Real* gb = static_cast<Real*>(h->gbuf);
  const dim3 grid(h->grid_elem), block(32 * kM3Warps);
#define M3_CASE(W)                                                    \
  case W:                                                             \
    if constexpr (NP > 10)                                            \
      k_mc3d_elem_hi<Real, NP, W><<<grid, block, 0, st>>>(A, kb, gb); \
    else                                                              \
      k_mc3d_elem<Real, NP, W><<<grid, block, 0, st>>>(A, kb, gb);    \
    break;
  switch (flags) {
    M3_CASE(1)
    M3_CASE(2)
    M3_CASE(3)
    M3_CASE(4)
    M3_CASE(5)
    M3_CASE(6)
    M3_CASE(7)
    default: return cudaErrorInvalidValue;
  }
#undef M3_CASE
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !(flags & 6) || h->n_rnodes == 0) return e;
  NodeGatherArgs G{h->n_rnodes, h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row, h->bp_rn_gpos,
                   h->bp_rn_inc, h->bp_blk,   h->bp_con,    h->bp_inc,    h->rhs};
  HOut* H = static_cast<HOut*>(hess);
  if (flags & 4) {
    const int gg = std::max(1, std::min(h->num_sms * 16, (h->n_rnodes + 7) / 8));
    if (flags & 2)
      k_node_gather<Real, HOut, 3, NP, true, true><<<gg, 256, 0, st>>>(G, kb, gb, H, grad);
    else
      k_node_gather<Real, HOut, 3, NP, true, false><<<gg, 256, 0, st>>>(G, kb, gb, H, grad);
  } else {
    const int gr = std::max(1, std::min(h->num_sms * 8, (h->n_rnodes + 255) / 256));
    k_rowgrad<Real, 3><<<gr, 256, 0, st>>>(h->n_rnodes, h->bp_rn_inc, h->bp_inc, h->bp_rn_gpos, gb, h->rhs, grad);
  }
  return cudaGetLastError();
}

template <typename Real, typename HOut>
cudaError_t m3_dispatch(Mc3dHandle* h, int flags, const double* u, double* energy, double* grad, void* hess,
                        cudaStream_t st) {
  if (h->np == 35) return m3_launch<Real, HOut, 35>(h, flags, u, energy, grad, hess, st);
  if (h->np == 10) return m3_launch<Real, HOut, 10>(h, flags, u, energy, grad, hess, st);
  return m3_launch<Real, HOut, 4>(h, flags, u, energy, grad, hess, st);
}

}  // namespace

void mc3d_destroy(Mc3dHandle* h) {
  if (!h) return;
  void* ptrs[] = {h->codes, h->grad, h->pt, h->dir, h->rhs, h->partials, h->wflag, h->counter, h->kbuf, h->gbuf,
                  h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row, h->bp_rn_gpos, h->bp_rn_inc, h->bp_con, h->bp_inc,
                  h->bp_blk};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete h;
}

int mc3d_create(const fne_desc* d, Mc3dHandle** out) {
  *out = nullptr;
  const int np = d->npe, nq = d->nq, n = 3 * np;
  if (d->block_size != 3) return set_error(FNE_EINVAL, "Mohr-Coulomb 3-D: block_size must be 3");
  if (np != 4 && np != 10 && np != 35)
    return set_error(FNE_EINVAL, "Mohr-Coulomb 3-D: P1 (4 nodes), P2 (10 nodes) or P4 (35 nodes) tetrahedra");
  if (nq < 1 || nq > (np == 35 ? kM3MaxQHi : kM3MaxQ))
    return set_error(FNE_EINVAL, "Mohr-Coulomb 3-D: 1 to 16 quadrature points (P1, P2) or 1 to 32 (P4)");
  if (d->n_elem > 0 && (!d->e0 || !d->e1 || !d->e2 || !d->e3))
    return set_error(FNE_EINVAL, "Mohr-Coulomb 3-D: missing basis gradients or per-point inputs");
  const int64_t E = d->n_elem, lo = d->lo, hi = d->hi;
  const int64_t* t2f = d->total_to_free_reord;
  const int npair = np * (np + 1) / 2;
  if (E * (int64_t)npair * 9 >= (int64_t)INT32_MAX * 4 || d->nnz >= (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS, "Mohr-Coulomb 3-D: sizes beyond the supported indexing");
  std::vector<int32_t> codes;
  std::vector<double> grad, pt;
  std::vector<uint8_t> wflag;
  std::vector<int64_t> local;
  for (int64_t e = 0; e < E; ++e) {
    bool own = false;
    for (int i = 0; i < n; ++i) {
      const int64_t dof = d->elems[e * n + i];
      if (dof < 0 || dof >= d->n_total) return set_error(FNE_EBOUNDS, "Mohr-Coulomb 3-D: element DOF out of range");
      const int64_t r = t2f[dof];
      own |= r >= lo && r < hi;
    }
    if (!own) continue;
    local.push_back(e);
    for (int i = 0; i < n; ++i) {
      const int64_t dof = d->elems[e * n + i];
      if (dof + 1 >= (int64_t)INT32_MAX) return set_error(FNE_EBOUNDS, "Mohr-Coulomb 3-D: DOF id beyond int32");
      codes.push_back(t2f[dof] >= 0 ? (int32_t)t2f[dof] : (int32_t)(-1 - dof));
    }
    for (const double* g : {d->e0, d->e1, d->e2})
      grad.insert(grad.end(), g + e * nq * np, g + (e + 1) * nq * np);
    pt.insert(pt.end(), d->e3 + e * nq * kM3Pt, d->e3 + (e + 1) * nq * kM3Pt);
    const double w = d->energy_weights ? d->energy_weights[e] : 1.0;
    if (w != 0.0 && w != 1.0) return set_error(FNE_EINVAL, "Mohr-Coulomb 3-D: energy weights must be 0 or 1");
    wflag.push_back(w != 0.0 ? 1 : 0);
  }
  const int64_t nl = (int64_t)local.size();
  BlockPlan bp;
  {
    std::vector<int64_t> edofs((size_t)nl * n);
    for (int64_t le = 0; le < nl; ++le)
      for (int i = 0; i < n; ++i) edofs[(size_t)le * n + i] = d->elems[local[le] * n + i];
    const int rc = build_block_plan(nl, np, 3, edofs.data(), d, bp);
    if (rc) return rc;
  }
  auto* h = new (std::nothrow) Mc3dHandle();
  if (!h) return set_error(FNE_ENOMEM, "Mohr-Coulomb 3-D: out of host memory");
  h->precision = d->precision;
  h->hess_fp32 = d->precision == FNE_FP32 && d->hess_fp32;
  h->np = np;
  h->nq = nq;
  h->n_local = (int)nl;
  h->nnz = d->nnz;
  h->lo = lo;
  h->hi = hi;
  h->n_free = d->n_free;
  h->n_total = d->n_total;
  h->tiny = d->s[0] > 0.0 ? d->s[0] : 1.0e-15;
  h->elastic = d->s[5] != 0.0;
  h->n_rnodes = bp.n_rnodes;
  h->n_contrib = (int64_t)bp.con.size();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    mc3d_destroy(h);
    return set_error(FNE_ECUDA, "Mohr-Coulomb 3-D: device query");
  }
  // tiles of 128 / nq elements (all their points in one pass of the CTA);
  // one wave of resident CTAs, each striding over the tiles
  const int64_t epc = 32 * kM3Warps / nq;
  const int per_sm = d->precision == FNE_FP64 ? m3_ctas_per_sm<double>(h->np) : m3_ctas_per_sm<float>(h->np);
  h->grid_elem = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)h->num_sms * per_sm, (nl + epc - 1) / epc));
  const size_t rsz = d->precision == FNE_FP32 ? sizeof(float) : sizeof(double);
  int rc = FNE_OK;
#define M3_TRY(x)       \
  do {                  \
    rc = (x);           \
    if (rc) {           \
      mc3d_destroy(h);  \
      return rc;        \
    }                   \
  } while (0)
  M3_TRY(m3_upload(h, &h->codes, codes.data(), codes.size()));
  M3_TRY(m3_upload(h, &h->grad, grad.data(), grad.size()));
  M3_TRY(m3_upload(h, &h->pt, pt.data(), pt.size()));
  M3_TRY(m3_upload(h, &h->wflag, wflag.data(), wflag.size()));
  M3_TRY(m3_upload(h, &h->dir, d->dirichlet, (size_t)d->n_total));
  if (d->rhs_owned) M3_TRY(m3_upload(h, &h->rhs, d->rhs_owned, (size_t)(hi - lo)));
  M3_TRY(m3_upload(h, &h->partials, (const double*)nullptr, (size_t)h->grid_elem));
  M3_TRY(m3_upload(h, &h->counter, (const unsigned*)nullptr, 1));
  if (cudaMemset(h->counter, 0, sizeof(unsigned)) != cudaSuccess) {
    mc3d_destroy(h);
    return set_error(FNE_ECUDA, "Mohr-Coulomb 3-D: cudaMemset");
  }
  M3_TRY(m3_upload(h, &h->bp_rn_blk, bp.rn_blk.data(), bp.rn_blk.size()));
  M3_TRY(m3_upload(h, &h->bp_rn_con, bp.rn_con.data(), bp.rn_con.size()));
  M3_TRY(m3_upload(h, &h->bp_rn_row, bp.rn_row.data(), bp.rn_row.size()));
  M3_TRY(m3_upload(h, &h->bp_rn_gpos, bp.rn_gpos.data(), bp.rn_gpos.size()));
  M3_TRY(m3_upload(h, &h->bp_rn_inc, bp.rn_inc.data(), bp.rn_inc.size()));
  M3_TRY(m3_upload(h, &h->bp_blk, bp.blk.data(), bp.blk.size()));
  M3_TRY(m3_upload(h, &h->bp_con, bp.con.data(), bp.con.size()));
  M3_TRY(m3_upload(h, &h->bp_inc, bp.inc.data(), bp.inc.size()));
  unsigned char* kb = nullptr;
  M3_TRY(m3_upload(h, &kb, (const unsigned char*)nullptr, std::max<size_t>(1, (size_t)nl * npair * 9 * rsz)));
  h->kbuf = kb;
  unsigned char* gb = nullptr;
  M3_TRY(m3_upload(h, &gb, (const unsigned char*)nullptr, std::max<size_t>(1, (size_t)nl * n * rsz)));
  h->gbuf = gb;
#undef M3_TRY
  *out = h;
  return FNE_OK;
}

int mc3d_eval(Mc3dHandle* h, const double* u, int flags, double* energy, double* grad, void* hess, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (h->precision == FNE_FP64)
    e = m3_dispatch<double, double>(h, flags, u, energy, grad, hess, st);
  else if (h->hess_fp32)
    e = m3_dispatch<float, float>(h, flags, u, energy, grad, hess, st);
  else
    e = m3_dispatch<float, double>(h, flags, u, energy, grad, hess, st);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_eval launch: ") + cudaGetErrorString(e));
  return FNE_OK;
}

int mc3d_set_dirichlet(Mc3dHandle* h, const double* dirichlet) {
  cudaError_t e = cudaMemcpy(h->dir, dirichlet, h->n_total * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_set_dirichlet: ") + cudaGetErrorString(e));
  return FNE_OK;
}

void mc3d_info(const Mc3dHandle* h, fne_info* info) {
  info->n_rows = h->hi - h->lo;
  info->nnz = h->nnz;
  info->n_elem = h->n_local;
  info->n_incidences = h->n_contrib;
  info->device_bytes = h->device_bytes;
  info->max_row_len = 0;
  info->kernel_variant = 11;
  info->row_lanes = 1;
}

}  // namespace fne
