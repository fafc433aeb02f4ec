// Plane-strain Mohr-Coulomb (slope stability) on Pk Lagrange triangles.
//
// Replaces the element kernels of the reference's slope assembler
// (src/problems/slope_stability/jax_petsc/reordered_element_assembler.py:152-243)
// and the energy of src/problems/slope_stability/jax/jax_energy.py:45-142:
//   e = sum_q w_q psi(B_q u - eps_p_old),  g = sum_q w_q B_q^T sigma_q,
//   K = sum_q w_q B_q^T C_q B_q,
// with sigma = dpsi/deps (the returned stress) and C = dsigma/deps (the
// consistent tangent of the line / apex return), written by hand instead of
// JAX's autodiff through lax.cond.  B_q is rebuilt on the fly from the
// affine element map: B_q = (reference basis gradients at q) x J^-1, so the
// element data is 5 numbers instead of the reference's nq x 3 x 2n elem_B.
//
// Three kernels: k_mc_elem (one warp per element: nodal values and basis
// gradients staged in shared memory, one lane per quadrature point for the
// constitutive update, lanes over node pairs for the 2x2 blocks of K), and
// two gathers that sum the element matrices / vectors into the owned COO
// values and the gradient in a fixed order (no atomics, deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fne_internal.h"

namespace fne {

namespace {

struct McConst {
  double C00, C01, C22, S00, S01, S22;
  double alpha, beta, kappa, z1, z2, nz, s_apex, reg;
  int elastic_only;
};

template <typename Real>
struct McConstR {
  Real C00, C01, C22, S00, S01, S22, alpha, beta, kappa, z1, z2, inz, s_apex, reg;
  int elastic_only;
};

template <typename Real>
__host__ McConstR<Real> cast_const(const McConst& m) {
  McConstR<Real> r;
  r.C00 = (Real)m.C00; r.C01 = (Real)m.C01; r.C22 = (Real)m.C22;
  r.S00 = (Real)m.S00; r.S01 = (Real)m.S01; r.S22 = (Real)m.S22;
  r.alpha = (Real)m.alpha; r.beta = (Real)m.beta; r.kappa = (Real)m.kappa;
  r.z1 = (Real)m.z1; r.z2 = (Real)m.z2; r.inz = (Real)(1.0 / m.nz);
  r.s_apex = (Real)m.s_apex; r.reg = (Real)m.reg;
  r.elastic_only = m.elastic_only;
  return r;
}

// One quadrature point: returned stress sig, upper triangle of the consistent
// tangent Ct (00, 01, 02, 11, 12, 22) and the energy density psi.
template <typename Real>
__device__ __forceinline__ void mc_point(const McConstR<Real>& M, const Real e[3], Real sig[3], Real Ct[6],
                                         Real& psi) {
  const Real sxx = M.C00 * e[0] + M.C01 * e[1];
  const Real syy = M.C01 * e[0] + M.C00 * e[1];
  const Real t = M.C22 * e[2];
  const Real m = Real(0.5) * (sxx + syy), d = Real(0.5) * (sxx - syy);
  const Real r = sqrt(d * d + t * t + M.reg * M.reg);
  const Real s1 = m + r, s2 = m - r;
  const Real f = M.alpha * s1 - M.beta * s2 - M.kappa;
  if (M.elastic_only || f <= Real(0)) {
    sig[0] = sxx; sig[1] = syy; sig[2] = t;
    Ct[0] = M.C00; Ct[1] = M.C01; Ct[2] = Real(0); Ct[3] = M.C00; Ct[4] = Real(0); Ct[5] = M.C22;
  } else {
    // line return in principal space (metric: plane-strain compliance), or apex
    const Real lam = f * M.inz;
    const Real s1L = s1 - lam * M.z1, s2L = s2 - lam * M.z2;
    Real s1p, s2p, P11, P12, P21, P22;
    if (s1L >= s2L) {
      s1p = s1L; s2p = s2L;
      P11 = Real(1) - M.alpha * M.z1 * M.inz; P12 = M.beta * M.z1 * M.inz;
      P21 = -M.alpha * M.z2 * M.inz;          P22 = Real(1) + M.beta * M.z2 * M.inz;
    } else {
      s1p = s2p = M.s_apex;
      P11 = P12 = P21 = P22 = Real(0);
    }
    const Real mp = Real(0.5) * (s1p + s2p), rp = Real(0.5) * (s1p - s2p);
    const Real rho2 = d * d + t * t;
    Real c = Real(1), s = Real(0), dc_d = Real(0), dc_t = Real(0), ds_d = Real(0), ds_t = Real(0);
    if (rho2 > Real(0)) {
      const Real rho = sqrt(rho2), ir3 = Real(1) / (rho2 * rho);
      c = d / rho; s = t / rho;
      dc_d = t * t * ir3; dc_t = -d * t * ir3; ds_d = dc_t; ds_t = d * d * ir3;
    }
    sig[0] = mp + rp * c; sig[1] = mp - rp * c; sig[2] = rp * s;
    // derivatives with respect to (m, d, t)
    const Real ir = Real(1) / r;
    const Real a1 = Real(0.5) * (P11 + P21), a2 = Real(0.5) * (P12 + P22);  // dmp = a1 ds1 + a2 ds2
    const Real b1 = Real(0.5) * (P11 - P21), b2 = Real(0.5) * (P12 - P22);  // drp = b1 ds1 + b2 ds2
    // ds1 = (1, d/r, t/r), ds2 = (1, -d/r, -t/r)
    const Real dmp_m = a1 + a2, dmp_d = (a1 - a2) * d * ir, dmp_t = (a1 - a2) * t * ir;
    const Real drp_m = b1 + b2, drp_d = (b1 - b2) * d * ir, drp_t = (b1 - b2) * t * ir;
    // dsig / d(m, d, t)
    const Real g0m = dmp_m + c * drp_m, g0d = dmp_d + c * drp_d + rp * dc_d, g0t = dmp_t + c * drp_t + rp * dc_t;
    const Real g1m = dmp_m - c * drp_m, g1d = dmp_d - c * drp_d - rp * dc_d, g1t = dmp_t - c * drp_t - rp * dc_t;
    const Real g2m = s * drp_m, g2d = s * drp_d + rp * ds_d, g2t = s * drp_t + rp * ds_t;
    // (m, d, t) = (0.5 (sxx + syy), 0.5 (sxx - syy), txy): D = dsig / dsig_tr
    const Real D00 = Real(0.5) * (g0m + g0d), D01 = Real(0.5) * (g0m - g0d), D02 = g0t;
    const Real D10 = Real(0.5) * (g1m + g1d), D11 = Real(0.5) * (g1m - g1d), D12 = g1t;
    const Real D20 = Real(0.5) * (g2m + g2d), D21 = Real(0.5) * (g2m - g2d), D22 = g2t;
    // Ct = D C (symmetric for the exact return; upper triangle kept)
    Ct[0] = D00 * M.C00 + D01 * M.C01;
    Ct[1] = D00 * M.C01 + D01 * M.C00;
    Ct[2] = D02 * M.C22;
    Ct[3] = D10 * M.C01 + D11 * M.C00;
    Ct[4] = D12 * M.C22;
    Ct[5] = D22 * M.C22;
    (void)D20; (void)D21;
  }
  // psi = sig . eps - 1/2 sig . S sig
  const Real Ss0 = M.S00 * sig[0] + M.S01 * sig[1], Ss1 = M.S01 * sig[0] + M.S00 * sig[1], Ss2 = M.S22 * sig[2];
  psi = sig[0] * e[0] + sig[1] * e[1] + sig[2] * e[2] - Real(0.5) * (sig[0] * Ss0 + sig[1] * Ss1 + sig[2] * Ss2);
}


// FP64 energy reduction: warp shuffles, per-CTA partial, last CTA sums the
// partials in index order (atomic ticket; no waiting).
__device__ double mc_block_sum(double v, double* ws) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? ws[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

__device__ void mc_energy_finalize(double v, double* partials, unsigned* counter, double* out) {
  __shared__ double ws[32];
  __shared__ int is_last;
  v = mc_block_sum(v, ws);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = v;
    __threadfence();
    is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s = 0.0;
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) s += __ldcg(partials + j);
  s = mc_block_sum(s, ws);
  if (threadIdx.x == 0) {
    out[0] = s;
    *counter = 0u;
  }
}

enum { MW_E = 1, MW_G = 2, MW_H = 4 };
constexpr int kMcWarps = 4;  // elements per CTA (one warp each)

struct McArgs {
  int n_el;
  const int* __restrict__ codes;     // [n_el * n] per-DOF gather codes
  const double* __restrict__ geom;   // [n_el * 5] J^-1 (4), |det J|
  const double* __restrict__ epsp;   // [n_el * nq * 3] or null
  const unsigned char* __restrict__ wflag;  // [n_el]
  const double* __restrict__ dhat1;  // [nq * np]
  const double* __restrict__ dhat2;  // [nq * np]
  const double* __restrict__ qw;     // [nq]
  const double* __restrict__ u;
  const double* __restrict__ dir;
  const double* __restrict__ rhs;    // [n_owned] or null
  int n_owned;
  long long lo;
};

template <typename Real, int NP, int NQ, int WANT>
__global__ void __launch_bounds__(32 * kMcWarps) k_mc_elem(McArgs A, McConstR<Real> M, Real* __restrict__ Kbuf,
                                                           Real* __restrict__ gbuf, double* __restrict__ partials,
                                                           unsigned* __restrict__ counter, double* __restrict__ eout) {
  constexpr int N = 2 * NP;
  constexpr int NPAIR = NP * (NP + 1) / 2;
  constexpr int PPL = (NPAIR + 31) / 32;  // node pairs per lane
  __shared__ Real s_dh1[NQ * NP], s_dh2[NQ * NP], s_w[NQ];
  __shared__ Real s_gx[kMcWarps][NQ * NP], s_gy[kMcWarps][NQ * NP];
  __shared__ Real s_u[kMcWarps][N];
  __shared__ Real s_sig[kMcWarps][NQ * 3], s_C[kMcWarps][NQ * 6];
  __shared__ Real s_T[kMcWarps][NP * 6];
  for (int i = threadIdx.x; i < NQ * NP; i += blockDim.x) {
    s_dh1[i] = (Real)A.dhat1[i];
    s_dh2[i] = (Real)A.dhat2[i];
  }
  for (int i = threadIdx.x; i < NQ; i += blockDim.x) s_w[i] = (Real)A.qw[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Real* gx = s_gx[wid];
  Real* gy = s_gy[wid];
  Real* ue = s_u[wid];
  Real* ws = s_sig[wid];
  Real* wC = s_C[wid];
  Real* T = s_T[wid];
  double eacc = 0.0;
  const int gwarps = gridDim.x * kMcWarps;
  for (int e = blockIdx.x * kMcWarps + wid; e < A.n_el; e += gwarps) {
    const double* gm = A.geom + 5LL * e;
    const Real i00 = (Real)gm[0], i01 = (Real)gm[1], i10 = (Real)gm[2], i11 = (Real)gm[3];
    const Real dj = (Real)gm[4];
    for (int i = lane; i < N; i += 32) {
      const int code = A.codes[(long long)e * N + i];
      ue[i] = (Real)(code >= 0 ? A.u[code] : A.dir[-1 - code]);
    }
    for (int i = lane; i < NQ * NP; i += 32) {
      gx[i] = i00 * s_dh1[i] + i01 * s_dh2[i];
      gy[i] = i10 * s_dh1[i] + i11 * s_dh2[i];
    }
    __syncwarp();
    if (lane < NQ) {  // constitutive update, one lane per quadrature point
      const int q = lane;
      Real ex = Real(0), ey = Real(0), exy = Real(0);
#pragma unroll 5
      for (int a = 0; a < NP; ++a) {
        const Real px = gx[q * NP + a], py = gy[q * NP + a];
        const Real ux = ue[2 * a], uy = ue[2 * a + 1];
        ex += px * ux;
        ey += py * uy;
        exy += py * ux + px * uy;
      }
      Real eps[3] = {ex, ey, exy};
      if (A.epsp) {
        const double* ep = A.epsp + ((long long)e * NQ + q) * 3;
        eps[0] -= (Real)ep[0]; eps[1] -= (Real)ep[1]; eps[2] -= (Real)ep[2];
      }
      Real sig[3], Ct[6], psi;
      mc_point(M, eps, sig, Ct, psi);
      const Real w = dj * s_w[q];
#pragma unroll
      for (int k = 0; k < 3; ++k) ws[q * 3 + k] = w * sig[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) wC[q * 6 + k] = w * Ct[k];
      if ((WANT & MW_E) && A.wflag[e]) eacc += (double)(w * psi);
    }
    __syncwarp();
    if (WANT & MW_G) {  // g_(a,c) = sum_q G_a^T (w sigma)_q
      for (int i = lane; i < N; i += 32) {
        const int a = i >> 1, c = i & 1;
        Real acc = Real(0);
#pragma unroll 5
        for (int q = 0; q < NQ; ++q) {
          const Real px = gx[q * NP + a], py = gy[q * NP + a];
          acc += c == 0 ? px * ws[q * 3] + py * ws[q * 3 + 2] : py * ws[q * 3 + 1] + px * ws[q * 3 + 2];
        }
        gbuf[(long long)e * N + i] = acc;
      }
    }
    if (WANT & MW_H) {  // K_ab = sum_q G_a^T (w C_q) G_b, node pairs a <= b spread over lanes
      Real kacc[PPL][4];
      int pa[PPL], pb[PPL];
#pragma unroll
      for (int k = 0; k < PPL; ++k) {
        int p = lane + 32 * k;
        int a = 0;
        while (p >= NP - a && a < NP) {  // pair index -> (a, b), b >= a
          p -= NP - a;
          ++a;
        }
        pa[k] = a;
        pb[k] = a + p;
        kacc[k][0] = kacc[k][1] = kacc[k][2] = kacc[k][3] = Real(0);
      }
      for (int q = 0; q < NQ; ++q) {
        // T_b = (w C_q) G_b : rows (xx, yy, xy) x cols (x, y)
        for (int i = lane; i < NP * 6; i += 32) {
          const int b = i / 6, k = i - 6 * b, row = k >> 1, col = k & 1;
          const Real px = gx[q * NP + b], py = gy[q * NP + b];
          const Real* C = wC + q * 6;
          const Real Cr0 = row == 0 ? C[0] : (row == 1 ? C[1] : C[2]);
          const Real Cr1 = row == 0 ? C[1] : (row == 1 ? C[3] : C[4]);
          const Real Cr2 = row == 0 ? C[2] : (row == 1 ? C[4] : C[5]);
          T[i] = col == 0 ? Cr0 * px + Cr2 * py : Cr1 * py + Cr2 * px;
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
          if (lane + 32 * k < NPAIR) {
            const Real ax = gx[q * NP + pa[k]], ay = gy[q * NP + pa[k]];
            const Real* Tb = T + 6 * pb[k];
            // rows (a,x): ax T0 + ay T2 ; rows (a,y): ay T1 + ax T2
            kacc[k][0] += ax * Tb[0] + ay * Tb[4];
            kacc[k][1] += ax * Tb[1] + ay * Tb[5];
            kacc[k][2] += ay * Tb[2] + ax * Tb[4];
            kacc[k][3] += ay * Tb[3] + ax * Tb[5];
          }
        }
        __syncwarp();
      }
      Real* Ke = Kbuf + (long long)e * N * N;
#pragma unroll
      for (int k = 0; k < PPL; ++k) {
        if (lane + 32 * k < NPAIR) {
          const int a = pa[k], b = pb[k];
          Ke[(2 * a) * N + 2 * b] = kacc[k][0];
          Ke[(2 * a) * N + 2 * b + 1] = kacc[k][1];
          Ke[(2 * a + 1) * N + 2 * b] = kacc[k][2];
          Ke[(2 * a + 1) * N + 2 * b + 1] = kacc[k][3];
          if (a != b) {
            Ke[(2 * b) * N + 2 * a] = kacc[k][0];
            Ke[(2 * b + 1) * N + 2 * a] = kacc[k][1];
            Ke[(2 * b) * N + 2 * a + 1] = kacc[k][2];
            Ke[(2 * b + 1) * N + 2 * a + 1] = kacc[k][3];
          }
        }
      }
    }
    __syncwarp();
  }
  if (WANT & MW_E) {
    if (A.rhs)
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n_owned; i += gridDim.x * blockDim.x)
        eacc -= A.rhs[i] * A.u[A.lo + i];
    mc_energy_finalize(eacc, partials, counter, eout);
  }
}

// COO values: position p sums its element-matrix entries in element order.
template <typename Real, typename HOut>
__global__ void k_mc_gather(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                            const Real* __restrict__ src, HOut* __restrict__ out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    Real acc = Real(0);
    for (int j = ptr[p]; j < ptr[p + 1]; ++j) acc += src[idx[j]];
    out[p] = (HOut)acc;
  }
}

template <typename Real>
__global__ void k_mc_grad_gather(int n_rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                                 const Real* __restrict__ src, const int* __restrict__ gpos,
                                 const double* __restrict__ rhs, double* __restrict__ grad) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_rows; k += gridDim.x * blockDim.x) {
    Real acc = Real(0);
    for (int j = ptr[k]; j < ptr[k + 1]; ++j) acc += src[idx[j]];
    const int g = gpos[k];
    grad[g] = (double)acc - (rhs ? rhs[g] : 0.0);
  }
}

}  // namespace

struct McHandle {
  int precision = 0, hess_fp32 = 0, np = 0, nq = 0, n = 0;
  int n_local = 0, n_rows = 0, num_sms = 148;
  int64_t nnz = 0, lo = 0, hi = 0, n_free = 0, n_total = 0;
  McConst mc{};
  int* codes = nullptr;
  double *geom = nullptr, *epsp = nullptr, *dhat1 = nullptr, *dhat2 = nullptr, *qw = nullptr;
  unsigned char* wflag = nullptr;
  double *dir = nullptr, *rhs = nullptr, *partials = nullptr;
  unsigned* counter = nullptr;
  int *hptr = nullptr, *hidx = nullptr, *gptr = nullptr, *gidx = nullptr, *row_gpos = nullptr;
  void *Kbuf = nullptr, *gbuf = nullptr;
  int grid_elem = 1, n_partials = 1;
  int64_t device_bytes = 0, n_contrib = 0;
};

namespace {

template <typename T>
int mc_upload(McHandle* h, T** p, const T* src, size_t count) {
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

template <typename Real, typename HOut, int NP, int NQ>
cudaError_t mc_launch(McHandle* h, int flags, const double* u, double* energy, double* grad, void* hess,
                      cudaStream_t st) {
  McArgs A;
  A.n_el = h->n_local;
  A.codes = h->codes;
  A.geom = h->geom;
  A.epsp = h->epsp;
  A.wflag = h->wflag;
  A.dhat1 = h->dhat1;
  A.dhat2 = h->dhat2;
  A.qw = h->qw;
  A.u = u;
  A.dir = h->dir;
  A.rhs = h->rhs;
  A.n_owned = (int)(h->hi - h->lo);
  A.lo = h->lo;
  const McConstR<Real> M = cast_const<Real>(h->mc);
  Real* K = static_cast<Real*>(h->Kbuf);
  Real* g = static_cast<Real*>(h->gbuf);
  const int grid = h->grid_elem;
  const int T = 32 * kMcWarps;
  switch (flags) {
    case 1: k_mc_elem<Real, NP, NQ, 1><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 2: k_mc_elem<Real, NP, NQ, 2><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 3: k_mc_elem<Real, NP, NQ, 3><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 4: k_mc_elem<Real, NP, NQ, 4><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 5: k_mc_elem<Real, NP, NQ, 5><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 6: k_mc_elem<Real, NP, NQ, 6><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 7: k_mc_elem<Real, NP, NQ, 7><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int gg = std::max(1, std::min(h->num_sms * 16, (int)((std::max<int64_t>(h->nnz, h->n_rows) + 255) / 256)));
  if ((flags & MW_H) && h->nnz > 0)
    k_mc_gather<Real, HOut><<<gg, 256, 0, st>>>((int)h->nnz, h->hptr, h->hidx, K, static_cast<HOut*>(hess));
  if ((flags & MW_G) && h->n_rows > 0)
    k_mc_grad_gather<Real><<<gg, 256, 0, st>>>(h->n_rows, h->gptr, h->gidx, g, h->row_gpos, h->rhs, grad);
  return cudaGetLastError();
}

template <typename Real, typename HOut>
cudaError_t mc_dispatch(McHandle* h, int flags, const double* u, double* energy, double* grad, void* hess,
                        cudaStream_t st) {
  if (h->np == 3 && h->nq == 1) return mc_launch<Real, HOut, 3, 1>(h, flags, u, energy, grad, hess, st);
  if (h->np == 6 && h->nq == 7) return mc_launch<Real, HOut, 6, 7>(h, flags, u, energy, grad, hess, st);
  if (h->np == 15 && h->nq == 25) return mc_launch<Real, HOut, 15, 25>(h, flags, u, energy, grad, hess, st);
  return cudaErrorInvalidValue;
}

}  // namespace

void mc_destroy(McHandle* h) {
  if (!h) return;
  void* ptrs[] = {h->codes, h->geom, h->epsp, h->dhat1, h->dhat2, h->qw, h->wflag, h->dir, h->rhs,
                  h->partials, h->counter, h->hptr, h->hidx, h->gptr, h->gidx, h->row_gpos, h->Kbuf, h->gbuf};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete h;
}

int mc_create(const fne_desc* d, McHandle** out) {
  *out = nullptr;
  const int np = d->npe, nq = d->nq, n = 2 * np;
  if (d->block_size != 2) return set_error(FNE_EINVAL, "Mohr-Coulomb: block_size must be 2");
  if (!((np == 3 && nq == 1) || (np == 6 && nq == 7) || (np == 15 && nq == 25)))
    return set_error(FNE_EINVAL, "Mohr-Coulomb: supported (nodes, quadrature points): (3,1), (6,7), (15,25)");
  if (d->n_elem > 0 && (!d->e0 || !d->e1 || !d->e3))
    return set_error(FNE_EINVAL, "Mohr-Coulomb: missing element geometry or reference tables");
  const int64_t E = d->n_elem, lo = d->lo, hi = d->hi;
  const int64_t* t2f = d->total_to_free_reord;
  if (E * (int64_t)n * n >= (int64_t)INT32_MAX || d->nnz >= (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS, "Mohr-Coulomb: element matrices exceed 32-bit indexing");
  // per-DOF gather codes and local elements
  std::vector<int32_t> codes;
  std::vector<double> geom, epsp;
  std::vector<uint8_t> wflag;
  std::vector<int64_t> local;
  for (int64_t e = 0; e < E; ++e) {
    bool own = false;
    for (int i = 0; i < n; ++i) {
      const int64_t dof = d->elems[e * n + i];
      if (dof < 0 || dof >= d->n_total) return set_error(FNE_EBOUNDS, "Mohr-Coulomb: element DOF out of range");
      const int64_t r = t2f[dof];
      own |= r >= lo && r < hi;
    }
    if (!own) continue;
    local.push_back(e);
    for (int i = 0; i < n; ++i) {
      const int64_t dof = d->elems[e * n + i];
      codes.push_back(t2f[dof] >= 0 ? (int32_t)t2f[dof] : (int32_t)(-1 - dof));
    }
    for (int k = 0; k < 4; ++k) geom.push_back(d->e0[e * 4 + k]);
    geom.push_back(d->e1[e]);
    if (d->e2)
      for (int k = 0; k < nq * 3; ++k) epsp.push_back(d->e2[e * nq * 3 + k]);
    const double w = d->energy_weights ? d->energy_weights[e] : 1.0;
    if (w != 0.0 && w != 1.0) return set_error(FNE_EINVAL, "Mohr-Coulomb: energy weights must be 0 or 1");
    wflag.push_back(w != 0.0 ? 1 : 0);
  }
  const int64_t nl = (int64_t)local.size();
  // rows of the owned COO pattern (row-grouped)
  const int64_t n_owned = hi - lo;
  std::vector<int32_t> rowof(n_owned, -1), row_ptr, row_gpos;
  for (int64_t j = 0; j < d->nnz; ++j) {
    const int64_t r = d->owned_rows[j];
    if (r < lo || r >= hi) return set_error(FNE_EBOUNDS, "Mohr-Coulomb: owned row outside [lo, hi)");
    if (j == 0 || d->owned_rows[j - 1] != r) {
      if (rowof[r - lo] >= 0) return set_error(FNE_ELAYOUT, "Mohr-Coulomb: COO pattern is not row-grouped");
      rowof[r - lo] = (int32_t)row_ptr.size();
      row_ptr.push_back((int32_t)j);
      row_gpos.push_back((int32_t)(r - lo));
    }
  }
  for (int64_t i = 0; i < n_owned; ++i)
    if (rowof[i] < 0) {
      rowof[i] = (int32_t)row_ptr.size();
      row_ptr.push_back((int32_t)d->nnz);
      row_gpos.push_back((int32_t)i);
    }
  row_ptr.push_back((int32_t)d->nnz);
  const int32_t n_rows = (int32_t)row_gpos.size();
  // column lookup: positions of every row sorted by column id
  std::vector<int32_t> bycol(d->nnz);
  for (int32_t k = 0; k < n_rows; ++k) {
    for (int32_t p = row_ptr[k]; p < row_ptr[k + 1]; ++p) bycol[p] = p;
    std::sort(bycol.begin() + row_ptr[k], bycol.begin() + row_ptr[k + 1],
              [&](int32_t a, int32_t b) { return d->owned_cols[a] < d->owned_cols[b]; });
  }
  auto find = [&](int32_t k, int64_t col) -> int32_t {
    int32_t a = row_ptr[k], b = row_ptr[k + 1];
    while (a < b) {
      const int32_t m = (a + b) >> 1;
      if (d->owned_cols[bycol[m]] < col) a = m + 1; else b = m;
    }
    return (a < row_ptr[k + 1] && d->owned_cols[bycol[a]] == col) ? bycol[a] : -1;
  };
  // contributions (two passes: count, fill), in element order
  std::vector<int32_t> hptr(d->nnz + 1, 0), gptr(n_rows + 1, 0), hidx, gidx, hfill, gfill;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      for (int64_t p = 0; p < d->nnz; ++p) hptr[p + 1] += hptr[p];
      for (int32_t k = 0; k < n_rows; ++k) gptr[k + 1] += gptr[k];
      hidx.assign(hptr[d->nnz], 0);
      gidx.assign(gptr[n_rows], 0);
      hfill.assign(hptr.begin(), hptr.end() - 1);
      gfill.assign(gptr.begin(), gptr.end() - 1);
    }
    for (int64_t le = 0; le < nl; ++le) {
      const int32_t* c = codes.data() + le * n;
      for (int i = 0; i < n; ++i) {
        if (c[i] < lo || c[i] >= hi) continue;
        const int32_t k = rowof[c[i] - lo];
        if (pass == 0) gptr[k + 1]++; else gidx[gfill[k]++] = (int32_t)(le * n + i);
        for (int j = 0; j < n; ++j) {
          if (c[j] < 0) continue;
          const int32_t p = find(k, c[j]);
          if (p < 0) return set_error(FNE_ELAYOUT, "Scatter lookup found mismatched owned COO entries");
          if (pass == 0) hptr[p + 1]++; else hidx[hfill[p]++] = (int32_t)(le * n * n + i * n + j);
        }
      }
    }
  }

  auto* h = new (std::nothrow) McHandle();
  if (!h) return set_error(FNE_ENOMEM, "Mohr-Coulomb: out of host memory");
  h->precision = d->precision;
  h->hess_fp32 = d->precision == FNE_FP32 && d->hess_fp32;
  h->np = np;
  h->nq = nq;
  h->n = n;
  h->n_local = (int)nl;
  h->n_rows = n_rows;
  h->nnz = d->nnz;
  h->lo = lo;
  h->hi = hi;
  h->n_free = d->n_free;
  h->n_total = d->n_total;
  // constitutive constants (src/problems/slope_stability/jax/jax_energy.py:11-30, 45-108)
  const double Ey = d->s[0], nu = d->s[1], phi = d->s[2] * M_PI / 180.0, coh = d->s[3];
  const double lam = Ey * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = Ey / (2.0 * (1.0 + nu));
  McConst& m = h->mc;
  m.C00 = lam + 2.0 * mu; m.C01 = lam; m.C22 = mu;
  m.S00 = (1.0 - nu * nu) / Ey; m.S01 = -(nu * (1.0 + nu)) / Ey; m.S22 = 1.0 / mu;
  m.alpha = 1.0 + std::sin(phi); m.beta = 1.0 - std::sin(phi); m.kappa = 2.0 * coh * std::cos(phi);
  const double n1 = m.alpha, n2 = -m.beta, dt = m.S00 * m.S00 - m.S01 * m.S01;
  m.z1 = (m.S00 * n1 - m.S01 * n2) / dt;
  m.z2 = (-m.S01 * n1 + m.S00 * n2) / dt;
  m.nz = n1 * m.z1 + n2 * m.z2;
  const double den = std::fabs(m.alpha - m.beta) > 1.0e-14 ? m.alpha - m.beta : 1.0;
  m.s_apex = m.kappa / den;
  m.reg = d->s[4];
  m.elastic_only = d->s[5] != 0.0;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev);
  h->grid_elem = (int)std::max<int64_t>(1, std::min<int64_t>(h->num_sms * 8, (nl + kMcWarps - 1) / kMcWarps));
  h->n_partials = h->grid_elem;
  const size_t rsz = d->precision == FNE_FP32 ? sizeof(float) : sizeof(double);
  int rc = FNE_OK;
#define MC_TRY(x)      \
  do {                 \
    rc = (x);          \
    if (rc) {          \
      mc_destroy(h);   \
      return rc;       \
    }                  \
  } while (0)
  MC_TRY(mc_upload(h, &h->codes, codes.data(), codes.size()));
  MC_TRY(mc_upload(h, &h->geom, geom.data(), geom.size()));
  if (!epsp.empty()) MC_TRY(mc_upload(h, &h->epsp, epsp.data(), epsp.size()));
  MC_TRY(mc_upload(h, &h->wflag, wflag.data(), wflag.size()));
  MC_TRY(mc_upload(h, &h->dhat1, d->e3, (size_t)nq * np));
  MC_TRY(mc_upload(h, &h->dhat2, d->e3 + (size_t)nq * np, (size_t)nq * np));
  MC_TRY(mc_upload(h, &h->qw, d->e3 + (size_t)2 * nq * np, (size_t)nq));
  MC_TRY(mc_upload(h, &h->dir, d->dirichlet, (size_t)d->n_total));
  if (d->rhs_owned) MC_TRY(mc_upload(h, &h->rhs, d->rhs_owned, (size_t)n_owned));
  MC_TRY(mc_upload(h, &h->partials, (const double*)nullptr, (size_t)h->n_partials));
  MC_TRY(mc_upload(h, &h->counter, (const unsigned*)nullptr, 1));
  if (cudaMemset(h->counter, 0, sizeof(unsigned)) != cudaSuccess) {
    mc_destroy(h);
    return set_error(FNE_ECUDA, "Mohr-Coulomb: cudaMemset");
  }
  MC_TRY(mc_upload(h, &h->hptr, hptr.data(), hptr.size()));
  MC_TRY(mc_upload(h, &h->hidx, hidx.data(), hidx.size()));
  MC_TRY(mc_upload(h, &h->gptr, gptr.data(), gptr.size()));
  MC_TRY(mc_upload(h, &h->gidx, gidx.data(), gidx.size()));
  MC_TRY(mc_upload(h, &h->row_gpos, row_gpos.data(), row_gpos.size()));
  {
    unsigned char* kb = nullptr;
    MC_TRY(mc_upload(h, &kb, (const unsigned char*)nullptr, (size_t)nl * n * n * rsz));
    h->Kbuf = kb;
    unsigned char* gb = nullptr;
    MC_TRY(mc_upload(h, &gb, (const unsigned char*)nullptr, (size_t)nl * n * rsz));
    h->gbuf = gb;
  }
  h->n_contrib = hptr[d->nnz];
#undef MC_TRY
  *out = h;
  return FNE_OK;
}

int mc_eval(McHandle* h, const double* u, int flags, double* energy, double* grad, void* hess, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (h->precision == FNE_FP64)
    e = mc_dispatch<double, double>(h, flags, u, energy, grad, hess, st);
  else if (h->hess_fp32)
    e = mc_dispatch<float, float>(h, flags, u, energy, grad, hess, st);
  else
    e = mc_dispatch<float, double>(h, flags, u, energy, grad, hess, st);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("Mohr-Coulomb launch: ") + cudaGetErrorString(e));
  return FNE_OK;
}

int mc_set_dirichlet(McHandle* h, const double* dirichlet) {
  if (h->n_total == 0) return FNE_OK;
  cudaError_t e = cudaMemcpy(h->dir, dirichlet, h->n_total * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_set_dirichlet: ") + cudaGetErrorString(e));
  return FNE_OK;
}

void mc_info(const McHandle* h, fne_info* info) {
  info->n_rows = h->n_rows;
  info->nnz = h->nnz;
  info->n_elem = h->n_local;
  info->n_incidences = h->n_contrib;
  info->device_bytes = h->device_bytes;
  info->max_row_len = 0;
  info->kernel_variant = 5;
}

}  // namespace fne
