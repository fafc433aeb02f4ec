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
// element map: B_q = (reference basis gradients at q) x J^-1, so the element
// data is 5 numbers (affine map: J^-1 and |det J|) -- or 5 per quadrature
// point for the isoparametric P2 map (GQ kernels) -- instead of the
// reference's nq x 3 x 2n elem_B.
//
// Three kernels: k_mc_elem (one warp per element: nodal values and basis
// gradients staged in shared memory, one lane per quadrature point for the
// constitutive update, lanes over node pairs for the 2x2 blocks of K), and
// two gathers that sum the element matrices / vectors into the owned COO
// values and the gradient in a fixed order (no atomics, deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fne_gather.cuh"
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
  const double* __restrict__ geom;   // [n_el * 5] J^-1 (4), |det J|; GQ kernels [n_el * nq * 5]
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

// Geometry values per element: 5 (affine map) or 5 per quadrature point (GQ).
template <int NQ, bool GQ>
__host__ __device__ constexpr int geo_stride() { return GQ ? 5 * NQ : 5; }

template <typename Real, int NP, int NQ, int WANT, bool GQ>
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
    const double* gm = A.geom + (long long)geo_stride<NQ, GQ>() * e;
    for (int i = lane; i < N; i += 32) {
      const int code = A.codes[(long long)e * N + i];
      ue[i] = (Real)(code >= 0 ? A.u[code] : A.dir[-1 - code]);
    }
    for (int i = lane; i < NQ * NP; i += 32) {
      const double* g = GQ ? gm + 5 * (i / NP) : gm;
      gx[i] = (Real)g[0] * s_dh1[i] + (Real)g[1] * s_dh2[i];
      gy[i] = (Real)g[2] * s_dh1[i] + (Real)g[3] * s_dh2[i];
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
      const Real w = (Real)gm[GQ ? 5 * q + 4 : 4] * s_w[q];
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
      // node-pair layout: Kbuf[e][pair][c * 2 + d] = K[(a, c), (b, d)], a <= b
      Real* Ke = Kbuf + (long long)e * NPAIR * 4;
#pragma unroll
      for (int k = 0; k < PPL; ++k) {
        if (lane + 32 * k < NPAIR) {
          Real* o = Ke + 4 * (lane + 32 * k);
          o[0] = kacc[k][0];
          o[1] = kacc[k][1];
          o[2] = kacc[k][2];
          o[3] = kacc[k][3];
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

// ---------------------------------------------------------------------------
// Matrix-free Hessian products (the reference's matrix_free_mult /
// matrix_free_get_diagonal, slope_stability/jax_petsc/
// reordered_element_assembler.py:335-562).  k_mc_lin stores, at the
// linearization point u, the weighted consistent tangent w_q C_q (upper
// triangle, 6 values) of every quadrature point; k_mc_hvp then evaluates per
// element y_e = sum_q B_q^T (w_q C_q) (B_q x_e) -- or, for the diagonal,
// d_(a,c) = sum_q B_q[:,(a,c)]^T (w_q C_q) B_q[:,(a,c)] -- without forming
// K_e; the element vectors are summed per owned row by k_rowgrad.  One warp
// per element, one lane per quadrature point, then one lane per element DOF.
// ---------------------------------------------------------------------------
template <typename Real, int NP, int NQ, bool GQ>
__global__ void __launch_bounds__(32 * kMcWarps) k_mc_lin(McArgs A, McConstR<Real> M, Real* __restrict__ wct) {
  constexpr int N = 2 * NP;
  __shared__ Real s_dh1[NQ * NP], s_dh2[NQ * NP], s_w[NQ];
  __shared__ Real s_u[kMcWarps][N];
  for (int i = threadIdx.x; i < NQ * NP; i += blockDim.x) {
    s_dh1[i] = (Real)A.dhat1[i];
    s_dh2[i] = (Real)A.dhat2[i];
  }
  for (int i = threadIdx.x; i < NQ; i += blockDim.x) s_w[i] = (Real)A.qw[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Real* ue = s_u[wid];
  for (int e = blockIdx.x * kMcWarps + wid; e < A.n_el; e += gridDim.x * kMcWarps) {
    for (int i = lane; i < N; i += 32) {
      const int code = A.codes[(long long)e * N + i];
      ue[i] = (Real)(code >= 0 ? A.u[code] : A.dir[-1 - code]);
    }
    __syncwarp();
    if (lane < NQ) {
      const int q = lane;
      const double* gm = A.geom + (long long)geo_stride<NQ, GQ>() * e + (GQ ? 5 * q : 0);
      const Real i00 = (Real)gm[0], i01 = (Real)gm[1], i10 = (Real)gm[2], i11 = (Real)gm[3], dj = (Real)gm[4];
      Real ex = Real(0), ey = Real(0), exy = Real(0);
      for (int a = 0; a < NP; ++a) {
        const Real r1 = s_dh1[q * NP + a], r2 = s_dh2[q * NP + a];
        const Real px = i00 * r1 + i01 * r2, py = i10 * r1 + i11 * r2;
        ex += px * ue[2 * a];
        ey += py * ue[2 * a + 1];
        exy += py * ue[2 * a] + px * ue[2 * a + 1];
      }
      Real eps[3] = {ex, ey, exy};
      if (A.epsp) {
        const double* ep = A.epsp + ((long long)e * NQ + q) * 3;
        eps[0] -= (Real)ep[0];
        eps[1] -= (Real)ep[1];
        eps[2] -= (Real)ep[2];
      }
      Real sig[3], Ct[6], psi;
      mc_point(M, eps, sig, Ct, psi);
      const Real w = dj * s_w[q];
      Real* o = wct + ((long long)e * NQ + q) * 6;
#pragma unroll
      for (int k = 0; k < 6; ++k) o[k] = w * Ct[k];
    }
    __syncwarp();
  }
}

template <typename Real, int NP, int NQ, bool DIAG, bool GQ>
__global__ void __launch_bounds__(32 * kMcWarps) k_mc_hvp(McArgs A, const Real* __restrict__ wct,
                                                          Real* __restrict__ ebuf) {
  constexpr int N = 2 * NP;
  __shared__ Real s_dh1[NQ * NP], s_dh2[NQ * NP];
  __shared__ Real s_x[kMcWarps][N];
  __shared__ Real s_s[kMcWarps][NQ * 4];
  for (int i = threadIdx.x; i < NQ * NP; i += blockDim.x) {
    s_dh1[i] = (Real)A.dhat1[i];
    s_dh2[i] = (Real)A.dhat2[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Real* xe = s_x[wid];
  Real* ss = s_s[wid];
  for (int e = blockIdx.x * kMcWarps + wid; e < A.n_el; e += gridDim.x * kMcWarps) {
    const double* gm = A.geom + (long long)geo_stride<NQ, GQ>() * e;
    const Real* wc = wct + (long long)e * NQ * 6;
    if (!DIAG) {
      // tangent direction: free DOFs from x, Dirichlet DOFs zero
      for (int i = lane; i < N; i += 32) {
        const int code = A.codes[(long long)e * N + i];
        xe[i] = code >= 0 ? (Real)A.u[code] : Real(0);
      }
      __syncwarp();
      if (lane < NQ) {
        // reference-gradient contraction z[d][l] = sum_b R_qbl x_(b,d); strain
        // B_q x_e = J^-T-weighted z; s = (w C_q) strain; pulled back
        // t[c][l] = sum_i J^-1_il s[v(c,i)], so that y_(a,c) = sum_q sum_l R_qal t[c][l]
        const int q = lane;
        const double* gq = gm + (GQ ? 5 * q : 0);
        const Real i00 = (Real)gq[0], i01 = (Real)gq[1], i10 = (Real)gq[2], i11 = (Real)gq[3];
        Real z01 = Real(0), z02 = Real(0), z11 = Real(0), z12 = Real(0);
        for (int a = 0; a < NP; ++a) {
          const Real r1 = s_dh1[q * NP + a], r2 = s_dh2[q * NP + a];
          const Real x0 = xe[2 * a], x1 = xe[2 * a + 1];
          z01 += r1 * x0;
          z02 += r2 * x0;
          z11 += r1 * x1;
          z12 += r2 * x1;
        }
        const Real ex = i00 * z01 + i01 * z02, ey = i10 * z11 + i11 * z12;
        const Real exy = i10 * z01 + i11 * z02 + i00 * z11 + i01 * z12;
        const Real* C = wc + q * 6;
        const Real s0 = C[0] * ex + C[1] * ey + C[2] * exy;
        const Real s1 = C[1] * ex + C[3] * ey + C[4] * exy;
        const Real s2 = C[2] * ex + C[4] * ey + C[5] * exy;
        ss[q * 4 + 0] = i00 * s0 + i10 * s2;  // c = 0, l = 1
        ss[q * 4 + 1] = i01 * s0 + i11 * s2;  // c = 0, l = 2
        ss[q * 4 + 2] = i10 * s1 + i00 * s2;  // c = 1, l = 1
        ss[q * 4 + 3] = i11 * s1 + i01 * s2;  // c = 1, l = 2
      }
      __syncwarp();
    }
    for (int i = lane; i < N; i += 32) {
      const int a = i >> 1, c = i & 1;
      Real acc = Real(0);
      for (int q = 0; q < NQ; ++q) {
        const Real r1 = s_dh1[q * NP + a], r2 = s_dh2[q * NP + a];
        if (DIAG) {
          // B column (a, c): c = 0 -> (px, 0, py); c = 1 -> (0, py, px)
          const double* gq = gm + (GQ ? 5 * q : 0);
          const Real px = (Real)gq[0] * r1 + (Real)gq[1] * r2, py = (Real)gq[2] * r1 + (Real)gq[3] * r2;
          const Real* C = wc + q * 6;
          acc += c == 0 ? px * (C[0] * px + C[2] * py) + py * (C[2] * px + C[5] * py)
                        : py * (C[3] * py + C[4] * px) + px * (C[4] * py + C[5] * px);
        } else {
          acc += r1 * ss[q * 4 + 2 * c] + r2 * ss[q * 4 + 2 * c + 1];
        }
      }
      ebuf[(long long)e * N + i] = acc;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Tensor-core element kernel (FP32, P2 / P4): tcgen05.mma, kind::tf32.
//
// For affine triangles the physical basis gradients are g_ai = sum_k J^-1_ik
// R_ak with R the reference gradients at the quadrature point, so
//   K[(a,c),(b,d)] = sum_q sum_{k,l} R_qak R_qbl  At_q[c,k,d,l],
//   At_q[c,k,d,l]  = w_q sum_{i,j} J^-1_ik J^-1_jl Ct_q[v(c,i), v(d,j)],
// (v: Voigt index of the strain component that DOF (c) feeds through the
// derivative in direction i).  Over a tile of TE elements this is one GEMM
//   D[(a,b), (e,c,d)] = P[(a,b), (q,k,l)] . At[(q,k,l), (e,c,d)]
// with a constant A operand P (node pairs a <= b x (q,k,l), built on the host)
// and the per-element B operand At (computed by the CTA from the constitutive
// update).  M = 128 node pairs (120 used for P4, 21 for P2), K = 4 nq padded to
// a multiple of 8, N = 4 TE.  FP32 accuracy from three TF32 products:
// D = P_hi At_hi + P_hi At_lo + P_lo At_hi (hi = top 19 bits, lo = remainder).
// Operands live in shared memory in the no-swizzle K-major core-matrix
// layout (8 rows x 16 bytes per core matrix); the accumulator lives in TMEM
// and is read back with tcgen05.ld into the node-pair layout of Kbuf.
// The element gradient (sum_q B^T w sigma) runs on the CUDA cores while the
// tensor core works.
// ---------------------------------------------------------------------------
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: no swizzle, K-major core matrices.
// lbo: byte distance between the two 16-byte K halves of one MMA step;
// sbo: byte distance between consecutive groups of 8 rows.
__device__ __forceinline__ uint64_t mat_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, absolute LBO mode, no swizzle
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
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

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

}  // namespace tc

// Tile geometry of the tensor-core kernel for (NP, NQ).
template <int NP, int NQ, bool GQ = false>
struct McTile {
  static constexpr int GS = geo_stride<NQ, GQ>();   // geometry values per element
  static constexpr int NPAIR = NP * (NP + 1) / 2;
  static constexpr int KK = 4 * NQ;                 // (q, k, l)
  static constexpr int KP = (KK + 7) / 8 * 8;       // padded to the MMA K step (8 tf32)
  static constexpr int M = 128;                     // node pairs (padded)
  static constexpr int TE = NP > 6 ? 24 : 48;       // elements per tile
  static constexpr int N = 4 * TE;                  // (c, d, e): row (c * 2 + d) * TE + e
  static constexpr int TMEM_COLS = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  static constexpr int THREADS = NP > 6 ? 512 : 256;
  static constexpr int MIN_BLOCKS = NP > 6 ? 1 : 2;
  // shared memory (bytes); operand buffers first (16-byte aligned)
  static constexpr int A_BYTES = M * KP * 4;
  static constexpr int B_BYTES = N * KP * 4;
  static constexpr int OFF_AHI = 0, OFF_ALO = A_BYTES, OFF_BHI = 2 * A_BYTES, OFF_BLO = 2 * A_BYTES + B_BYTES;
  static constexpr int OFF_S = 2 * A_BYTES + 2 * B_BYTES;          // [NQ][TE][4] gradient helper
  static constexpr int OFF_R = OFF_S + TE * NQ * 16;                // dh1, dh2 [NQ * NP], qw [NQ]
  static constexpr int OFF_U = OFF_R + ((2 * NQ * NP + NQ) * 4 + 15) / 16 * 16;  // [TE][2 NP]
  static constexpr int OFF_G = OFF_U + (TE * 2 * NP * 4 + 15) / 16 * 16;          // [TE][GS]
  static constexpr int OFF_PLAN = OFF_G + (TE * GS * 4 + 15) / 16 * 16;           // [TE][NP * NP] uint16 codes
  static constexpr int PLAN_WORDS = (TE * NP * NP + 1) / 2;                       // as uint32 words
  static constexpr int OFF_ROW = OFF_PLAN + (PLAN_WORDS * 4 + 15) / 16 * 16;      // [TE][NP][2] row starts
  static constexpr int OFF_SB = OFF_ROW + (TE * NP * 2 * 4 + 15) / 16 * 16;       // [TE] shared-slot bases
  static constexpr int OFF_BAR = OFF_SB + (TE * 4 + 15) / 16 * 16;                // mbarrier, tmem addr, flags
  static constexpr int SMEM = OFF_BAR + 64;
};

// try_wait polls before the kernel gives up on an MMA completion (each poll
// may itself suspend briefly): far above any tile's MMA time, still bounded.
constexpr long long kMcWaitLimit = 1LL << 22;

struct McTcArgs {
  const float* Phi;  // [KP/4][M][4] constant operand, hi part (core-matrix order)
  const float* Plo;  // same, lo part
  int* err;          // device status word (0 = ok; 1 = MMA completion wait timed out)
  long long wait_limit;  // polls of each tile's MMA-completion wait (kMcWaitLimit unless a test lowers it)
  // direct-write epilogue (DirectPlan): per element and directed node pair a
  // 16-bit code, shared-slot base, row node of every element node, COO start
  // of every row (row node, component), and the shared-block buffer
  const uint16_t* code;
  const int* sbase;
  const int* elem_rn;
  const int* rn_row;
  float* sbuf;
};

template <int NP, int NQ, int WANT, typename HOut, bool GQ>
__global__ void __launch_bounds__(McTile<NP, NQ, GQ>::THREADS, McTile<NP, NQ, GQ>::MIN_BLOCKS)
    k_mc_tc(McArgs A, McConstR<float> C, McTcArgs T, HOut* __restrict__ hout, float* __restrict__ gbuf,
            double* __restrict__ partials, unsigned* __restrict__ counter, double* __restrict__ eout) {
  using G = McTile<NP, NQ, GQ>;
  constexpr int N2 = 2 * NP, TE = G::TE, N = G::N, M = G::M, KP = G::KP, NPAIR = G::NPAIR, NT = G::THREADS;
  constexpr int GS = G::GS;
  constexpr int UPT = (TE * N2 + NT - 1) / NT;  // nodal values per thread (prefetch)
  constexpr int GPT = (TE * GS + NT - 1) / NT;  // geometry values per thread (prefetch)
  extern __shared__ __align__(1024) unsigned char smem[];
  float* sAhi = reinterpret_cast<float*>(smem + G::OFF_AHI);
  float* sAlo = reinterpret_cast<float*>(smem + G::OFF_ALO);
  float* sBhi = reinterpret_cast<float*>(smem + G::OFF_BHI);
  float* sBlo = reinterpret_cast<float*>(smem + G::OFF_BLO);
  float4* sS = reinterpret_cast<float4*>(smem + G::OFF_S);  // [NQ][TE]
  float* sD1 = reinterpret_cast<float*>(smem + G::OFF_R);
  float* sD2 = sD1 + NQ * NP;
  float* sW = sD2 + NQ * NP;
  float* sU = reinterpret_cast<float*>(smem + G::OFF_U);
  float* sGm = reinterpret_cast<float*>(smem + G::OFF_G);
  uint32_t* sPlanW = reinterpret_cast<uint32_t*>(smem + G::OFF_PLAN);
  const uint16_t* sPlan = reinterpret_cast<const uint16_t*>(smem + G::OFF_PLAN);
  int* sRow = reinterpret_cast<int*>(smem + G::OFF_ROW);
  int* sSb = reinterpret_cast<int*>(smem + G::OFF_SB);
  unsigned long long* sBar = reinterpret_cast<unsigned long long*>(smem + G::OFF_BAR);
  uint32_t* sTmem = reinterpret_cast<uint32_t*>(smem + G::OFF_BAR + 8);
  int* sFail = reinterpret_cast<int*>(smem + G::OFF_BAR + 12);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // constant operand and reference tables (once per CTA)
  {
    const float4* ph = reinterpret_cast<const float4*>(T.Phi);
    const float4* pl = reinterpret_cast<const float4*>(T.Plo);
    float4* ah = reinterpret_cast<float4*>(sAhi);
    float4* al = reinterpret_cast<float4*>(sAlo);
    for (int i = tid; i < M * KP / 4; i += NT) {
      ah[i] = ph[i];
      al[i] = pl[i];
    }
    // B padding chunks (k >= KK) stay zero for the whole kernel
    for (int i = tid; i < (KP - G::KK) / 4 * N; i += NT) {
      const int off = (G::KK / 4) * N * 4 + i * 4;
      reinterpret_cast<float4*>(sBhi + off)[0] = make_float4(0.f, 0.f, 0.f, 0.f);
      reinterpret_cast<float4*>(sBlo + off)[0] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    for (int i = tid; i < NQ * NP; i += NT) {
      sD1[i] = (float)A.dhat1[i];
      sD2[i] = (float)A.dhat2[i];
    }
    for (int i = tid; i < NQ; i += NT) sW[i] = (float)A.qw[i];
  }
  const uint32_t bar = tc::smem_u32(sBar);
  if (tid == 0) {
    *sFail = 0;
    tc::mbar_init(bar);
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(sTmem), G::TMEM_COLS);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *sTmem;
  constexpr uint32_t idesc = tc::idesc_tf32(M, N);
  const int n_tiles = (A.n_el + TE - 1) / TE;

  // register prefetch of one tile's gather codes, nodal values and geometry
  constexpr int NN = NP * NP;
  constexpr int RPT = (TE * NP + NT - 1) / NT;              // element nodes per thread (row starts)
  constexpr int WPT = (G::PLAN_WORDS + NT - 1) / NT;       // plan words per thread
  int cv[UPT], rnv[RPT], rsv[RPT][2], sbv = 0;
  uint32_t pw[WPT];
  float uv[UPT], gv[GPT];
  auto fetch_codes = [&](int tile) {
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
      const int i = tid + k * NT, el = i / N2;
      const int e = tile * TE + el;
      cv[k] = (tile < n_tiles && i < TE * N2 && e < A.n_el) ? __ldg(A.codes + (long long)e * N2 + (i - el * N2))
                                                             : INT_MIN;
    }
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      const int i = tid + k * NT, el = i / GS;
      const int e = tile * TE + el;
      gv[k] = (tile < n_tiles && i < TE * GS && e < A.n_el) ? (float)__ldg(A.geom + (long long)tile * TE * GS + i)
                                                            : 0.f;
    }
    if (WANT & MW_H) {
      const int ne_t = tile < n_tiles ? min(TE, A.n_el - tile * TE) : 0;
      const int nw = (ne_t * NN + 1) / 2;
      const uint32_t* cw = reinterpret_cast<const uint32_t*>(T.code) + (long long)tile * TE * NN / 2;
#pragma unroll
      for (int k = 0; k < WPT; ++k) {
        const int i = tid + k * NT;
        pw[k] = i < nw ? __ldg(cw + i) : 0xFFFFFFFFu;
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int i = tid + k * NT;
        rnv[k] = i < ne_t * NP ? __ldg(T.elem_rn + (long long)tile * TE * NP + i) : -1;
      }
      sbv = tid < ne_t ? __ldg(T.sbase + (long long)tile * TE + tid) : 0;
    }
  };
  auto fetch_values = [&]() {
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
      const int c = cv[k];
      uv[k] = c == INT_MIN ? 0.f : (float)(c >= 0 ? __ldg(A.u + c) : __ldg(A.dir + (-1 - c)));
    }
    if (WANT & MW_H) {
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int rn = rnv[k];
        rsv[k][0] = rn >= 0 ? __ldg(T.rn_row + 2LL * rn) : -1;
        rsv[k][1] = rn >= 0 ? __ldg(T.rn_row + 2LL * rn + 1) : -1;
      }
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int k = 0; k < UPT; ++k)
      if (tid + k * NT < TE * N2) sU[tid + k * NT] = uv[k];
#pragma unroll
    for (int k = 0; k < GPT; ++k)
      if (tid + k * NT < TE * GS) sGm[tid + k * NT] = gv[k];
    if (WANT & MW_H) {
#pragma unroll
      for (int k = 0; k < WPT; ++k)
        if (tid + k * NT < G::PLAN_WORDS) sPlanW[tid + k * NT] = pw[k];
#pragma unroll
      for (int k = 0; k < RPT; ++k)
        if (tid + k * NT < TE * NP) {
          sRow[2 * (tid + k * NT)] = rsv[k][0];
          sRow[2 * (tid + k * NT) + 1] = rsv[k][1];
        }
      if (tid < TE) sSb[tid] = sbv;
    }
  };

  double eacc = 0.0;
  uint32_t phase = 0;
  fetch_codes(blockIdx.x);
  fetch_values();
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int e0 = tile * TE;
    const int ne = min(TE, A.n_el - e0);
    // (1) nodal values and element geometry of the tile (prefetched)
    stash();
    __syncthreads();
    // (2) constitutive update per (quadrature point, element) -> At (B operand rows j * TE + el), helper
    for (int p = tid; p < TE * NQ; p += NT) {
      const int q = p / TE, el = p - q * TE;
      float4 at[4];  // (c, d) blocks j = c * 2 + d: [k * 2 + l]
      float4 sg = make_float4(0.f, 0.f, 0.f, 0.f);
      if (el < ne) {
        const float* gm = sGm + el * GS + (GQ ? 5 * q : 0);
        const float i00 = gm[0], i01 = gm[1], i10 = gm[2], i11 = gm[3];
        const float* ue = sU + el * N2;
        float gx1 = 0.f, gx2 = 0.f, gy1 = 0.f, gy2 = 0.f;  // reference-gradient contractions
#pragma unroll 5
        for (int a = 0; a < NP; ++a) {
          const float r1 = sD1[q * NP + a], r2 = sD2[q * NP + a];
          const float ux = ue[2 * a], uy = ue[2 * a + 1];
          gx1 += r1 * ux;
          gx2 += r2 * ux;
          gy1 += r1 * uy;
          gy2 += r2 * uy;
        }
        const float uxx = i00 * gx1 + i01 * gx2, uxy = i10 * gx1 + i11 * gx2;
        const float uyx = i00 * gy1 + i01 * gy2, uyy = i10 * gy1 + i11 * gy2;
        float eps[3] = {uxx, uyy, uxy + uyx};
        if (A.epsp) {
          const double* ep = A.epsp + ((long long)(e0 + el) * NQ + q) * 3;
          eps[0] -= (float)ep[0];
          eps[1] -= (float)ep[1];
          eps[2] -= (float)ep[2];
        }
        float sig[3], Ct[6], psi;
        mc_point(C, eps, sig, Ct, psi);
        const float w = gm[4] * sW[q];
        if ((WANT & MW_E) && A.wflag[e0 + el]) eacc += (double)(w * psi);
        // full symmetric tangent (Voigt 0 = xx, 1 = yy, 2 = xy)
        const float Cf[3][3] = {{Ct[0], Ct[1], Ct[2]}, {Ct[1], Ct[3], Ct[4]}, {Ct[2], Ct[4], Ct[5]}};
        // v(c, i): component c of the DOF, physical derivative direction i
        const int vci[2][2] = {{0, 2}, {2, 1}};
        const float Mx[2][2] = {{i00, i01}, {i10, i11}};  // g_i = sum_k Mx[i][k] R_k
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
          for (int d = 0; d < 2; ++d) {
            float Acd[2][2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) Acd[i][j] = w * Cf[vci[c][i]][vci[d][j]];
            float r[4];
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
              for (int l = 0; l < 2; ++l)
                r[k * 2 + l] = Mx[0][k] * (Acd[0][0] * Mx[0][l] + Acd[0][1] * Mx[1][l]) +
                               Mx[1][k] * (Acd[1][0] * Mx[0][l] + Acd[1][1] * Mx[1][l]);
            at[c * 2 + d] = make_float4(r[0], r[1], r[2], r[3]);
          }
        }
        // gradient helper s[c][k] = w sum_i Mx[i][k] sigma[v(c, i)]
        sg = make_float4(w * (Mx[0][0] * sig[0] + Mx[1][0] * sig[2]), w * (Mx[0][1] * sig[0] + Mx[1][1] * sig[2]),
                         w * (Mx[0][0] * sig[2] + Mx[1][0] * sig[1]), w * (Mx[0][1] * sig[2] + Mx[1][1] * sig[1]));
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) at[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      sS[q * TE + el] = sg;
      // B operand row n = j * TE + el, K chunk q (16 bytes: k * 2 + l); consecutive
      // threads (elements) write consecutive 16-byte rows
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int off = q * N * 4 + (j * TE + el) * 4;
        const float4 v = at[j];
        const float4 hi = make_float4(tc::tf32_hi(v.x), tc::tf32_hi(v.y), tc::tf32_hi(v.z), tc::tf32_hi(v.w));
        reinterpret_cast<float4*>(sBhi + off)[0] = hi;
        reinterpret_cast<float4*>(sBlo + off)[0] = make_float4(v.x - hi.x, v.y - hi.y, v.z - hi.z, v.w - hi.w);
      }
    }
    tc::fence_proxy_async();  // generic-proxy smem writes -> visible to the tensor core
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    // (3) one thread issues the MMAs: 3 TF32 products per K step of 8
    if ((WANT & MW_H) && tid == 0) {
      const uint32_t ahi = tc::smem_u32(sAhi), alo = tc::smem_u32(sAlo);
      const uint32_t bhi = tc::smem_u32(sBhi), blo = tc::smem_u32(sBlo);
#pragma unroll 1
      for (int s = 0; s < KP / 8; ++s) {
        const uint32_t ao = (uint32_t)(s * 2 * M * 16), bo = (uint32_t)(s * 2 * N * 16);
        const uint64_t dAh = tc::mat_desc(ahi + ao, M * 16, 128), dAl = tc::mat_desc(alo + ao, M * 16, 128);
        const uint64_t dBh = tc::mat_desc(bhi + bo, N * 16, 128), dBl = tc::mat_desc(blo + bo, N * 16, 128);
        tc::mma_tf32(tmem, dAh, dBh, idesc, s > 0 ? 1u : 0u);
        tc::mma_tf32(tmem, dAh, dBl, idesc, 1u);
        tc::mma_tf32(tmem, dAl, dBh, idesc, 1u);
      }
      tc::commit(bar);
    }
    // next tile's gather codes and geometry in flight during the gradient / epilogue
    fetch_codes(tile + gridDim.x);
    // (4) element gradient on the CUDA cores while the MMAs run
    if (WANT & MW_G) {
      for (int i = tid; i < TE * N2; i += NT) {
        const int el = i / N2, r = i - el * N2, a = r >> 1, c = r & 1;
        if (el >= ne) continue;
        float acc = 0.f;
#pragma unroll 5
        for (int q = 0; q < NQ; ++q) {
          const float4 s = sS[q * TE + el];
          const float r1 = sD1[q * NP + a], r2 = sD2[q * NP + a];
          acc += c == 0 ? r1 * s.x + r2 * s.y : r1 * s.z + r2 * s.w;
        }
        gbuf[(long long)(e0 + el) * N2 + r] = acc;
      }
    }
    fetch_values();
    // (5) epilogue: TMEM -> Kbuf[e][pair][c * 2 + d]; warp w reads lanes 32 (w % 4) ..
    // (node pairs) for its share of the tile's elements
    if (WANT & MW_H) {
      if (tc::mbar_wait(bar, phase, T.wait_limit))
        phase ^= 1u;
      else if (lane == 0)
        atomicExch(sFail, 1);
      tc::fence_after();
      constexpr int NGRP = NT / 128, EPG = TE / NGRP;  // element groups, elements per group
      const int quad = warp & 3, grp = warp >> 2;
      const int m = quad * 32 + lane;
      // node pair of this lane: m -> (pa, pb), pa <= pb
      int pa = 0, pb = m;
      while (pa < NP && pb >= NP - pa) {
        pb -= NP - pa;
        ++pa;
      }
      pb += pa;
      // one directed block (ra -> cb) of element el: straight into the COO rows,
      // or into the shared-block buffer
      auto put = [&](int el, int ra, int cb, float w00, float w01, float w10, float w11) {
        const unsigned code = sPlan[el * NN + ra * NP + cb];
        if (code == 0xFFFFu) return;
        if (code & 0x8000u) {
          reinterpret_cast<float4*>(T.sbuf)[(long long)sSb[el] + (code & 0x7FFFu)] = make_float4(w00, w01, w10, w11);
          return;
        }
        const int off = (int)(code & 0xFFFu);
        const unsigned dm = (code >> 12) & 3u;
        const float w[2][2] = {{w00, w01}, {w10, w11}};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int rs = sRow[(el * NP + ra) * 2 + c];
          if (rs < 0) continue;
          int k = 0;
#pragma unroll
          for (int d = 0; d < 2; ++d)
            if ((dm >> d) & 1u) hout[rs + off + k++] = (HOut)w[c][d];
        }
      };
      if (!*sFail && quad * 32 < NPAIR) {
#pragma unroll 1
        for (int el = grp * EPG; el < (grp + 1) * EPG; el += 2) {
          uint32_t r[4][2];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const uint32_t ta = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(j * TE + el);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                         : "=r"(r[j][0]), "=r"(r[j][1])
                         : "r"(ta)
                         : "memory");
          }
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (m < NPAIR) {
#pragma unroll
            for (int x = 0; x < 2; ++x)
              if (el + x < ne) {
                const float v0 = __uint_as_float(r[0][x]), v1 = __uint_as_float(r[1][x]);
                const float v2 = __uint_as_float(r[2][x]), v3 = __uint_as_float(r[3][x]);
                put(el + x, pa, pb, v0, v1, v2, v3);                // K[(a,c),(b,d)], (c,d) row-major
                if (pa != pb) put(el + x, pb, pa, v0, v2, v1, v3);  // transposed block (b, a)
              }
          }
        }
      }
      tc::fence_before();
    }
    __syncthreads();
    if (*sFail) break;
  }
  if (*sFail && tid == 0) {
    // one more bounded wait so no MMA is in flight when TMEM is released
    tc::mbar_wait(bar, phase, kMcWaitLimit);
    atomicExch(T.err, 1);
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0) tc::tmem_dealloc(tmem, G::TMEM_COLS);
  if (WANT & MW_E) {
    if (A.rhs)
      for (int i = blockIdx.x * NT + threadIdx.x; i < A.n_owned; i += gridDim.x * NT)
        eacc -= A.rhs[i] * A.u[A.lo + i];
    mc_energy_finalize(eacc, partials, counter, eout);
  }
}

// ---------------------------------------------------------------------------
// Energy and / or gradient without the Hessian (the line-search and gradient
// callbacks): tiles of 32 elements; the tile's gathered nodal values and
// geometry are staged in shared memory, then threads run over (quadrature
// point, element): strain from the reference tables and J^-1, return map
// (the tangent it would also form is not used and is compiled out), energy
// density, and for the gradient the pulled-back helper s[c][k] =
// w sum_i J^-1_ik sigma[v(c, i)]; the element gradient g_(a,c) = sum_q R_qak
// s_q[c][k] follows per (element, DOF).
// ---------------------------------------------------------------------------
constexpr int kEgTile = 32, kEgThreads = 256;

template <typename Real, int NP, int NQ, int WANT, bool GQ>
__global__ void __launch_bounds__(kEgThreads) k_mc_eg(McArgs A, McConstR<Real> M, Real* __restrict__ gbuf,
                                                      double* __restrict__ partials, unsigned* __restrict__ counter,
                                                      double* __restrict__ eout) {
  constexpr int TE = kEgTile, N2 = 2 * NP, NT = kEgThreads;
  constexpr int US = N2 + 1;  // odd row stride of the staged nodal values: no bank conflicts
  __shared__ Real sD1[NQ * NP], sD2[NQ * NP], sW[NQ];
  __shared__ Real sU[TE * US];
  constexpr int GS = geo_stride<NQ, GQ>();
  __shared__ Real sGm[TE * GS];
  __shared__ Real sS[(WANT & MW_G) ? NQ * TE * 4 : 1];
  const int tid = threadIdx.x;
  for (int i = tid; i < NQ * NP; i += NT) {
    sD1[i] = (Real)A.dhat1[i];
    sD2[i] = (Real)A.dhat2[i];
  }
  for (int i = tid; i < NQ; i += NT) sW[i] = (Real)A.qw[i];
  double eacc = 0.0;
  const int n_tiles = (A.n_el + TE - 1) / TE;
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int e0 = tile * TE;
    const int ne = min(TE, A.n_el - e0);
    __syncthreads();  // previous tile's readers are done (and the tables are loaded)
    for (int i = tid; i < ne * N2; i += NT) {
      const int code = __ldg(A.codes + (long long)e0 * N2 + i);
      sU[(i / N2) * US + i % N2] = (Real)(code >= 0 ? __ldg(A.u + code) : __ldg(A.dir + (-1 - code)));
    }
    for (int i = tid; i < ne * GS; i += NT) sGm[i] = (Real)__ldg(A.geom + (long long)e0 * GS + i);
    __syncthreads();
    for (int p = tid; p < TE * NQ; p += NT) {
      const int q = p / TE, el = p - q * TE;
      if (el >= ne) continue;
      const Real* gm = sGm + el * GS + (GQ ? 5 * q : 0);
      const Real i00 = gm[0], i01 = gm[1], i10 = gm[2], i11 = gm[3];
      const Real* ue = sU + el * US;
      // reference-gradient contractions first (4 multiply-adds per node),
      // then J^-1: grad u = [[i00 Gx1 + i01 Gx2, ...]]
      Real gx1 = Real(0), gx2 = Real(0), gy1 = Real(0), gy2 = Real(0);
#pragma unroll 5
      for (int a = 0; a < NP; ++a) {
        const Real r1 = sD1[q * NP + a], r2 = sD2[q * NP + a];
        const Real ux = ue[2 * a], uy = ue[2 * a + 1];
        gx1 += r1 * ux;
        gx2 += r2 * ux;
        gy1 += r1 * uy;
        gy2 += r2 * uy;
      }
      const Real uxx = i00 * gx1 + i01 * gx2, uxy = i10 * gx1 + i11 * gx2;  // d ux / dx, d ux / dy
      const Real uyx = i00 * gy1 + i01 * gy2, uyy = i10 * gy1 + i11 * gy2;  // d uy / dx, d uy / dy
      Real eps[3] = {uxx, uyy, uxy + uyx};
      if (A.epsp) {
        const double* ep = A.epsp + ((long long)(e0 + el) * NQ + q) * 3;
        eps[0] -= (Real)ep[0];
        eps[1] -= (Real)ep[1];
        eps[2] -= (Real)ep[2];
      }
      Real sig[3], Ct[6], psi;
      mc_point(M, eps, sig, Ct, psi);
      const Real w = gm[4] * sW[q];
      if ((WANT & MW_E) && A.wflag[e0 + el]) eacc += (double)(w * psi);
      if (WANT & MW_G) {
        Real* sg = sS + (q * TE + el) * 4;
        sg[0] = w * (i00 * sig[0] + i10 * sig[2]);
        sg[1] = w * (i01 * sig[0] + i11 * sig[2]);
        sg[2] = w * (i00 * sig[2] + i10 * sig[1]);
        sg[3] = w * (i01 * sig[2] + i11 * sig[1]);
      }
    }
    if (WANT & MW_G) {
      __syncthreads();
      for (int i = tid; i < ne * N2; i += NT) {
        const int el = i / N2, r = i - el * N2, a = r >> 1, c = r & 1;
        Real acc = Real(0);
#pragma unroll 5
        for (int q = 0; q < NQ; ++q) {
          const Real* sg = sS + (q * TE + el) * 4 + 2 * c;
          acc += sD1[q * NP + a] * sg[0] + sD2[q * NP + a] * sg[1];
        }
        gbuf[(long long)(e0 + el) * N2 + r] = acc;
      }
    }
  }
  if (WANT & MW_E) {
    if (A.rhs)
      for (int i = blockIdx.x * NT + threadIdx.x; i < A.n_owned; i += gridDim.x * NT)
        eacc -= A.rhs[i] * A.u[A.lo + i];
    mc_energy_finalize(eacc, partials, counter, eout);
  }
}

// ---------------------------------------------------------------------------
// FP64 P2 / P4: the same contraction K[(a,b),(c,d,e)] = P[(a,b),(q,k,l)] ·
// Ã[(q,k,l),(c,d,e)] as the tensor-core kernel, in FP64 on the DMMA units
// (mma.sync m16n8k4 f64) with the direct-write epilogue straight from the
// accumulator registers.  One MMA K step of 4 is one quadrature point, and
// P[(a,b),(q,k,l)] = R_qak R_qbl, so the A fragments are formed from the
// reference gradient tables in registers (no P in shared memory).  Each
// tile of TE elements: return map per (quadrature point, element) -> Ã and
// the gradient helper in shared memory; warp task (16 node pairs,
// 8 elements) runs NQ MMA steps of four n8 tiles (one per (c, d) component)
// and writes its blocks; the element gradient follows on the CUDA cores.
// Two CTAs per SM, so one CTA's return map overlaps the other's MMAs.
// ---------------------------------------------------------------------------
template <int NP, int NQ, bool GQ = false>
struct McTileD {
  static constexpr int GS = geo_stride<NQ, GQ>();        // geometry values per element
  static constexpr int NPAIR = NP * (NP + 1) / 2;
  static constexpr int MT = (NPAIR + 15) / 16;          // m16 tiles of node pairs
  static constexpr int KK = 4 * NQ;                      // (q, k, l)
  static constexpr int TE = 16;                          // elements per tile
  static constexpr int N = 4 * TE;                       // column (c * 2 + d) * TE + e
  static constexpr int NS = N + 4;                       // B row stride (doubles), = 4 (mod 16)
  static constexpr int THREADS = 256;
  static constexpr int MIN_BLOCKS = 2;
  static constexpr int NWARPS = THREADS / 32;
  static constexpr int NTASK = MT * 2;                   // (m16 tile, element half)
  static constexpr int R16(int b) { return (b + 15) / 16 * 16; }
  static constexpr int OFF_B = 0;
  static constexpr int OFF_S = OFF_B + R16(KK * NS * 8);             // [NQ][TE] 4 doubles
  static constexpr int OFF_R = OFF_S + NQ * TE * 32;                 // dh1, dh2 [NQ * NP], qw [NQ]
  static constexpr int OFF_U = OFF_R + R16((2 * NQ * NP + NQ) * 8);  // [TE][2 NP]
  static constexpr int OFF_G = OFF_U + R16(TE * 2 * NP * 8);         // [TE][GS]
  static constexpr int OFF_PLAN = OFF_G + R16(TE * GS * 8);          // [TE][NP * NP] uint16 codes
  static constexpr int PLAN_WORDS = (TE * NP * NP + 1) / 2;
  static constexpr int OFF_ROW = OFF_PLAN + R16(PLAN_WORDS * 4);     // [TE][NP][2] row starts
  static constexpr int OFF_SB = OFF_ROW + R16(TE * NP * 2 * 4);      // [TE] shared-slot bases
  static constexpr int SMEM = OFF_SB + R16(TE * 4);
};

struct McDmArgs {
  const uint16_t* code;
  const int* sbase;
  const int* elem_rn;
  const int* rn_row;
  double* sbuf;      // shared-block buffer, 4 doubles per slot
  const int* sidx;   // buffer position of each element slot (fix-up order), or null (element order)
};

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, {%0, %1, %2, %3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(b0));
}

template <int NP, int NQ, int WANT, bool GQ>
__global__ void __launch_bounds__(McTileD<NP, NQ, GQ>::THREADS, McTileD<NP, NQ, GQ>::MIN_BLOCKS)
    k_mc_dmma(McArgs A, McConstR<double> C, McDmArgs T, double* __restrict__ hout, double* __restrict__ gbuf,
              double* __restrict__ partials, unsigned* __restrict__ counter, double* __restrict__ eout) {
  using G = McTileD<NP, NQ, GQ>;
  constexpr int N2 = 2 * NP, TE = G::TE, NS = G::NS, NPAIR = G::NPAIR, NT = G::THREADS;
  constexpr int NN = NP * NP, GS = G::GS;
  constexpr int UPT = (TE * N2 + NT - 1) / NT;
  constexpr int GPT = (TE * GS + NT - 1) / NT;
  constexpr int RPT = (TE * NP + NT - 1) / NT;
  constexpr int WPT = (G::PLAN_WORDS + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char smem[];
  double* sB = reinterpret_cast<double*>(smem + G::OFF_B);
  double2* sS = reinterpret_cast<double2*>(smem + G::OFF_S);  // [NQ][TE] x 2 double2
  double* sD1 = reinterpret_cast<double*>(smem + G::OFF_R);
  double* sD2 = sD1 + NQ * NP;
  double* sW = sD2 + NQ * NP;
  double* sU = reinterpret_cast<double*>(smem + G::OFF_U);
  double* sGm = reinterpret_cast<double*>(smem + G::OFF_G);
  uint32_t* sPlanW = reinterpret_cast<uint32_t*>(smem + G::OFF_PLAN);
  const uint16_t* sPlan = reinterpret_cast<const uint16_t*>(smem + G::OFF_PLAN);
  int* sRow = reinterpret_cast<int*>(smem + G::OFF_ROW);
  int* sSb = reinterpret_cast<int*>(smem + G::OFF_SB);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gq = lane >> 2, tq = lane & 3;  // MMA fragment group / thread in group

  for (int i = tid; i < NQ * NP; i += NT) {
    sD1[i] = A.dhat1[i];
    sD2[i] = A.dhat2[i];
  }
  for (int i = tid; i < NQ; i += NT) sW[i] = A.qw[i];
  const int n_tiles = (A.n_el + TE - 1) / TE;

  int cv[UPT], rnv[RPT], rsv[RPT][2], sbv = 0;
  uint32_t pw[WPT];
  double uv[UPT], gv[GPT];
  auto fetch_codes = [&](int tile) {
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
      const int i = tid + k * NT, el = i / N2;
      const int e = tile * TE + el;
      cv[k] = (tile < n_tiles && i < TE * N2 && e < A.n_el) ? __ldg(A.codes + (long long)e * N2 + (i - el * N2))
                                                             : INT_MIN;
    }
#pragma unroll
    for (int k = 0; k < GPT; ++k) {
      const int i = tid + k * NT, el = i / GS;
      const int e = tile * TE + el;
      gv[k] = (tile < n_tiles && i < TE * GS && e < A.n_el) ? __ldg(A.geom + (long long)tile * TE * GS + i) : 0.0;
    }
    const int ne_t = tile < n_tiles ? min(TE, A.n_el - tile * TE) : 0;
    const int nw = (ne_t * NN + 1) / 2;
    const uint32_t* cw = reinterpret_cast<const uint32_t*>(T.code) + (long long)tile * TE * NN / 2;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
      const int i = tid + k * NT;
      pw[k] = i < nw ? __ldg(cw + i) : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int i = tid + k * NT;
      rnv[k] = i < ne_t * NP ? __ldg(T.elem_rn + (long long)tile * TE * NP + i) : -1;
    }
    sbv = tid < ne_t ? __ldg(T.sbase + (long long)tile * TE + tid) : 0;
  };
  auto fetch_values = [&]() {
#pragma unroll
    for (int k = 0; k < UPT; ++k) {
      const int c = cv[k];
      uv[k] = c == INT_MIN ? 0.0 : (c >= 0 ? __ldg(A.u + c) : __ldg(A.dir + (-1 - c)));
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int rn = rnv[k];
      rsv[k][0] = rn >= 0 ? __ldg(T.rn_row + 2LL * rn) : -1;
      rsv[k][1] = rn >= 0 ? __ldg(T.rn_row + 2LL * rn + 1) : -1;
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int k = 0; k < UPT; ++k)
      if (tid + k * NT < TE * N2) sU[tid + k * NT] = uv[k];
#pragma unroll
    for (int k = 0; k < GPT; ++k)
      if (tid + k * NT < TE * GS) sGm[tid + k * NT] = gv[k];
#pragma unroll
    for (int k = 0; k < WPT; ++k)
      if (tid + k * NT < G::PLAN_WORDS) sPlanW[tid + k * NT] = pw[k];
#pragma unroll
    for (int k = 0; k < RPT; ++k)
      if (tid + k * NT < TE * NP) {
        sRow[2 * (tid + k * NT)] = rsv[k][0];
        sRow[2 * (tid + k * NT) + 1] = rsv[k][1];
      }
    if (tid < TE) sSb[tid] = sbv;
  };
  // one directed block (ra -> cb) of element el: into the COO rows or the
  // shared-block buffer
  auto put = [&](int el, int ra, int cb, double w00, double w01, double w10, double w11) {
    const unsigned code = sPlan[el * NN + ra * NP + cb];
    if (code == 0xFFFFu) return;
    if (code & 0x8000u) {
      const int slot = sSb[el] + (int)(code & 0x7FFFu);
      double2* sb = reinterpret_cast<double2*>(T.sbuf) + 2 * (long long)(T.sidx ? __ldg(T.sidx + slot) : slot);
      sb[0] = make_double2(w00, w01);
      sb[1] = make_double2(w10, w11);
      return;
    }
    const int off = (int)(code & 0xFFFu);
    const unsigned dm = (code >> 12) & 3u;
    const double w[2][2] = {{w00, w01}, {w10, w11}};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int rs = sRow[(el * NP + ra) * 2 + c];
      if (rs < 0) continue;
      int k = 0;
#pragma unroll
      for (int d = 0; d < 2; ++d)
        if ((dm >> d) & 1u) hout[rs + off + k++] = w[c][d];
    }
  };

  double eacc = 0.0;
  fetch_codes(blockIdx.x);
  fetch_values();
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int e0 = tile * TE;
    const int ne = min(TE, A.n_el - e0);
    stash();
    __syncthreads();
    // (1) constitutive update per (quadrature point, element) -> Ã (rows
    // q * 4 + k * 2 + l, columns (c * 2 + d) * TE + el) and the gradient helper
    for (int p = tid; p < TE * NQ; p += NT) {
      const int q = p / TE, el = p - q * TE;
      double at[4][4];
      double2 s01 = make_double2(0.0, 0.0), s23 = make_double2(0.0, 0.0);
      if (el < ne) {
        const double* gm = sGm + el * GS + (GQ ? 5 * q : 0);
        const double i00 = gm[0], i01 = gm[1], i10 = gm[2], i11 = gm[3];
        const double* ue = sU + el * N2;
        double gx1 = 0.0, gx2 = 0.0, gy1 = 0.0, gy2 = 0.0;  // reference-gradient contractions
#pragma unroll 5
        for (int a = 0; a < NP; ++a) {
          const double r1 = sD1[q * NP + a], r2 = sD2[q * NP + a];
          const double ux = ue[2 * a], uy = ue[2 * a + 1];
          gx1 += r1 * ux;
          gx2 += r2 * ux;
          gy1 += r1 * uy;
          gy2 += r2 * uy;
        }
        const double uxx = i00 * gx1 + i01 * gx2, uxy = i10 * gx1 + i11 * gx2;
        const double uyx = i00 * gy1 + i01 * gy2, uyy = i10 * gy1 + i11 * gy2;
        double eps[3] = {uxx, uyy, uxy + uyx};
        if (A.epsp) {
          const double* ep = A.epsp + ((long long)(e0 + el) * NQ + q) * 3;
          eps[0] -= ep[0];
          eps[1] -= ep[1];
          eps[2] -= ep[2];
        }
        double sig[3], Ct[6], psi;
        mc_point(C, eps, sig, Ct, psi);
        const double w = gm[4] * sW[q];
        if ((WANT & MW_E) && A.wflag[e0 + el]) eacc += w * psi;
        const double Cf[3][3] = {{Ct[0], Ct[1], Ct[2]}, {Ct[1], Ct[3], Ct[4]}, {Ct[2], Ct[4], Ct[5]}};
        const int vci[2][2] = {{0, 2}, {2, 1}};
        const double Mx[2][2] = {{i00, i01}, {i10, i11}};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
#pragma unroll
          for (int d = 0; d < 2; ++d) {
            double Acd[2][2];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int j = 0; j < 2; ++j) Acd[i][j] = w * Cf[vci[c][i]][vci[d][j]];
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
              for (int l = 0; l < 2; ++l)
                at[c * 2 + d][k * 2 + l] = Mx[0][k] * (Acd[0][0] * Mx[0][l] + Acd[0][1] * Mx[1][l]) +
                                           Mx[1][k] * (Acd[1][0] * Mx[0][l] + Acd[1][1] * Mx[1][l]);
          }
        }
        s01 = make_double2(w * (Mx[0][0] * sig[0] + Mx[1][0] * sig[2]), w * (Mx[0][1] * sig[0] + Mx[1][1] * sig[2]));
        s23 = make_double2(w * (Mx[0][0] * sig[2] + Mx[1][0] * sig[1]), w * (Mx[0][1] * sig[2] + Mx[1][1] * sig[1]));
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int kl = 0; kl < 4; ++kl) at[j][kl] = 0.0;
      }
      sS[2 * (q * TE + el)] = s01;
      sS[2 * (q * TE + el) + 1] = s23;
#pragma unroll
      for (int kl = 0; kl < 4; ++kl)
#pragma unroll
        for (int j = 0; j < 4; ++j) sB[(q * 4 + kl) * NS + j * TE + el] = at[j][kl];
    }
    __syncthreads();
    // next tile's gather codes and geometry in flight during the MMAs
    fetch_codes(tile + gridDim.x);
    // (2) warp task (16 node pairs, 8 elements): NQ steps of four m16n8k4
    // MMAs (one n8 tile per (c, d) component), then the blocks from registers
    for (int task = warp; task < G::NTASK; task += G::NWARPS) {
      const int mt = task >> 1, hf = task & 1;
      // node pairs of this lane's fragment rows (pairs beyond NPAIR compute
      // with pair 0 and are not stored)
      int pa_[2], pb_[2];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int m = mt * 16 + gq + 8 * r;
        int a = 0, b = m < NPAIR ? m : 0;
        while (a < NP && b >= NP - a) {
          b -= NP - a;
          ++a;
        }
        pa_[r] = a;
        pb_[r] = a + b;
      }
      // A fragment (row m, column q * 4 + tq): R_q[pa][k] * R_q[pb][l], k = tq / 2, l = tq % 2
      const double* ra0 = ((tq >> 1) ? sD2 : sD1) + pa_[0];
      const double* rb0 = ((tq & 1) ? sD2 : sD1) + pb_[0];
      const double* ra1 = ((tq >> 1) ? sD2 : sD1) + pa_[1];
      const double* rb1 = ((tq & 1) ? sD2 : sD1) + pb_[1];
      double acc[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[j][r] = 0.0;
      const double* pb = sB + tq * NS + hf * 8 + gq;
#pragma unroll 5
      for (int q = 0; q < NQ; ++q) {
        const double a0 = ra0[q * NP] * rb0[q * NP], a1 = ra1[q * NP] * rb1[q * NP];
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[j], a0, a1, pb[q * 4 * NS + j * TE]);
      }
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int m = mt * 16 + gq + 8 * r;
        if (m >= NPAIR) continue;
#pragma unroll
        for (int x = 0; x < 2; ++x) {
          const int el = hf * 8 + 2 * tq + x;
          if (el >= ne) continue;
          const double v0 = acc[0][2 * r + x], v1 = acc[1][2 * r + x];
          const double v2 = acc[2][2 * r + x], v3 = acc[3][2 * r + x];
          put(el, pa_[r], pb_[r], v0, v1, v2, v3);                      // K[(a,c),(b,d)], (c,d) row-major
          if (pa_[r] != pb_[r]) put(el, pb_[r], pa_[r], v0, v2, v1, v3);  // transposed block (b, a)
        }
      }
    }
    // (3) element gradient
    if (WANT & MW_G) {
      for (int i = tid; i < TE * N2; i += NT) {
        const int el = i / N2, r = i - el * N2, a = r >> 1, c = r & 1;
        if (el >= ne) continue;
        double acc = 0.0;
#pragma unroll 5
        for (int q = 0; q < NQ; ++q) {
          const double2 s = sS[2 * (q * TE + el) + c];
          acc += sD1[q * NP + a] * s.x + sD2[q * NP + a] * s.y;
        }
        gbuf[(long long)(e0 + el) * N2 + r] = acc;
      }
    }
    fetch_values();
    __syncthreads();
  }
  if (WANT & MW_E) {
    if (A.rhs)
      for (int i = blockIdx.x * NT + threadIdx.x; i < A.n_owned; i += gridDim.x * NT)
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
  // node-block gather (default) or per-position contribution lists
  int use_blk = 0, n_rnodes = 0;
  int *bp_rn_blk = nullptr, *bp_rn_con = nullptr, *bp_rn_row = nullptr, *bp_rn_gpos = nullptr,
      *bp_rn_inc = nullptr, *bp_con = nullptr, *bp_inc = nullptr;
  unsigned* bp_blk = nullptr;
  // tensor-core path (FP32, P2 / P4): constant operand halves, status word
  int gq = 0;  // 1: geometry per quadrature point (isoparametric P2), 5 * nq values per element
  int tc = 0, grid_tc = 1;
  float *Phi = nullptr, *Plo = nullptr;
  int* err = nullptr;
  int* err_host = nullptr;               // pinned copy of *err after each tensor-core pass
  long long wait_limit = kMcWaitLimit;   // MMA-completion wait bound of the tensor-core kernel
  // direct-write epilogue: per-element codes, shared-block buffer and the
  // fix-up plan over the shared blocks
  uint16_t* dp_code = nullptr;
  int *dp_sbase = nullptr, *dp_elem_rn = nullptr, *dp_sidx = nullptr;
  void* dp_sbuf = nullptr;  // 4 floats (tensor-core path) or 4 doubles (DMMA path) per slot
  // FP64 DMMA path (P2 / P4)
  int dm = 0, grid_dm = 1;
  // tiled energy / gradient kernel for the calls without the Hessian
  int use_eg = 0, grid_eg = 1;
  int n_fix = 0;
  int *fx_con = nullptr, *fx_desc = nullptr;
  // matrix-free products: weighted tangents at the linearization point and
  // the element vectors (allocated by the first fne_hvp_prepare)
  void *lin_wct = nullptr, *lin_ebuf = nullptr;
  int lin_ready = 0;
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

// Hessian / gradient gathers after the element kernel (checks its launch first).
template <typename Real, typename HOut, int NP>
cudaError_t mc_gathers(McHandle* h, int flags, const Real* K, const Real* g, double* grad, void* hess,
                       cudaStream_t st) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (h->use_blk) {
    if (h->n_rnodes == 0) return cudaSuccess;
    HOut* H = static_cast<HOut*>(hess);
    if (flags & MW_H) {
      if (h->tc || h->dm) {  // direct-write epilogue: only the shared blocks remain
        if (h->n_fix > 0) {
          const int gf = std::max(1, std::min(h->num_sms * 16, (h->n_fix + 255) / 256));
          if (h->dm)
            k_fixup2<HOut, double><<<gf, 256, 0, st>>>(h->n_fix, reinterpret_cast<const int4*>(h->fx_desc),
                                                       h->dp_sidx ? nullptr : h->fx_con,
                                                       static_cast<const double*>(h->dp_sbuf), H);
          else
            k_fixup2<HOut, float><<<gf, 256, 0, st>>>(h->n_fix, reinterpret_cast<const int4*>(h->fx_desc),
                                                      h->fx_con, static_cast<const float*>(h->dp_sbuf), H);
        }
      } else {
        NodeGatherArgs G{h->n_rnodes, h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row, h->bp_rn_gpos,
                         h->bp_rn_inc, h->bp_blk, h->bp_con, h->bp_inc, h->rhs};
        const int grid = std::max(1, std::min(h->num_sms * 16, (h->n_rnodes + 7) / 8));
        k_node_gather<Real, HOut, 2, NP, true, false><<<grid, 256, 0, st>>>(G, K, g, H, grad);
      }
    }
    if (flags & MW_G) {
      const int gr = std::max(1, std::min(h->num_sms * 8, (h->n_rnodes + 255) / 256));
      k_rowgrad<Real, 2><<<gr, 256, 0, st>>>(h->n_rnodes, h->bp_rn_inc, h->bp_inc, h->bp_rn_gpos, g, h->rhs, grad);
    }
    return cudaGetLastError();
  }
  const int gg = std::max(1, std::min(h->num_sms * 16, (int)((std::max<int64_t>(h->nnz, h->n_rows) + 255) / 256)));
  if ((flags & MW_H) && h->nnz > 0)
    k_mc_gather<Real, HOut><<<gg, 256, 0, st>>>((int)h->nnz, h->hptr, h->hidx, K, static_cast<HOut*>(hess));
  if ((flags & MW_G) && h->n_rows > 0)
    k_mc_grad_gather<Real><<<gg, 256, 0, st>>>(h->n_rows, h->gptr, h->gidx, g, h->row_gpos, h->rhs, grad);
  return cudaGetLastError();
}

template <typename Real, typename HOut, int NP, int NQ, bool GQ>
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
  if constexpr (sizeof(Real) == 4 && NP > 3) {
    if (h->tc && (flags & MW_H)) {
      using G = McTile<NP, NQ, GQ>;
      McTcArgs T{h->Phi, h->Plo, h->err, h->wait_limit, h->dp_code, h->dp_sbase, h->dp_elem_rn, h->bp_rn_row,
                 static_cast<float*>(h->dp_sbuf)};
      float* g = static_cast<float*>(h->gbuf);
      HOut* H = static_cast<HOut*>(hess);
      const McConstR<float> Mf = cast_const<float>(h->mc);
      switch (flags) {
        case 4: k_mc_tc<NP, NQ, 4, HOut, GQ><<<h->grid_tc, G::THREADS, G::SMEM, st>>>(A, Mf, T, H, g, h->partials, h->counter, energy); break;
        case 5: k_mc_tc<NP, NQ, 5, HOut, GQ><<<h->grid_tc, G::THREADS, G::SMEM, st>>>(A, Mf, T, H, g, h->partials, h->counter, energy); break;
        case 6: k_mc_tc<NP, NQ, 6, HOut, GQ><<<h->grid_tc, G::THREADS, G::SMEM, st>>>(A, Mf, T, H, g, h->partials, h->counter, energy); break;
        default: k_mc_tc<NP, NQ, 7, HOut, GQ><<<h->grid_tc, G::THREADS, G::SMEM, st>>>(A, Mf, T, H, g, h->partials, h->counter, energy); break;
      }
      // stream-ordered copy of the status word for fne_poll_device_status
      cudaError_t ce = cudaGetLastError();
      if (ce == cudaSuccess) ce = cudaMemcpyAsync(h->err_host, h->err, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (ce != cudaSuccess) return ce;
      return mc_gathers<float, HOut, NP>(h, flags, static_cast<const float*>(nullptr), g, grad, hess, st);
    }
  }
  if constexpr (sizeof(Real) == 8 && NP > 3) {
    if (h->dm && (flags & MW_H)) {
      using G = McTileD<NP, NQ, GQ>;
      McDmArgs T{h->dp_code, h->dp_sbase, h->dp_elem_rn, h->bp_rn_row, static_cast<double*>(h->dp_sbuf),
                 h->dp_sidx};
      double* g = static_cast<double*>(h->gbuf);
      double* H = static_cast<double*>(hess);
      const McConstR<double> Md = cast_const<double>(h->mc);
      switch (flags) {
        case 4: k_mc_dmma<NP, NQ, 4, GQ><<<h->grid_dm, G::THREADS, G::SMEM, st>>>(A, Md, T, H, g, h->partials, h->counter, energy); break;
        case 5: k_mc_dmma<NP, NQ, 5, GQ><<<h->grid_dm, G::THREADS, G::SMEM, st>>>(A, Md, T, H, g, h->partials, h->counter, energy); break;
        case 6: k_mc_dmma<NP, NQ, 6, GQ><<<h->grid_dm, G::THREADS, G::SMEM, st>>>(A, Md, T, H, g, h->partials, h->counter, energy); break;
        default: k_mc_dmma<NP, NQ, 7, GQ><<<h->grid_dm, G::THREADS, G::SMEM, st>>>(A, Md, T, H, g, h->partials, h->counter, energy); break;
      }
      return mc_gathers<double, double, NP>(h, flags, static_cast<const double*>(nullptr), g, grad, hess, st);
    }
  }
  if (!(flags & MW_H) && h->use_eg) {  // energy / gradient callbacks
    const int ge = h->grid_eg;
    switch (flags) {
      case 1: k_mc_eg<Real, NP, NQ, 1, GQ><<<ge, kEgThreads, 0, st>>>(A, M, g, h->partials, h->counter, energy); break;
      case 2: k_mc_eg<Real, NP, NQ, 2, GQ><<<ge, kEgThreads, 0, st>>>(A, M, g, h->partials, h->counter, energy); break;
      case 3: k_mc_eg<Real, NP, NQ, 3, GQ><<<ge, kEgThreads, 0, st>>>(A, M, g, h->partials, h->counter, energy); break;
      default: return cudaErrorInvalidValue;
    }
    return mc_gathers<Real, HOut, NP>(h, flags, K, g, grad, hess, st);
  }
  switch (flags) {
    case 1: k_mc_elem<Real, NP, NQ, 1, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 2: k_mc_elem<Real, NP, NQ, 2, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 3: k_mc_elem<Real, NP, NQ, 3, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 4: k_mc_elem<Real, NP, NQ, 4, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 5: k_mc_elem<Real, NP, NQ, 5, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 6: k_mc_elem<Real, NP, NQ, 6, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    case 7: k_mc_elem<Real, NP, NQ, 7, GQ><<<grid, T, 0, st>>>(A, M, K, g, h->partials, h->counter, energy); break;
    default: return cudaErrorInvalidValue;
  }
  return mc_gathers<Real, HOut, NP>(h, flags, K, g, grad, hess, st);
}

template <typename Real, typename HOut>
cudaError_t mc_dispatch(McHandle* h, int flags, const double* u, double* energy, double* grad, void* hess,
                        cudaStream_t st) {
  if (h->np == 3 && h->nq == 1) return mc_launch<Real, HOut, 3, 1, false>(h, flags, u, energy, grad, hess, st);
  if (h->np == 6 && h->nq == 7)
    return h->gq ? mc_launch<Real, HOut, 6, 7, true>(h, flags, u, energy, grad, hess, st)
                 : mc_launch<Real, HOut, 6, 7, false>(h, flags, u, energy, grad, hess, st);
  if (h->np == 15 && h->nq == 19) return mc_launch<Real, HOut, 15, 19, false>(h, flags, u, energy, grad, hess, st);
  return cudaErrorInvalidValue;
}

// Constant operand P[(a, b), (q, k, l)] = R_qak R_qbl of the tensor-core
// kernel, split into TF32 hi / lo parts and laid out as the kernel's shared
// memory image ([K / 4][M][4] floats, zero padding); also sizes the grid and
// opts the kernel into its shared memory.
template <int NP, int NQ, bool GQ>
int mc_tc_prepare(McHandle* h, const double* tables, std::vector<float>& phi, std::vector<float>& plo) {
  using G = McTile<NP, NQ, GQ>;
  const double* d1 = tables;
  const double* d2 = tables + NQ * NP;
  phi.assign((size_t)G::M * G::KP, 0.f);
  plo.assign((size_t)G::M * G::KP, 0.f);
  int m = 0;
  for (int a = 0; a < NP; ++a)
    for (int b = a; b < NP; ++b, ++m)
      for (int q = 0; q < NQ; ++q)
        for (int k = 0; k < 2; ++k)
          for (int l = 0; l < 2; ++l) {
            const double ra = k == 0 ? d1[q * NP + a] : d2[q * NP + a];
            const double rb = l == 0 ? d1[q * NP + b] : d2[q * NP + b];
            const float v = (float)(ra * rb);
            uint32_t bits;
            std::memcpy(&bits, &v, 4);
            bits &= 0xFFFFE000u;
            float hi;
            std::memcpy(&hi, &bits, 4);
            const int kk = q * 4 + k * 2 + l;
            const size_t off = (size_t)(kk / 4) * G::M * 4 + (size_t)m * 4 + (kk % 4);
            phi[off] = hi;
            plo[off] = v - hi;
          }
  cudaError_t e = cudaSuccess;
  auto opt_in = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
  };
  opt_in((const void*)k_mc_tc<NP, NQ, 4, float, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 5, float, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 6, float, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 7, float, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 4, double, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 5, double, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 6, double, GQ>);
  opt_in((const void*)k_mc_tc<NP, NQ, 7, double, GQ>);
  if (e != cudaSuccess)
    return set_error(FNE_ECUDA, std::string("Mohr-Coulomb: tensor-core kernel shared memory: ") +
                                    cudaGetErrorString(e));
  const int n_tiles = (h->n_local + G::TE - 1) / G::TE;
  h->grid_tc = std::max(1, std::min(n_tiles, h->num_sms * G::MIN_BLOCKS));
  return FNE_OK;
}

// FP64 DMMA kernel: grid (two CTAs per SM) and the shared-memory opt-in.
template <int NP, int NQ, bool GQ>
int mc_dm_prepare(McHandle* h) {
  using G = McTileD<NP, NQ, GQ>;
  cudaError_t e = cudaSuccess;
  auto opt_in = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM);
  };
  opt_in((const void*)k_mc_dmma<NP, NQ, 4, GQ>);
  opt_in((const void*)k_mc_dmma<NP, NQ, 5, GQ>);
  opt_in((const void*)k_mc_dmma<NP, NQ, 6, GQ>);
  opt_in((const void*)k_mc_dmma<NP, NQ, 7, GQ>);
  if (e != cudaSuccess)
    return set_error(FNE_ECUDA, std::string("Mohr-Coulomb: FP64 DMMA kernel shared memory: ") + cudaGetErrorString(e));
  const int n_tiles = (h->n_local + G::TE - 1) / G::TE;
  h->grid_dm = std::max(1, std::min({n_tiles, h->num_sms * G::MIN_BLOCKS, h->n_partials}));
  return FNE_OK;
}

}  // namespace

void mc_destroy(McHandle* h) {
  if (!h) return;
  void* ptrs[] = {h->codes, h->geom, h->epsp, h->dhat1, h->dhat2, h->qw, h->wflag, h->dir, h->rhs,
                  h->partials, h->counter, h->hptr, h->hidx, h->gptr, h->gidx, h->row_gpos, h->Kbuf, h->gbuf,
                  h->Phi, h->Plo, h->err, h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row, h->bp_rn_gpos,
                  h->bp_rn_inc, h->bp_con, h->bp_inc, h->bp_blk, h->dp_code, h->dp_sbase, h->dp_elem_rn,
                  h->dp_sbuf, h->fx_con, h->fx_desc, h->lin_wct, h->lin_ebuf, h->dp_sidx};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->err_host) cudaFreeHost(h->err_host);
  delete h;
}

int mc_create(const fne_desc* d, McHandle** out) {
  *out = nullptr;
  const int np = d->npe, nq = d->nq, n = 2 * np;
  if (d->block_size != 2) return set_error(FNE_EINVAL, "Mohr-Coulomb: block_size must be 2");
  if (!((np == 3 && nq == 1) || (np == 6 && nq == 7) || (np == 15 && nq == 19)))
    return set_error(FNE_EINVAL, "Mohr-Coulomb: supported (nodes, quadrature points): (3,1), (6,7), (15,19)");
  if (d->n_elem > 0 && (!d->e0 || !d->e1 || !d->e3))
    return set_error(FNE_EINVAL, "Mohr-Coulomb: missing element geometry or reference tables");
  const int64_t E = d->n_elem, lo = d->lo, hi = d->hi;
  const int64_t* t2f = d->total_to_free_reord;
  if (E * (int64_t)n * n >= (int64_t)INT32_MAX || d->nnz >= (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS, "Mohr-Coulomb: element matrices exceed 32-bit indexing");
  // s[6] = 1: e0 / e1 hold J^-1 / |det J| per quadrature point (isoparametric map)
  const bool per_point = d->s[6] != 0.0 && nq > 1;
  if (per_point && np != 6)
    return set_error(FNE_EINVAL, "Mohr-Coulomb: per-quadrature-point geometry is supported for P2 (6 nodes) only");
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
    if (per_point) {  // J_q^-1 (4) and |det J_q| per quadrature point
      for (int q = 0; q < nq; ++q) {
        for (int k = 0; k < 4; ++k) geom.push_back(d->e0[(e * nq + q) * 4 + k]);
        geom.push_back(d->e1[e * nq + q]);
      }
    } else {
      for (int k = 0; k < 4; ++k) geom.push_back(d->e0[e * 4 + k]);
      geom.push_back(d->e1[e]);
    }
    if (d->e2)
      for (int k = 0; k < nq * 3; ++k) epsp.push_back(d->e2[e * nq * 3 + k]);
    const double w = d->energy_weights ? d->energy_weights[e] : 1.0;
    if (w != 0.0 && w != 1.0) return set_error(FNE_EINVAL, "Mohr-Coulomb: energy weights must be 0 or 1");
    wflag.push_back(w != 0.0 ? 1 : 0);
  }
  const int64_t nl = (int64_t)local.size();
  // node-block gather plan (default); per-position contribution lists below
  // only when the pattern is not node-blocked
  const int64_t n_owned = hi - lo;
  BlockPlan bp;
  bool use_blk = false;
  {
    std::vector<int64_t> edofs((size_t)nl * n);
    for (int64_t le = 0; le < nl; ++le)
      for (int i = 0; i < n; ++i) edofs[(size_t)le * n + i] = d->elems[local[le] * n + i];
    use_blk = build_block_plan(nl, np, 2, edofs.data(), d, bp) == FNE_OK;
  }
  const int npair = np * (np + 1) / 2;
  std::vector<int32_t> rowof, row_ptr, row_gpos;
  std::vector<int32_t> hptr, gptr, hidx, gidx;
  int32_t n_rows = 0;
  if (!use_blk) {
  rowof.assign(n_owned, -1);
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
  n_rows = (int32_t)row_gpos.size();
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
  // contributions (two passes: count, fill), in element order; element
  // matrices are stored per node pair a <= b: slot pair(a, b) * 4 + c * 2 + d
  auto pair_slot = [np](int i, int j) -> int {
    int a = i >> 1, c = i & 1, b = j >> 1, dd = j & 1;
    if (a > b) {
      std::swap(a, b);
      std::swap(c, dd);
    }
    return (a * np - a * (a - 1) / 2 + (b - a)) * 4 + c * 2 + dd;
  };
  hptr.assign(d->nnz + 1, 0);
  gptr.assign(n_rows + 1, 0);
  std::vector<int32_t> hfill, gfill;
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
          if (pass == 0) hptr[p + 1]++; else hidx[hfill[p]++] = (int32_t)(le * npair * 4 + pair_slot(i, j));
        }
      }
    }
  }
  }  // !use_blk

  auto* h = new (std::nothrow) McHandle();
  if (!h) return set_error(FNE_ENOMEM, "Mohr-Coulomb: out of host memory");
  h->precision = d->precision;
  h->hess_fp32 = d->precision == FNE_FP32 && d->hess_fp32;
  h->np = np;
  h->nq = nq;
  h->gq = per_point ? 1 : 0;
  h->n = n;
  h->n_local = (int)nl;
  h->n_rows = use_blk ? (int32_t)n_owned : n_rows;
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
  // energy / gradient calls: the tiled kernel unless the CUDA-core kernel is requested
  h->use_eg = d->kernel_variant != 1;
  h->grid_eg = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)h->num_sms * 4, (nl + kEgTile - 1) / kEgTile,
                                                            (int64_t)h->n_partials}));
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
  h->use_blk = use_blk ? 1 : 0;
  if (use_blk) {
    h->n_rnodes = bp.n_rnodes;
    MC_TRY(mc_upload(h, &h->bp_rn_blk, bp.rn_blk.data(), bp.rn_blk.size()));
    MC_TRY(mc_upload(h, &h->bp_rn_con, bp.rn_con.data(), bp.rn_con.size()));
    MC_TRY(mc_upload(h, &h->bp_rn_row, bp.rn_row.data(), bp.rn_row.size()));
    MC_TRY(mc_upload(h, &h->bp_rn_gpos, bp.rn_gpos.data(), bp.rn_gpos.size()));
    MC_TRY(mc_upload(h, &h->bp_rn_inc, bp.rn_inc.data(), bp.rn_inc.size()));
    MC_TRY(mc_upload(h, &h->bp_blk, bp.blk.data(), bp.blk.size()));
    MC_TRY(mc_upload(h, &h->bp_con, bp.con.data(), bp.con.size()));
    MC_TRY(mc_upload(h, &h->bp_inc, bp.inc.data(), bp.inc.size()));
  }
  MC_TRY(mc_upload(h, &h->hptr, hptr.data(), hptr.size()));
  MC_TRY(mc_upload(h, &h->hidx, hidx.data(), hidx.size()));
  MC_TRY(mc_upload(h, &h->gptr, gptr.data(), gptr.size()));
  MC_TRY(mc_upload(h, &h->gidx, gidx.data(), gidx.size()));
  MC_TRY(mc_upload(h, &h->row_gpos, row_gpos.data(), row_gpos.size()));
  // tensor-core path: FP32 P2 / P4 on a node-blocked pattern unless CUDA
  // cores are requested; its epilogue writes the COO values directly
  h->tc = d->precision == FNE_FP32 && np > 3 && d->kernel_variant != 1 && use_blk;
  // FP64 DMMA path: FP64 P2 / P4 on a node-blocked pattern, same epilogue
  h->dm = d->precision == FNE_FP64 && np > 3 && d->kernel_variant != 1 && use_blk;
  DirectPlan dp;
  if ((h->tc || h->dm) && build_direct_plan(bp, nl, np, 2, dp) != FNE_OK) h->tc = h->dm = 0;
  {
    unsigned char* kb = nullptr;
    if (!h->tc && !h->dm) MC_TRY(mc_upload(h, &kb, (const unsigned char*)nullptr, (size_t)nl * npair * 4 * rsz));
    h->Kbuf = kb;
    unsigned char* gb = nullptr;
    MC_TRY(mc_upload(h, &gb, (const unsigned char*)nullptr, (size_t)nl * n * rsz));
    h->gbuf = gb;
  }
  h->n_contrib = use_blk ? (int64_t)bp.con.size() : (int64_t)hptr[d->nnz];
  if (h->tc || h->dm) {
    dp.code.push_back(0xFFFF);  // the kernels read codes in 32-bit words
    dp.code.push_back(0xFFFF);
    MC_TRY(mc_upload(h, &h->dp_code, dp.code.data(), dp.code.size()));
    MC_TRY(mc_upload(h, &h->dp_sbase, dp.sbase.data(), dp.sbase.size()));
    MC_TRY(mc_upload(h, &h->dp_elem_rn, bp.elem_rn.data(), bp.elem_rn.size()));
    unsigned char* sb = nullptr;
    MC_TRY(mc_upload(h, &sb, (const unsigned char*)nullptr,
                     (size_t)std::max<int64_t>(1, dp.n_slots) * 4 * (h->dm ? sizeof(double) : sizeof(float))));
    h->dp_sbuf = sb;
    h->n_fix = (int)(dp.fdesc.size() / 4);
    // FP64 DMMA path on P4: shared buffer in fix-up order -- the epilogue
    // writes each 32-byte slot at its fix-up position (sidx), every shared
    // block's contributions are consecutive and the fix-up streams the buffer
    // (P4 at h = 0.08: 1707 -> 1602-1614 us per pass).  Elsewhere the slots
    // stay element-major and the fix-up gathers them through fix.con: P2,
    // where every block of the element is shared, measured 323 -> 367 us in
    // fix-up order, and the tensor-core path's 16-byte slots (half-sector
    // scattered writes) 857 -> 1007 us.
    if (h->dm && np == 15)
      MC_TRY(mc_upload(h, &h->dp_sidx, dp.sidx.data(), dp.sidx.size()));
    else
      MC_TRY(mc_upload(h, &h->fx_con, dp.fix.con.data(), dp.fix.con.size()));
    MC_TRY(mc_upload(h, &h->fx_desc, dp.fdesc.data(), dp.fdesc.size()));
  }
  if (h->dm) {
    const int rc_dm = np == 15 ? mc_dm_prepare<15, 19, false>(h)
                               : (h->gq ? mc_dm_prepare<6, 7, true>(h) : mc_dm_prepare<6, 7, false>(h));
    if (rc_dm) {
      mc_destroy(h);
      return rc_dm;
    }
  }
  if (h->tc) {
    std::vector<float> phi, plo;
    int rc_tc = np == 15 ? mc_tc_prepare<15, 19, false>(h, d->e3, phi, plo)
                         : (h->gq ? mc_tc_prepare<6, 7, true>(h, d->e3, phi, plo)
                                  : mc_tc_prepare<6, 7, false>(h, d->e3, phi, plo));
    if (rc_tc) {
      mc_destroy(h);
      return rc_tc;
    }
    MC_TRY(mc_upload(h, &h->Phi, phi.data(), phi.size()));
    MC_TRY(mc_upload(h, &h->Plo, plo.data(), plo.size()));
    MC_TRY(mc_upload(h, &h->err, (const int*)nullptr, 1));
    if (cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess ||
        cudaHostAlloc((void**)&h->err_host, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
      mc_destroy(h);
      return set_error(FNE_ECUDA, "Mohr-Coulomb: status word");
    }
    *h->err_host = 0;
  }
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

namespace {

template <typename Real, int NP, int NQ, bool GQ>
cudaError_t mc_lin_launch_g(McHandle* h, int op, const double* v, double* out, cudaStream_t st) {
  McArgs A{};
  A.n_el = h->n_local;
  A.codes = h->codes;
  A.geom = h->geom;
  A.epsp = h->epsp;
  A.wflag = h->wflag;
  A.dhat1 = h->dhat1;
  A.dhat2 = h->dhat2;
  A.qw = h->qw;
  A.u = v;
  A.dir = h->dir;
  A.rhs = nullptr;
  A.n_owned = (int)(h->hi - h->lo);
  A.lo = h->lo;
  Real* wct = static_cast<Real*>(h->lin_wct);
  Real* eb = static_cast<Real*>(h->lin_ebuf);
  const int grid = h->grid_elem, T = 32 * kMcWarps;
  if (op == 0) {
    k_mc_lin<Real, NP, NQ, GQ><<<grid, T, 0, st>>>(A, cast_const<Real>(h->mc), wct);
    return cudaGetLastError();
  }
  if (op == 1)
    k_mc_hvp<Real, NP, NQ, false, GQ><<<grid, T, 0, st>>>(A, wct, eb);
  else
    k_mc_hvp<Real, NP, NQ, true, GQ><<<grid, T, 0, st>>>(A, wct, eb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (h->use_blk) {
    if (h->n_rnodes == 0) return cudaSuccess;
    const int gr = std::max(1, std::min(h->num_sms * 8, (h->n_rnodes + 255) / 256));
    k_rowgrad<Real, 2><<<gr, 256, 0, st>>>(h->n_rnodes, h->bp_rn_inc, h->bp_inc, h->bp_rn_gpos, eb, nullptr, out);
  } else if (h->n_rows > 0) {
    const int gg = std::max(1, std::min(h->num_sms * 16, (h->n_rows + 255) / 256));
    k_mc_grad_gather<Real><<<gg, 256, 0, st>>>(h->n_rows, h->gptr, h->gidx, eb, h->row_gpos, nullptr, out);
  }
  return cudaGetLastError();
}

template <typename Real, int NP, int NQ>
cudaError_t mc_lin_launch(McHandle* h, int op, const double* v, double* out, cudaStream_t st) {
  if constexpr (NP == 6)
    if (h->gq) return mc_lin_launch_g<Real, NP, NQ, true>(h, op, v, out, st);
  return mc_lin_launch_g<Real, NP, NQ, false>(h, op, v, out, st);
}

template <typename Real>
cudaError_t mc_lin_dispatch(McHandle* h, int op, const double* v, double* out, cudaStream_t st) {
  if (h->np == 3 && h->nq == 1) return mc_lin_launch<Real, 3, 1>(h, op, v, out, st);
  if (h->np == 6 && h->nq == 7) return mc_lin_launch<Real, 6, 7>(h, op, v, out, st);
  if (h->np == 15 && h->nq == 19) return mc_lin_launch<Real, 15, 19>(h, op, v, out, st);
  return cudaErrorInvalidValue;
}

int mc_lin(McHandle* h, int op, const double* v, double* out, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (op == 0 && !h->lin_wct) {
    const size_t rsz = h->precision == FNE_FP32 ? sizeof(float) : sizeof(double);
    unsigned char *w = nullptr, *eb = nullptr;
    int rc = mc_upload(h, &w, (const unsigned char*)nullptr, std::max<size_t>(1, (size_t)h->n_local * h->nq * 6 * rsz));
    if (!rc) rc = mc_upload(h, &eb, (const unsigned char*)nullptr, std::max<size_t>(1, (size_t)h->n_local * h->n * rsz));
    if (rc) {
      if (w) cudaFree(w);
      if (eb) cudaFree(eb);
      return rc;
    }
    h->lin_wct = w;
    h->lin_ebuf = eb;
  }
  if (op != 0 && !h->lin_ready)
    return set_error(FNE_EINVAL, "matrix-free product: call fne_hvp_prepare first (no linearization point)");
  const cudaError_t e = h->precision == FNE_FP32 ? mc_lin_dispatch<float>(h, op, v, out, st)
                                                  : mc_lin_dispatch<double>(h, op, v, out, st);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("matrix-free product launch: ") + cudaGetErrorString(e));
  if (op == 0) h->lin_ready = 1;
  return FNE_OK;
}

}  // namespace

int mc_hvp_prepare(McHandle* h, const double* u, void* stream) { return mc_lin(h, 0, u, nullptr, stream); }
int mc_hvp(McHandle* h, const double* x, double* y, void* stream) { return mc_lin(h, 1, x, y, stream); }
int mc_hvp_diagonal(McHandle* h, double* diag, void* stream) { return mc_lin(h, 2, nullptr, diag, stream); }

int mc_check_status(McHandle* h) {
  if (!h->err) return FNE_OK;
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_error(FNE_ECUDA, std::string("fne_check_device_status: ") + cudaGetErrorString(e));
  if (v == 0) return FNE_OK;
  cudaMemset(h->err, 0, sizeof(int));
  if (h->err_host) *h->err_host = 0;
  return set_error(FNE_ETIMEOUT, "Mohr-Coulomb tensor-core kernel: an MMA completion wait gave up");
}

int mc_poll_status(McHandle* h) {
  if (!h->err_host || *(volatile int*)h->err_host == 0) return FNE_OK;
  *h->err_host = 0;
  cudaMemset(h->err, 0, sizeof(int));
  return set_error(FNE_ETIMEOUT, "Mohr-Coulomb tensor-core kernel: an MMA completion wait gave up");
}

int mc_set_wait_limit(McHandle* h, long long polls) {
  if (!h->tc) return set_error(FNE_EINVAL, "fne_set_wait_limit: the handle runs no tensor-core kernel");
  h->wait_limit = polls < 0 ? kMcWaitLimit : polls;
  return FNE_OK;
}

void mc_info(const McHandle* h, fne_info* info) {
  info->n_rows = h->n_rows;
  info->nnz = h->nnz;
  info->n_elem = h->n_local;
  info->n_incidences = h->n_contrib;
  info->device_bytes = h->device_bytes;
  info->max_row_len = 0;
  info->kernel_variant = h->tc ? 6 : h->dm ? 9 : 5;
  info->row_lanes = 1;
}

}  // namespace fne
