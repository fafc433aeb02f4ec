// libfne_asm.so -- element energy / gradient / Hessian assembly on sm_100a.
//
// Two kernel shapes (one per launch, no atomics, bit-reproducible):
//
//  * row-gather kernels (k_rows_tri, k_rows_tet): one thread per OUTPUT ROW
//    of the owned COO pattern.  A CTA owns a contiguous block of rows, which
//    is a contiguous slice of the COO value array -- the reference's overlap
//    domain (every element touching an owned row is evaluated, owned rows
//    need no reduction; src/core/petsc/reordered_element_base.py:509-597)
//    applied at CTA granularity.  A thread walks the incidences of its row's
//    node, evaluates the element's gradient entry and Hessian row with
//    hand-written adjoints, and accumulates them in shared memory laid out
//    exactly like the CTA's output slice; the slice is then written with
//    fully coalesced stores.  The energy (FP64) is added once per element by
//    the incidence that carries the element's energy flag.
//  * element kernels (k_energy_*): one thread per element, FP64 energy only
//    (the golden-section / trust-region line-search callback).
//
// Energies always reduce in FP64: warp shuffles, a per-CTA partial, and the
// last CTA to finish (atomic ticket, no waiting) sums the partials in index
// order, so the result does not depend on CTA scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "fne_gather.cuh"
#include "fne_internal.h"

namespace fne {
static thread_local std::string g_err;
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace fne

using namespace fne;

// ---------------------------------------------------------------------------
// parameters and element records
// ---------------------------------------------------------------------------
struct Phys {
  double p;       // p-Laplace exponent
  double eps;     // GL
  double ip[9];   // GL ip[a*3+q]
  double w[3];    // GL quadrature weights
  double C1, D1;  // Neo-Hookean
  int absdet;
  int p_is3;      // p == 3 (sqrt fast path)
  // float copies: FP32 kernels never convert parameters per element
  float pf, epsf, ipf[9], wf[3], C1f, D1f;
};

// parameter in the kernel's arithmetic type, without a per-use conversion
template <typename Real>
__device__ __forceinline__ Real prm(double d, float f);
template <>
__device__ __forceinline__ float prm<float>(double, float f) {
  return f;
}
template <>
__device__ __forceinline__ double prm<double>(double d, float) {
  return d;
}

// Element records are stored as "chunk planes": plane k of an element record
// is the 16-byte chunk  base[k * n + e], so a warp loading plane k of 32
// consecutive elements reads 512 contiguous bytes.
//   P1 triangle, FP32 (3 planes, 48 B): {src0,src1,src2,wflag} {dvx0,dvx1,dvx2,vol} {dvy0,dvy1,dvy2,-}
//   P1 triangle, FP64 (5 planes, 80 B): {src0,src1,src2,wflag} {vol,dvx0} {dvx1,dvx2} {dvy0,dvy1} {dvy2,-}
//   P1 tet, FP32 (5 planes, 80 B):  {src0..3} {gx0..3} {gy0..3} {gz0..3} {vol,wflag,-,-}
//   P1 tet, FP64 (8 planes, 128 B): {src0..3} {gx0,gx1} {gx2,gx3} {gy..} {gy..} {gz..} {gz..} {vol,wflag}
struct __align__(16) Chunk {
  unsigned w[4];
};
template <typename Real>
struct TriPlanes {
  static constexpr int n = sizeof(Real) == 4 ? 3 : 5;
};
template <typename Real>
struct TetPlanes {
  static constexpr int n = sizeof(Real) == 4 ? 5 : 8;
};

template <typename Real>
struct TriElem {
  int src[3];
  int wflag;
  Real dvx[3], dvy[3], vol;
};
template <typename Real>
struct TetElem {
  int src[4];
  int wflag;
  Real g[4][3];
  Real vol;
};

__device__ __forceinline__ int4 ldc_i(const Chunk* __restrict__ R, long long off) {
  return __ldg(reinterpret_cast<const int4*>(R + off));
}
__device__ __forceinline__ float4 ldc_f(const Chunk* __restrict__ R, long long off) {
  return __ldg(reinterpret_cast<const float4*>(R + off));
}
__device__ __forceinline__ double2 ldc_d(const Chunk* __restrict__ R, long long off) {
  return __ldg(reinterpret_cast<const double2*>(R + off));
}

__device__ __forceinline__ void load_tri(const Chunk* __restrict__ R, int n, int e, TriElem<float>& t) {
  const int4 c0 = ldc_i(R, e);
  const float4 c1 = ldc_f(R, (long long)n + e);
  const float4 c2 = ldc_f(R, 2LL * n + e);
  t.src[0] = c0.x; t.src[1] = c0.y; t.src[2] = c0.z; t.wflag = c0.w;
  t.dvx[0] = c1.x; t.dvx[1] = c1.y; t.dvx[2] = c1.z; t.vol = c1.w;
  t.dvy[0] = c2.x; t.dvy[1] = c2.y; t.dvy[2] = c2.z;
}
__device__ __forceinline__ void load_tri(const Chunk* __restrict__ R, int n, int e, TriElem<double>& t) {
  const int4 c0 = ldc_i(R, e);
  const double2 d0 = ldc_d(R, (long long)n + e);
  const double2 d1 = ldc_d(R, 2LL * n + e);
  const double2 d2 = ldc_d(R, 3LL * n + e);
  const double2 d3 = ldc_d(R, 4LL * n + e);
  t.src[0] = c0.x; t.src[1] = c0.y; t.src[2] = c0.z; t.wflag = c0.w;
  t.vol = d0.x; t.dvx[0] = d0.y; t.dvx[1] = d1.x; t.dvx[2] = d1.y;
  t.dvy[0] = d2.x; t.dvy[1] = d2.y; t.dvy[2] = d3.x;
}
__device__ __forceinline__ void load_tet(const Chunk* __restrict__ R, int n, int e, TetElem<float>& t) {
  const int4 c0 = ldc_i(R, e);
  const float4 x = ldc_f(R, (long long)n + e);
  const float4 y = ldc_f(R, 2LL * n + e);
  const float4 z = ldc_f(R, 3LL * n + e);
  const float4 v = ldc_f(R, 4LL * n + e);
  t.src[0] = c0.x; t.src[1] = c0.y; t.src[2] = c0.z; t.src[3] = c0.w;
  t.g[0][0] = x.x; t.g[1][0] = x.y; t.g[2][0] = x.z; t.g[3][0] = x.w;
  t.g[0][1] = y.x; t.g[1][1] = y.y; t.g[2][1] = y.z; t.g[3][1] = y.w;
  t.g[0][2] = z.x; t.g[1][2] = z.y; t.g[2][2] = z.z; t.g[3][2] = z.w;
  t.vol = v.x;
  t.wflag = __float_as_int(v.y);
}
__device__ __forceinline__ void load_tet(const Chunk* __restrict__ R, int n, int e, TetElem<double>& t) {
  const int4 c0 = ldc_i(R, e);
  t.src[0] = c0.x; t.src[1] = c0.y; t.src[2] = c0.z; t.src[3] = c0.w;
  double2 a;
  a = ldc_d(R, 1LL * n + e); t.g[0][0] = a.x; t.g[1][0] = a.y;
  a = ldc_d(R, 2LL * n + e); t.g[2][0] = a.x; t.g[3][0] = a.y;
  a = ldc_d(R, 3LL * n + e); t.g[0][1] = a.x; t.g[1][1] = a.y;
  a = ldc_d(R, 4LL * n + e); t.g[2][1] = a.x; t.g[3][1] = a.y;
  a = ldc_d(R, 5LL * n + e); t.g[0][2] = a.x; t.g[1][2] = a.y;
  a = ldc_d(R, 6LL * n + e); t.g[2][2] = a.x; t.g[3][2] = a.y;
  a = ldc_d(R, 7LL * n + e); t.vol = a.x;
  t.wflag = __double2loint(a.y);
}

__device__ __forceinline__ double gather(const double* __restrict__ u, const double* __restrict__ dir,
                                         int code, int c) {
  return code >= 0 ? __ldg(u + code + c) : __ldg(dir + (-1 - code) + c);
}


// ---------------------------------------------------------------------------
// physics: p-Laplace, Ginzburg-Landau (P1 triangles, scalar)
// ---------------------------------------------------------------------------
enum { FAM_PLAP = 1, FAM_GL = 2 };
enum { W_E = 1, W_G = 2, W_H = 4 };

// Row a of the element gradient and Hessian.  Hand-written adjoints of
//   p-Laplace:  e = vol/p * s^(p/2),  s = Fx^2 + Fy^2
//     g_a = vol s^(p/2-1) G_a,  G_a = Fx dvx_a + Fy dvy_a
//     H_ab = vol [ s^(p/2-1) (dvx_a dvx_b + dvy_a dvy_b) + (p-2) s^(p/2-2) G_a G_b ]
//     (at s = 0 the limit: 0 for p > 2, where JAX's autodiff gives inf*0)
//   GL:  e = vol [ eps/2 s + 1/4 sum_q w_q (n_q^2 - 1)^2 ],  n_q = sum_b v_b ip[b][q]
//     g_a = vol [ eps G_a + sum_q w_q (n_q^2 - 1) n_q ip[a][q] ]
//     H_ab = vol [ eps (dvx_a dvx_b + dvy_a dvy_b) + sum_q w_q (3 n_q^2 - 1) ip[a][q] ip[b][q] ]
template <typename Real, int FAM>
__device__ __forceinline__ void tri_row(const Phys& P, int a, const Real v[3], const TriElem<Real>& t,
                                        Real& ga, Real h[3]) {
  const Real fx = v[0] * t.dvx[0] + v[1] * t.dvx[1] + v[2] * t.dvx[2];
  const Real fy = v[0] * t.dvy[0] + v[1] * t.dvy[1] + v[2] * t.dvy[2];
  const Real dxa = a == 0 ? t.dvx[0] : (a == 1 ? t.dvx[1] : t.dvx[2]);
  const Real dya = a == 0 ? t.dvy[0] : (a == 1 ? t.dvy[1] : t.dvy[2]);
  if (FAM == FAM_PLAP) {
    const Real s = fx * fx + fy * fy;
    const Real p = prm<Real>(P.p, P.pf);
    Real t1, t2;
    if (s > Real(0)) {
      if (P.p_is3) {
        t1 = sqrt(s);
        t2 = Real(1) / t1;
      } else {
        t1 = pow(s, p * Real(0.5) - Real(1));
        t2 = (p - Real(2)) * pow(s, p * Real(0.5) - Real(2));
      }
    } else {
      t1 = P.p == 2.0 ? Real(1) : (P.p > 2.0 ? Real(0) : Real(INFINITY));
      t2 = Real(0);
    }
    const Real Ga = fx * dxa + fy * dya;
    ga = t.vol * t1 * Ga;
#pragma unroll
    for (int b = 0; b < 3; ++b)
      h[b] = t.vol * (t1 * (dxa * t.dvx[b] + dya * t.dvy[b]) + t2 * Ga * (fx * t.dvx[b] + fy * t.dvy[b]));
  } else {
    const Real eps = prm<Real>(P.eps, P.epsf);
    Real ipa[3], n[3], c1[3], c2[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      n[q] = v[0] * prm<Real>(P.ip[q], P.ipf[q]) + v[1] * prm<Real>(P.ip[3 + q], P.ipf[3 + q]) + v[2] * prm<Real>(P.ip[6 + q], P.ipf[6 + q]);
      ipa[q] = a == 0 ? prm<Real>(P.ip[q], P.ipf[q]) : (a == 1 ? prm<Real>(P.ip[3 + q], P.ipf[3 + q]) : prm<Real>(P.ip[6 + q], P.ipf[6 + q]));
      c1[q] = prm<Real>(P.w[q], P.wf[q]) * (n[q] * n[q] - Real(1)) * n[q];
      c2[q] = prm<Real>(P.w[q], P.wf[q]) * (Real(3) * n[q] * n[q] - Real(1)) * ipa[q];
    }
    ga = t.vol * (eps * (fx * dxa + fy * dya) + c1[0] * ipa[0] + c1[1] * ipa[1] + c1[2] * ipa[2]);
#pragma unroll
    for (int b = 0; b < 3; ++b)
      h[b] = t.vol * (eps * (dxa * t.dvx[b] + dya * t.dvy[b]) + c2[0] * prm<Real>(P.ip[3 * b], P.ipf[3 * b]) +
                      c2[1] * prm<Real>(P.ip[3 * b + 1], P.ipf[3 * b + 1]) + c2[2] * prm<Real>(P.ip[3 * b + 2], P.ipf[3 * b + 2]));
  }
}

// FP64 element energy (always double, from the stored geometry).
template <typename Real, int FAM>
__device__ __forceinline__ double tri_energy(const Phys& P, const double v[3], const TriElem<Real>& t) {
  const double fx = v[0] * (double)t.dvx[0] + v[1] * (double)t.dvx[1] + v[2] * (double)t.dvx[2];
  const double fy = v[0] * (double)t.dvy[0] + v[1] * (double)t.dvy[1] + v[2] * (double)t.dvy[2];
  const double s = fx * fx + fy * fy;
  if (FAM == FAM_PLAP) {
    const double ps = P.p == 3.0 ? s * sqrt(s) : pow(s, 0.5 * P.p);
    return (1.0 / P.p) * ps * (double)t.vol;
  } else {
    double pot = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double n = v[0] * P.ip[q] + v[1] * P.ip[3 + q] + v[2] * P.ip[6 + q];
      const double m = n * n - 1.0;
      pot += 0.25 * m * m * P.w[q];
    }
    return (0.5 * P.eps * s + pot) * (double)t.vol;
  }
}

// All three rows at once: gradient g[3] and the symmetric Hessian as its upper
// triangle H = {H00, H01, H02, H11, H12, H22}; with WITH_E also the element
// energy, formed from the same intermediates in the arithmetic (and to the
// bit) of tri_energy_r.
template <typename Real, int FAM, bool WITH_E = false>
__device__ __forceinline__ void tri_full(const Phys& P, const Real v[3], const TriElem<Real>& t, Real g[3],
                                         Real H[6], double* energy = nullptr) {
  const Real fx = v[0] * t.dvx[0] + v[1] * t.dvx[1] + v[2] * t.dvx[2];
  const Real fy = v[0] * t.dvy[0] + v[1] * t.dvy[1] + v[2] * t.dvy[2];
  Real G[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) G[b] = fx * t.dvx[b] + fy * t.dvy[b];
  Real K[6];
  K[0] = t.dvx[0] * t.dvx[0] + t.dvy[0] * t.dvy[0];
  K[1] = t.dvx[0] * t.dvx[1] + t.dvy[0] * t.dvy[1];
  K[2] = t.dvx[0] * t.dvx[2] + t.dvy[0] * t.dvy[2];
  K[3] = t.dvx[1] * t.dvx[1] + t.dvy[1] * t.dvy[1];
  K[4] = t.dvx[1] * t.dvx[2] + t.dvy[1] * t.dvy[2];
  K[5] = t.dvx[2] * t.dvx[2] + t.dvy[2] * t.dvy[2];
  if (FAM == FAM_PLAP) {
    const Real s = fx * fx + fy * fy;
    const Real p = prm<Real>(P.p, P.pf);
    Real t1, t2;
    if (s > Real(0)) {
      if (P.p_is3) {
        t1 = sqrt(s);
        t2 = Real(1) / t1;
      } else {
        t1 = pow(s, p * Real(0.5) - Real(1));
        t2 = (p - Real(2)) * pow(s, p * Real(0.5) - Real(2));
      }
    } else {
      t1 = P.p == 2.0 ? Real(1) : (P.p > 2.0 ? Real(0) : Real(INFINITY));
      t2 = Real(0);
    }
    if (WITH_E) {
      const Real ps = P.p_is3 ? s * sqrt(s) : pow(s, Real(0.5) * p);
      *energy = (double)(ps * t.vol / p);
    }
    const Real vt1 = t.vol * t1, vt2 = t.vol * t2;
#pragma unroll
    for (int b = 0; b < 3; ++b) g[b] = vt1 * G[b];
    H[0] = vt1 * K[0] + vt2 * G[0] * G[0];
    H[1] = vt1 * K[1] + vt2 * G[0] * G[1];
    H[2] = vt1 * K[2] + vt2 * G[0] * G[2];
    H[3] = vt1 * K[3] + vt2 * G[1] * G[1];
    H[4] = vt1 * K[4] + vt2 * G[1] * G[2];
    H[5] = vt1 * K[5] + vt2 * G[2] * G[2];
  } else {
    const Real eps = prm<Real>(P.eps, P.epsf);
    Real ip[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) ip[k] = prm<Real>(P.ip[k], P.ipf[k]);
    Real c1[3], c2[3];
    Real pot = Real(0);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const Real n = v[0] * ip[q] + v[1] * ip[3 + q] + v[2] * ip[6 + q];
      c1[q] = prm<Real>(P.w[q], P.wf[q]) * (n * n - Real(1)) * n;
      c2[q] = prm<Real>(P.w[q], P.wf[q]) * (Real(3) * n * n - Real(1));
      if (WITH_E) {
        const Real m = n * n - Real(1);
        pot += m * m * prm<Real>(P.w[q], P.wf[q]);
      }
    }
    if (WITH_E) {
      const Real s = fx * fx + fy * fy;
      *energy = (double)((Real(0.5) * eps * s + Real(0.25) * pot) * t.vol);
    }
#pragma unroll
    for (int b = 0; b < 3; ++b)
      g[b] = t.vol * (eps * G[b] + c1[0] * ip[3 * b] + c1[1] * ip[3 * b + 1] + c1[2] * ip[3 * b + 2]);
    int m = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b, ++m)
        H[m] = t.vol * (eps * K[m] + c2[0] * ip[3 * a] * ip[3 * b] + c2[1] * ip[3 * a + 1] * ip[3 * b + 1] +
                        c2[2] * ip[3 * a + 2] * ip[3 * b + 2]);
  }
}

// Element energy in the kernel's arithmetic type (FP32 mode: FP32 element
// energies, reduced in FP64 by the caller).
template <typename Real, int FAM>
__device__ __forceinline__ double tri_energy_r(const Phys& P, const Real v[3], const TriElem<Real>& t) {
  const Real fx = v[0] * t.dvx[0] + v[1] * t.dvx[1] + v[2] * t.dvx[2];
  const Real fy = v[0] * t.dvy[0] + v[1] * t.dvy[1] + v[2] * t.dvy[2];
  const Real s = fx * fx + fy * fy;
  if (FAM == FAM_PLAP) {
    const Real ps = P.p_is3 ? s * sqrt(s) : pow(s, Real(0.5) * prm<Real>(P.p, P.pf));
    return (double)(ps * t.vol / prm<Real>(P.p, P.pf));
  } else {
    Real pot = Real(0);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const Real n = v[0] * prm<Real>(P.ip[q], P.ipf[q]) + v[1] * prm<Real>(P.ip[3 + q], P.ipf[3 + q]) +
                     v[2] * prm<Real>(P.ip[6 + q], P.ipf[6 + q]);
      const Real m = n * n - Real(1);
      pot += m * m * prm<Real>(P.w[q], P.wf[q]);
    }
    return (double)((Real(0.5) * prm<Real>(P.eps, P.epsf) * s + Real(0.25) * pot) * t.vol);
  }
}

// ---------------------------------------------------------------------------
// physics: compressible Neo-Hookean (P1 tetrahedra, 3 DOFs per node)
//   W(F) = C1 (|F|^2 - 3 - 2 ln J) + D1 (J - 1)^2,  F = sum_a y_a (x) g_a,  J = det F
//   dW/dF = 2 C1 F + c3 cof(F),            c3 = -2 C1 / J + 2 D1 (J - s)
//   H_(a,c)(b,d) = vol [ 2 C1 (g_a.g_b) delta_cd + c2 (cof g_a)_c (cof g_b)_d
//                        + c3 eps_cdm (F (g_a x g_b))_m ],   c2 = 2 C1 / J^2 + 2 D1
//   (s = 1, or sign(J) when |J| enters the energy; the last term is the
//   contraction of d^2 J / dF^2 = eps_cdm eps_jlp F_mp with g_a, g_b).
// ---------------------------------------------------------------------------
template <typename Real>
struct HeState {
  Real F[3][3], cof[3][3], J, c2, c3;
};

template <typename Real>
__device__ __forceinline__ void he_state(const Phys& P, const Real y[4][3], const TetElem<Real>& t,
                                         HeState<Real>& S) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      S.F[i][j] = y[0][i] * t.g[0][j] + y[1][i] * t.g[1][j] + y[2][i] * t.g[2][j] + y[3][i] * t.g[3][j];
  const Real(&F)[3][3] = S.F;
  S.cof[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
  S.cof[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
  S.cof[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
  S.cof[1][0] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
  S.cof[1][1] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
  S.cof[1][2] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
  S.cof[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
  S.cof[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
  S.cof[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
  S.J = F[0][0] * S.cof[0][0] + F[0][1] * S.cof[0][1] + F[0][2] * S.cof[0][2];
  const Real C1 = prm<Real>(P.C1, P.C1f), D1 = prm<Real>(P.D1, P.D1f);
  const Real sg = P.absdet ? (S.J > Real(0) ? Real(1) : (S.J < Real(0) ? Real(-1) : Real(0))) : Real(1);
  const Real iJ = Real(1) / S.J;
  S.c2 = Real(2) * C1 * iJ * iJ + Real(2) * D1;
  S.c3 = -Real(2) * C1 * iJ + Real(2) * D1 * (S.J - sg);
}

// Gradient entry (a, c) and Hessian row (a, c) over all 12 element DOFs.
template <typename Real>
__device__ __forceinline__ void he_row(const Phys& P, int a, int c, const HeState<Real>& S,
                                       const TetElem<Real>& t, Real& gac, Real h[4][3], bool want_h) {
  Real ga[3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
    ga[j] = a == 0 ? t.g[0][j] : (a == 1 ? t.g[1][j] : (a == 2 ? t.g[2][j] : t.g[3][j]));
  const Real C1 = prm<Real>(P.C1, P.C1f);
  const Real Fc0 = c == 0 ? S.F[0][0] : (c == 1 ? S.F[1][0] : S.F[2][0]);
  const Real Fc1 = c == 0 ? S.F[0][1] : (c == 1 ? S.F[1][1] : S.F[2][1]);
  const Real Fc2 = c == 0 ? S.F[0][2] : (c == 1 ? S.F[1][2] : S.F[2][2]);
  const Real Cc0 = c == 0 ? S.cof[0][0] : (c == 1 ? S.cof[1][0] : S.cof[2][0]);
  const Real Cc1 = c == 0 ? S.cof[0][1] : (c == 1 ? S.cof[1][1] : S.cof[2][1]);
  const Real Cc2 = c == 0 ? S.cof[0][2] : (c == 1 ? S.cof[1][2] : S.cof[2][2]);
  const Real Pg = Real(2) * C1 * (Fc0 * ga[0] + Fc1 * ga[1] + Fc2 * ga[2]);
  const Real cga_c = Cc0 * ga[0] + Cc1 * ga[1] + Cc2 * ga[2];  // (cof g_a)_c
  gac = t.vol * (Pg + S.c3 * cga_c);
  if (!want_h) return;
  const Real k1 = t.vol * Real(2) * C1, k2 = t.vol * S.c2 * cga_c, k3 = t.vol * S.c3;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const Real* gb = t.g[b];
    const Real dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
    // (cof g_b)_d
    Real cgb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) cgb[d] = S.cof[d][0] * gb[0] + S.cof[d][1] * gb[1] + S.cof[d][2] * gb[2];
    // w = F (g_a x g_b)
    const Real x0 = ga[1] * gb[2] - ga[2] * gb[1];
    const Real x1 = ga[2] * gb[0] - ga[0] * gb[2];
    const Real x2 = ga[0] * gb[1] - ga[1] * gb[0];
    Real w[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) w[m] = S.F[m][0] * x0 + S.F[m][1] * x1 + S.F[m][2] * x2;
    // skew row c of eps_cdm w_m: c=0 -> (0, w2, -w1); c=1 -> (-w2, 0, w0); c=2 -> (w1, -w0, 0)
    const Real s0 = c == 0 ? Real(0) : (c == 1 ? -w[2] : w[1]);
    const Real s1 = c == 0 ? w[2] : (c == 1 ? Real(0) : -w[0]);
    const Real s2 = c == 0 ? -w[1] : (c == 1 ? w[0] : Real(0));
    h[b][0] = k2 * cgb[0] + k3 * s0 + (c == 0 ? k1 * dot : Real(0));
    h[b][1] = k2 * cgb[1] + k3 * s1 + (c == 1 ? k1 * dot : Real(0));
    h[b][2] = k2 * cgb[2] + k3 * s2 + (c == 2 ? k1 * dot : Real(0));
  }
}

// FP64 element energy of one tetrahedron.
template <typename Real>
__device__ __forceinline__ double he_energy(const Phys& P, const double y[4][3], const TetElem<Real>& t) {
  double F[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      F[i][j] = y[0][i] * (double)t.g[0][j] + y[1][i] * (double)t.g[1][j] + y[2][i] * (double)t.g[2][j] +
                y[3][i] * (double)t.g[3][j];
  double I1 = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) I1 += F[i][j] * F[i][j];
  double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
             F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
  if (P.absdet) J = fabs(J);
  return (P.C1 * (I1 - 3.0 - 2.0 * log(J)) + P.D1 * (J - 1.0) * (J - 1.0)) * (double)t.vol;
}

// ---------------------------------------------------------------------------
// FP64 reduction: per-CTA partial + last-CTA finalisation (no spin-waits)
// ---------------------------------------------------------------------------
struct EnergyOut {
  double* partials;
  unsigned* counter;
  double* out;            // destination of the total
  const double* addend;   // optional constant added to the total (device)
};

__device__ __forceinline__ double block_sum(double v, double* ws) {
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
  return v;  // valid in thread 0
}

__device__ void energy_finalize(double v, const EnergyOut& eo) {
  __shared__ double ws[32];
  __shared__ int is_last;
  v = block_sum(v, ws);
  if (threadIdx.x == 0) {
    eo.partials[blockIdx.x] = v;
    __threadfence();
    const unsigned ticket = atomicAdd(eo.counter, 1u);
    is_last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s = 0.0;
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) s += __ldcg(eo.partials + j);
  s = block_sum(s, ws);
  if (threadIdx.x == 0) {
    eo.out[0] = s + (eo.addend ? *eo.addend : 0.0);
    *eo.counter = 0u;
  }
}


// ---------------------------------------------------------------------------
// row-gather kernels (one thread per owned row; incidences recomputed)
// ---------------------------------------------------------------------------
struct RowArgs {
  int n_rows;
  const int* __restrict__ row_ptr;
  const int* __restrict__ row_node;
  const unsigned char* __restrict__ row_comp;
  const int* __restrict__ row_gpos;
  const int* __restrict__ inc_ptr;
  const int* __restrict__ inc_elem;
  const unsigned* __restrict__ inc_info;
  const double* __restrict__ u;
  const double* __restrict__ dir;
  const double* __restrict__ rhs;  // may be null
  long long lo;
  int nrec;                        // records (plane stride)
};

constexpr int kTriRows = 256;
constexpr int kTetRows = 128;

template <typename Real, int FAM, int WANT, typename HOut>
__global__ void __launch_bounds__(kTriRows) k_rows_tri(RowArgs A, const Chunk* __restrict__ R, Phys P,
                                                       double* __restrict__ grad, HOut* __restrict__ hess,
                                                       EnergyOut eo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* sacc = reinterpret_cast<Real*>(smem_raw);
  const int r0 = blockIdx.x * blockDim.x;
  const int r = r0 + threadIdx.x;
  const int rend = min(r0 + (int)blockDim.x, A.n_rows);
  const int cs = A.row_ptr[r0];
  const int clen = A.row_ptr[rend] - cs;
  if (WANT & W_H) {
    for (int j = threadIdx.x; j < clen; j += blockDim.x) sacc[j] = Real(0);
    __syncthreads();
  }
  double eacc = 0.0;
  if (r < A.n_rows) {
    const int node = A.row_node[r];
    const int base = A.row_ptr[r] - cs;
    const int ib = A.inc_ptr[node], ie = A.inc_ptr[node + 1];
    Real g = Real(0);
    for (int i = ib; i < ie; ++i) {
      const int el = __ldg(A.inc_elem + i);
      const unsigned info = __ldg(A.inc_info + i);
      TriElem<Real> t;
      load_tri(R, A.nrec, el, t);
      double vd[3];
#pragma unroll
      for (int b = 0; b < 3; ++b) vd[b] = gather(A.u, A.dir, t.src[b], 0);
      const Real v[3] = {(Real)vd[0], (Real)vd[1], (Real)vd[2]};
      const int a = info & 7u;
      Real ga, h[3];
      tri_row<Real, FAM>(P, a, v, t, ga, h);
      if (WANT & W_G) g += ga;
      if (WANT & W_H) {
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const unsigned off = (info >> (kOffShift + kOffBits * b)) & 127u;
          if (off != kNoCol) sacc[base + off] += h[b];
        }
      }
      if ((WANT & W_E) && (info & kEnergyFlag)) eacc += tri_energy<Real, FAM>(P, vd, t);
    }
    const int gp = A.row_gpos[r];
    if (WANT & W_G) grad[gp] = (double)g - (A.rhs ? A.rhs[gp] : 0.0);
    if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
  }
  if (WANT & W_H) {
    __syncthreads();
    for (int j = threadIdx.x; j < clen; j += blockDim.x) hess[cs + j] = (HOut)sacc[j];
  }
  if (WANT & W_E) energy_finalize(eacc, eo);
}

template <typename Real, int WANT, typename HOut, int G>
__global__ void __launch_bounds__(kTetRows) k_rows_tet(RowArgs A, const Chunk* __restrict__ R, Phys P,
                                                       double* __restrict__ grad, HOut* __restrict__ hess,
                                                       EnergyOut eo) {
  // G lanes per output row (consecutive threads): lane s takes the row's
  // incident elements s, s + G, ... into its own shared-memory slice of the
  // CTA's rows; the slices are summed in lane order at the end and the
  // gradient over the lanes by a fixed shuffle tree (deterministic).
  constexpr int RP = kTetRows / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* sacc = reinterpret_cast<Real*>(smem_raw);
  const int r0 = blockIdx.x * RP;
  const int sub = threadIdx.x % G;
  const int r = r0 + threadIdx.x / G;
  const int rend = min(r0 + RP, A.n_rows);
  const int cs = A.row_ptr[r0];
  const int clen = A.row_ptr[rend] - cs;
  Real* slice = sacc + sub * clen;
  if (WANT & W_H) {
    for (int j = threadIdx.x; j < G * clen; j += blockDim.x) sacc[j] = Real(0);
    __syncthreads();
  }
  double eacc = 0.0;
  Real g = Real(0);
  int c = 0, gp = 0;
  if (r < A.n_rows) {
    const int node = A.row_node[r];
    c = A.row_comp[r];
    const int base = A.row_ptr[r] - cs;
    const int ib = A.inc_ptr[node], ie = A.inc_ptr[node + 1];
    for (int i = ib + sub; i < ie; i += G) {
      const int el = __ldg(A.inc_elem + i);
      const unsigned info = __ldg(A.inc_info + i);
      TetElem<Real> t;
      load_tet(R, A.nrec, el, t);
      double yd[4][3];
      Real y[4][3];
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          yd[b][d] = gather(A.u, A.dir, t.src[b], d);
          y[b][d] = (Real)yd[b][d];
        }
      HeState<Real> S;
      he_state(P, y, t, S);
      const int a = info & 7u;
      Real gac, h[4][3];
      he_row(P, a, c, S, t, gac, h, (WANT & W_H) != 0);
      if (WANT & W_G) g += gac;
      if (WANT & W_H) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const unsigned off = (info >> (kOffShift + kOffBits * b)) & 127u;
          if (off != kNoCol) {
            slice[base + off] += h[b][0];
            slice[base + off + 1] += h[b][1];
            slice[base + off + 2] += h[b][2];
          }
        }
      }
      if ((WANT & W_E) && c == 0 && (info & kEnergyFlag)) eacc += he_energy<Real>(P, yd, t);
    }
    gp = A.row_gpos[r];
  }
  if (WANT & W_G) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o, G);
    if (r < A.n_rows && sub == 0) grad[gp] = (double)g - (A.rhs ? A.rhs[gp] : 0.0);
  }
  if ((WANT & W_E) && A.rhs && r < A.n_rows && sub == 0) eacc -= A.rhs[gp] * A.u[A.lo + gp];
  if (WANT & W_H) {
    __syncthreads();
    for (int j = threadIdx.x; j < clen; j += blockDim.x) {
      Real v = sacc[j];
#pragma unroll
      for (int s2 = 1; s2 < G; ++s2) v += sacc[s2 * clen + j];
      hess[cs + j] = (HOut)v;
    }
  }
  if (WANT & W_E) energy_finalize(eacc, eo);
}

// ---------------------------------------------------------------------------
// Element-parallel Neo-Hookean pass (P1 tets, kernel_variant 2): one thread evaluates
// one tetrahedron once -- FP64 energy, the 12 gradient entries and the 10
// node-pair blocks (a <= b) of the element Hessian,
//   H_(a,c),(b,d) = vol [2 C1 (g_a . g_b) delta_cd + c2 (cof g_a)_c (cof g_b)_d
//                        + c3 eps_cdm (F (g_a x g_b))_m],
// stored per element (90 + 12 values); k_node_gather (fne_gather.cuh) then
// sums them per output block of the owned COO values and per gradient row in
// a fixed order (no atomics, deterministic), replacing the reference's
// np.add.at scatter.
// ---------------------------------------------------------------------------
constexpr int kHePairs = 10;
constexpr int kHeSlots = 9 * kHePairs;

template <typename Real, int WANT>
__global__ void __launch_bounds__(256) k_he_elem(const Chunk* __restrict__ R, int n_el, const double* __restrict__ u,
                                                 const double* __restrict__ dir, Phys P, Real* __restrict__ kbuf,
                                                 Real* __restrict__ gbuf, const double* __restrict__ rhs,
                                                 int n_owned, long long lo, EnergyOut eo) {
  double eacc = 0.0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_el; e += gridDim.x * blockDim.x) {
    TetElem<Real> t;
    load_tet(R, n_el, e, t);
    double yd[4][3];
    Real y[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        yd[b][d] = gather(u, dir, t.src[b], d);
        y[b][d] = (Real)yd[b][d];
      }
    if ((WANT & W_E) && t.wflag) eacc += he_energy<Real>(P, yd, t);
    if (!(WANT & (W_G | W_H))) continue;
    HeState<Real> S;
    he_state(P, y, t, S);
    const Real C1 = prm<Real>(P.C1, P.C1f);
    Real cg[4][3];  // (cof g_a)_c
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        cg[a][c] = S.cof[c][0] * t.g[a][0] + S.cof[c][1] * t.g[a][1] + S.cof[c][2] * t.g[a][2];
    if (WANT & W_G) {
      Real* gb = gbuf + (long long)e * 12;
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const Real Fg = S.F[c][0] * t.g[a][0] + S.F[c][1] * t.g[a][1] + S.F[c][2] * t.g[a][2];
          gb[a * 3 + c] = t.vol * (Real(2) * C1 * Fg + S.c3 * cg[a][c]);
        }
    }
    if (WANT & W_H) {
      Real* kb = kbuf + (long long)e * kHeSlots;
      const Real k1 = t.vol * Real(2) * C1, k2 = t.vol * S.c2, k3 = t.vol * S.c3;
      int pr = 0;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
#pragma unroll
        for (int b = a; b < 4; ++b, ++pr) {
          const Real* ga = t.g[a];
          const Real* gbv = t.g[b];
          const Real dot = ga[0] * gbv[0] + ga[1] * gbv[1] + ga[2] * gbv[2];
          const Real x0 = ga[1] * gbv[2] - ga[2] * gbv[1];
          const Real x1 = ga[2] * gbv[0] - ga[0] * gbv[2];
          const Real x2 = ga[0] * gbv[1] - ga[1] * gbv[0];
          Real w[3];
#pragma unroll
          for (int m = 0; m < 3; ++m) w[m] = k3 * (S.F[m][0] * x0 + S.F[m][1] * x1 + S.F[m][2] * x2);
          Real* o = kb + pr * 9;
          o[0] = k2 * cg[a][0] * cg[b][0] + k1 * dot;
          o[1] = k2 * cg[a][0] * cg[b][1] + w[2];
          o[2] = k2 * cg[a][0] * cg[b][2] - w[1];
          o[3] = k2 * cg[a][1] * cg[b][0] - w[2];
          o[4] = k2 * cg[a][1] * cg[b][1] + k1 * dot;
          o[5] = k2 * cg[a][1] * cg[b][2] + w[0];
          o[6] = k2 * cg[a][2] * cg[b][0] + w[1];
          o[7] = k2 * cg[a][2] * cg[b][1] - w[0];
          o[8] = k2 * cg[a][2] * cg[b][2] + k1 * dot;
        }
      }
    }
  }
  if (WANT & W_E) {
    if (rhs)
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += gridDim.x * blockDim.x)
        eacc -= rhs[i] * u[lo + i];
    energy_finalize(eacc, eo);
  }
}

// ---------------------------------------------------------------------------
// Incidence-parallel kernel (P1 triangles): one thread per (row, element)
// incidence.  Each thread runs one short chain of independent loads
// (incidence word -> element record -> 3 nodal values), evaluates the
// element's gradient entry and Hessian row for its local node, and the CTA
// sums the incidences of each row in shared memory in rank order (round k
// adds the k-th incidence of every row: no two writers per address, fixed
// order).  The CTA's rows are one contiguous slice of the COO values, written
// with coalesced stores.
// ---------------------------------------------------------------------------
struct IncArgs {
  const int* __restrict__ cta_row;
  const int* __restrict__ cta_inc;
  const int* __restrict__ inc_elem;
  const unsigned* __restrict__ inc_word;
  const unsigned short* __restrict__ inc_rowl;
  int max_rank;
  int max_rows;
  int max_len;
};
constexpr int kIncThreads = 512;

template <typename Real, int FAM, int WANT, typename HOut>
__global__ void __launch_bounds__(kIncThreads, 2) k_inc_tri(RowArgs A, IncArgs Q, const Chunk* __restrict__ R,
                                                            Phys P, double* __restrict__ grad,
                                                            HOut* __restrict__ hess, EnergyOut eo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int cta = blockIdx.x;
  const int r0 = Q.cta_row[cta], r1 = Q.cta_row[cta + 1];
  const int i0 = Q.cta_inc[cta], i1 = Q.cta_inc[cta + 1];
  const int cs = A.row_ptr[r0];
  const int clen = A.row_ptr[r1] - cs;
  const int nrows = r1 - r0;
  Real* sgrad = reinterpret_cast<Real*>(smem_raw);        // [max_rows]
  Real* srow = sgrad + Q.max_rows;                         // [max_len]
  int* sbase = reinterpret_cast<int*>(srow + Q.max_len);   // [max_rows] slice offset of each row
  for (int k = threadIdx.x; k < nrows; k += blockDim.x) {
    sbase[k] = A.row_ptr[r0 + k] - cs;
    if (WANT & W_G) sgrad[k] = Real(0);
  }
  if (WANT & W_H)
    for (int j = threadIdx.x; j < clen; j += blockDim.x) srow[j] = Real(0);
  const int i = i0 + threadIdx.x;
  const bool active = i < i1;
  unsigned w = 0;
  int rl = 0;
  Real ga = Real(0), h[3] = {Real(0), Real(0), Real(0)};
  double eacc = 0.0;
  if (active) {
    const int el = __ldg(Q.inc_elem + i);
    w = __ldg(Q.inc_word + i);
    rl = __ldg(Q.inc_rowl + i);
    TriElem<Real> t;
    load_tri(R, A.nrec, el, t);
    double vd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) vd[b] = gather(A.u, A.dir, t.src[b], 0);
    const Real v[3] = {(Real)vd[0], (Real)vd[1], (Real)vd[2]};
    tri_row<Real, FAM>(P, (int)(w & 3u), v, t, ga, h);
    if ((WANT & W_E) && (w & 4u)) eacc = tri_energy<Real, FAM>(P, vd, t);
  }
  __syncthreads();
  if (WANT & (W_G | W_H)) {
    const int rank = (w >> 3) & 15u;
    const int base = active ? sbase[rl] : 0;
    for (int k = 0; k <= Q.max_rank; ++k) {
      if (active && rank == k) {
        if (WANT & W_G) sgrad[rl] += ga;
        if (WANT & W_H) {
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            const unsigned off = (w >> (7 + kOffBits * b)) & 127u;
            if (off != kNoCol) srow[base + off] += h[b];
          }
        }
      }
      __syncthreads();
    }
  }
  for (int k = threadIdx.x; k < nrows; k += blockDim.x) {
    const int gp = A.row_gpos[r0 + k];
    if (WANT & W_G) grad[gp] = (double)sgrad[k] - (A.rhs ? A.rhs[gp] : 0.0);
    if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
  }
  if (WANT & W_H)
    for (int j = threadIdx.x; j < clen; j += blockDim.x) hess[cs + j] = (HOut)srow[j];
  if (WANT & W_E) energy_finalize(eacc, eo);
}

// ---------------------------------------------------------------------------
// Banded-sweep kernel (P1 triangles): CTA s owns the row segment
// [seg_row[s], seg_row[s+1]) and sweeps the elements that feed it in order of
// their first row, in batches of NB: every element is evaluated once (plus the
// few "pre" elements shared with the previous segment), the records are read
// with coalesced 16-byte loads and the next batch's records are in flight
// while the current batch is reduced.  Row sums live in a shared-memory ring
// window over the COO positions; after each batch the rows that no later
// element can touch are streamed out (contiguous, coalesced) and their window
// slots cleared.  Each row entry of a batch is summed by one thread in a
// fixed order: no atomics, bit-reproducible.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int sym_index(int a, int b) {  // upper-triangle slot of (a, b)
  const int lo = min(a, b), hi = max(a, b);
  return lo == 0 ? hi : (lo == 1 ? 2 + hi : 5);
}

struct SweepArgs {
  const int* __restrict__ seg_row;
  const int* __restrict__ seg_elem;
  const int* __restrict__ seg_batch;
  const int* __restrict__ batch_done;
  const int* __restrict__ ent_ptr;
  const int* __restrict__ inc_base;
  const int* __restrict__ ent_row;
  const int* __restrict__ ent_pos;
  const unsigned* __restrict__ ent_meta;
  const unsigned* __restrict__ inc_word;
  int win_mask;
  int rwin_mask;
  int gpos_identity;
  // push variant: per element the 7-bit column offsets of its 3 x 3 entries
  // inside the rows of its nodes (21 bits per local node), and the COO row
  // index of every owned reordered DOF
  const unsigned long long* __restrict__ eoff;
  const int* __restrict__ row_of;
};

// Per-thread prefetch state of one batch: the element it evaluates and the
// row entry it reduces (first kPfWords incidence words in registers).
constexpr int kPfWords = 4;
template <typename Real>
struct SweepPf {
  TriElem<Real> t;
  Real v[3];
  int row, pos;
  unsigned meta;
  unsigned w[kPfWords];
  bool elem_ok, ent_ok;
};

// level-1 loads of batch b: element record and row-entry header
template <typename Real>
__device__ __forceinline__ void sweep_load1(const SweepArgs& S, const Chunk* __restrict__ R, int nrec, int e,
                                            bool elem_ok, int ent, bool ent_ok, SweepPf<Real>& f) {
  f.elem_ok = elem_ok;
  f.ent_ok = ent_ok;
  if (elem_ok) load_tri(R, nrec, e, f.t);
  if (ent_ok) {
    f.row = __ldg(S.ent_row + ent);
    f.pos = __ldg(S.ent_pos + ent);
    f.meta = __ldg(S.ent_meta + ent);
  }
}
// level-2 loads of batch b: nodal values and incidence words
template <typename Real>
__device__ __forceinline__ void sweep_load2(const SweepArgs& S, const double* __restrict__ u,
                                            const double* __restrict__ dir, int ibase, SweepPf<Real>& f) {
  if (f.elem_ok) {
#pragma unroll
    for (int k = 0; k < 3; ++k) f.v[k] = (Real)gather(u, dir, f.t.src[k], 0);
  }
  if (f.ent_ok) {
    const unsigned* __restrict__ iw = S.inc_word + ibase + (f.meta & 0xffffu);
    const int cnt = f.meta >> 16;
#pragma unroll
    for (int k = 0; k < kPfWords; ++k) f.w[k] = k < cnt ? __ldg(iw + k) : 0u;
  }
}

template <typename Real, int WANT, int NB>
__device__ __forceinline__ void sweep_reduce_word(unsigned w, int pos0, const Real* sH, const Real* sG, Real* swin,
                                                  int win_mask, Real& gs) {
  const int j = w & 511u;
  const int a = (w >> 9) & 3u;
  if (WANT & W_G) gs += sG[a * NB + j];
  if (WANT & W_H) {
    const Real* hrow = sH + 3 * a * NB + j;  // row a of the element Hessian
#pragma unroll
    for (int bb = 0; bb < 3; ++bb) {
      const unsigned off = (w >> (11 + kOffBits * bb)) & 127u;
      if (off != kNoCol) swin[(pos0 + (int)off) & win_mask] += hrow[bb * NB];
    }
  }
}

template <typename Real, int FAM, int WANT, typename HOut, int NB>
__global__ void __launch_bounds__(NB, 2) k_sweep_tri(RowArgs A, SweepArgs S, const Chunk* __restrict__ R, Phys P,
                                                     double* __restrict__ grad, HOut* __restrict__ hess,
                                                     EnergyOut eo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* sH = reinterpret_cast<Real*>(smem_raw);  // [9][NB] element Hessians, row-major 3x3
  Real* sG = sH + 9 * NB;                         // [3][NB]
  Real* swin = sG + 3 * NB;                       // [win_mask + 1]
  Real* sgw = swin + (S.win_mask + 1);            // [rwin_mask + 1]
  const int seg = blockIdx.x;
  const int R0 = S.seg_row[seg], R1 = S.seg_row[seg + 1];
  const int p_lo = S.seg_elem[3 * seg], o_lo = S.seg_elem[3 * seg + 1], o_hi = S.seg_elem[3 * seg + 2];
  const int b0 = S.seg_batch[seg], b1 = S.seg_batch[seg + 1];
  if (WANT & W_H)
    for (int j = threadIdx.x; j <= S.win_mask; j += NB) swin[j] = Real(0);
  if (WANT & W_G)
    for (int j = threadIdx.x; j <= S.rwin_mask; j += NB) sgw[j] = Real(0);
  double eacc = 0.0;
  int done = R0;
  int p_done = A.row_ptr[R0];
  // batch b0 (prologue)
  SweepPf<Real> cur, nxt;
  int c_eb = 0, c_ee = 0, c_ib = 0, c_bd = R0, c_p1 = p_done;
  if (b0 < b1) {
    c_eb = S.ent_ptr[b0];
    c_ee = S.ent_ptr[b0 + 1];
    c_ib = S.inc_base[b0];
    c_bd = S.batch_done[b0];
    c_p1 = A.row_ptr[c_bd];
    const int e = p_lo + threadIdx.x;
    sweep_load1(S, R, A.nrec, e, e < o_hi, c_eb + threadIdx.x, c_eb + (int)threadIdx.x < c_ee, cur);
    sweep_load2(S, A.u, A.dir, c_ib, cur);
  }
  for (int b = b0; b < b1; ++b) {
    const int e = p_lo + (b - b0) * NB + threadIdx.x;
    // (1) level-1 loads of batch b+1 while batch b is processed
    const bool has_next = b + 1 < b1;
    int n_eb = 0, n_ee = 0, n_ib = 0, n_bd = c_bd, n_p1 = c_p1;
    if (has_next) {
      n_eb = S.ent_ptr[b + 1];
      n_ee = S.ent_ptr[b + 2];
      n_ib = S.inc_base[b + 1];
      n_bd = S.batch_done[b + 1];
    }
    sweep_load1(S, R, A.nrec, e + NB, has_next && e + NB < o_hi, n_eb + threadIdx.x,
                has_next && n_eb + (int)threadIdx.x < n_ee, nxt);
    // (2) phase A: element gradient / Hessian of batch b into shared memory
    if (cur.elem_ok) {
      Real g[3], H[6];
      if ((WANT & W_E) && e >= o_lo && cur.t.wflag) {
        double ee;
        tri_full<Real, FAM, true>(P, cur.v, cur.t, g, H, &ee);
        eacc += ee;
      } else {
        tri_full<Real, FAM>(P, cur.v, cur.t, g, H);
      }
      if (WANT & W_H) {
        Real* hs = sH + threadIdx.x;
        hs[0 * NB] = H[0]; hs[1 * NB] = H[1]; hs[2 * NB] = H[2];
        hs[3 * NB] = H[1]; hs[4 * NB] = H[3]; hs[5 * NB] = H[4];
        hs[6 * NB] = H[2]; hs[7 * NB] = H[4]; hs[8 * NB] = H[5];
      }
      if (WANT & W_G) {
#pragma unroll
        for (int k = 0; k < 3; ++k) sG[k * NB + threadIdx.x] = g[k];
      }
    }
    // (3) level-2 loads of batch b+1
    if (has_next) {
      sweep_load2(S, A.u, A.dir, n_ib, nxt);
      n_p1 = A.row_ptr[n_bd];
    }
    __syncthreads();
    // (4) phase B: row entries of batch b (prefetched entry + rare overflow entries)
    if (cur.ent_ok) {
      const int cnt = cur.meta >> 16;
      Real gs = Real(0);
#pragma unroll
      for (int k = 0; k < kPfWords; ++k)
        if (k < cnt) sweep_reduce_word<Real, WANT, NB>(cur.w[k], cur.pos, sH, sG, swin, S.win_mask, gs);
      for (int k = kPfWords; k < cnt; ++k)
        sweep_reduce_word<Real, WANT, NB>(__ldg(S.inc_word + c_ib + (cur.meta & 0xffffu) + k), cur.pos, sH, sG,
                                          swin, S.win_mask, gs);
      if (WANT & W_G) sgw[cur.row & S.rwin_mask] += gs;
    }
    for (int ent = c_eb + NB + threadIdx.x; ent < c_ee; ent += NB) {
      const int r = __ldg(S.ent_row + ent);
      const int pos0 = __ldg(S.ent_pos + ent);
      const unsigned meta = __ldg(S.ent_meta + ent);
      const unsigned* __restrict__ iw = S.inc_word + c_ib + (meta & 0xffffu);
      Real gs = Real(0);
      for (int k = 0; k < (int)(meta >> 16); ++k)
        sweep_reduce_word<Real, WANT, NB>(__ldg(iw + k), pos0, sH, sG, swin, S.win_mask, gs);
      if (WANT & W_G) sgw[r & S.rwin_mask] += gs;
    }
    __syncthreads();
    // (5) phase C: stream out the rows that are now final
    if (c_bd > done) {
      if (WANT & W_H)
        for (int q = p_done + threadIdx.x; q < c_p1; q += NB) {
          hess[q] = (HOut)swin[q & S.win_mask];
          swin[q & S.win_mask] = Real(0);
        }
      for (int r = done + threadIdx.x; r < c_bd; r += NB) {
        const int gp = S.gpos_identity ? r : A.row_gpos[r];
        if (WANT & W_G) {
          grad[gp] = (double)sgw[r & S.rwin_mask] - (A.rhs ? A.rhs[gp] : 0.0);
          sgw[r & S.rwin_mask] = Real(0);
        }
        if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
      }
      done = c_bd;
      p_done = c_p1;
    }
    cur = nxt;
    c_eb = n_eb;
    c_ee = n_ee;
    c_ib = n_ib;
    c_bd = n_bd;
    c_p1 = n_p1;
  }
  if (done < R1) {  // rows no element of the segment touches (gradient-only rows)
    __syncthreads();
    const int p1 = A.row_ptr[R1];
    if (WANT & W_H)
      for (int q = p_done + threadIdx.x; q < p1; q += NB) hess[q] = (HOut)swin[q & S.win_mask];
    for (int r = done + threadIdx.x; r < R1; r += NB) {
      const int gp = S.gpos_identity ? r : A.row_gpos[r];
      if (WANT & W_G) grad[gp] = (double)sgw[r & S.rwin_mask] - (A.rhs ? A.rhs[gp] : 0.0);
      if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
    }
  }
  if (WANT & W_E) energy_finalize(eacc, eo);
}

// ---------------------------------------------------------------------------
// Push variant of the banded sweep (P1 triangles, kernel_variant 3): same
// segments, batches and streamed row windows, but every element thread adds
// its 3 x 3 Hessian and 3 gradient entries straight into the shared-memory
// windows with shared-memory atomics (positions = row start + the element's
// 7-bit column offsets), so no row entries, incidence words or staged
// element matrices are needed.  Sums of three or more contributions to one
// entry within a batch are not bit-reproducible from run to run (FP32/FP64
// rounding order); the pull sweep above is.
// ---------------------------------------------------------------------------
template <typename Real>
struct PushPf {
  TriElem<Real> t;
  Real v[3];
  unsigned long long off;
  int row[3], pos[3];
  bool ok;
};

template <typename Real>
__device__ __forceinline__ void push_load1(const SweepArgs& S, const Chunk* __restrict__ R, int nrec, int e, bool ok,
                                           PushPf<Real>& f) {
  f.ok = ok;
  if (ok) {
    load_tri(R, nrec, e, f.t);
    f.off = __ldg(S.eoff + e);
  }
}

template <typename Real>
__device__ __forceinline__ void push_load2(const RowArgs& A, const SweepArgs& S, PushPf<Real>& f) {
  if (!f.ok) return;
  const long long n_owned = A.n_rows;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int code = f.t.src[k];
    f.v[k] = (Real)gather(A.u, A.dir, code, 0);
    const long long g = (long long)code - A.lo;
    const int r = (code >= 0 && g >= 0 && g < n_owned) ? __ldg(S.row_of + g) : -1;
    f.row[k] = r;
    f.pos[k] = r >= 0 ? __ldg(A.row_ptr + r) : 0;
  }
}

template <typename Real, int FAM, int WANT, typename HOut, int NB>
__global__ void __launch_bounds__(NB, 2) k_push_tri(RowArgs A, SweepArgs S, const Chunk* __restrict__ R, Phys P,
                                                    double* __restrict__ grad, HOut* __restrict__ hess,
                                                    EnergyOut eo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* swin = reinterpret_cast<Real*>(smem_raw);  // [win_mask + 1]
  Real* sgw = swin + (S.win_mask + 1);             // [rwin_mask + 1]
  const int seg = blockIdx.x;
  const int R0 = S.seg_row[seg], R1 = S.seg_row[seg + 1];
  const int p_lo = S.seg_elem[3 * seg], o_lo = S.seg_elem[3 * seg + 1], o_hi = S.seg_elem[3 * seg + 2];
  const int b0 = S.seg_batch[seg], b1 = S.seg_batch[seg + 1];
  if (WANT & W_H)
    for (int j = threadIdx.x; j <= S.win_mask; j += NB) swin[j] = Real(0);
  if (WANT & W_G)
    for (int j = threadIdx.x; j <= S.rwin_mask; j += NB) sgw[j] = Real(0);
  double eacc = 0.0;
  int done = R0;
  int p_done = A.row_ptr[R0];
  PushPf<Real> cur, nxt;
  int c_bd = R0, c_p1 = p_done;
  if (b0 < b1) {
    c_bd = S.batch_done[b0];
    c_p1 = A.row_ptr[c_bd];
    const int e = p_lo + threadIdx.x;
    push_load1(S, R, A.nrec, e, e < o_hi, cur);
    push_load2(A, S, cur);
  }
  __syncthreads();
  for (int b = b0; b < b1; ++b) {
    const int e = p_lo + (b - b0) * NB + threadIdx.x;
    const bool has_next = b + 1 < b1;
    int n_bd = c_bd, n_p1 = c_p1;
    if (has_next) n_bd = S.batch_done[b + 1];
    push_load1(S, R, A.nrec, e + NB, has_next && e + NB < o_hi, nxt);
    if (cur.ok) {
      Real g[3], H[6];
      tri_full<Real, FAM>(P, cur.v, cur.t, g, H);
      if ((WANT & W_E) && e >= o_lo && cur.t.wflag) eacc += tri_energy_r<Real, FAM>(P, cur.v, cur.t);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int r = cur.row[a];
        if (r < R0 || r >= R1) continue;
        if (WANT & W_G) atomicAdd(sgw + (r & S.rwin_mask), g[a]);
        if (WANT & W_H) {
          const unsigned bits = (unsigned)(cur.off >> (21 * a)) & 0x1FFFFFu;
#pragma unroll
          for (int bb = 0; bb < 3; ++bb) {
            const unsigned o = (bits >> (kOffBits * bb)) & 127u;
            if (o != kNoCol) atomicAdd(swin + ((cur.pos[a] + (int)o) & S.win_mask), H[sym_index(a, bb)]);
          }
        }
      }
    }
    if (has_next) {
      push_load2(A, S, nxt);
      n_p1 = A.row_ptr[n_bd];
    }
    __syncthreads();
    // stream out the rows that are now final
    if (c_bd > done) {
      if (WANT & W_H)
        for (int q = p_done + threadIdx.x; q < c_p1; q += NB) {
          hess[q] = (HOut)swin[q & S.win_mask];
          swin[q & S.win_mask] = Real(0);
        }
      for (int r = done + threadIdx.x; r < c_bd; r += NB) {
        const int gp = S.gpos_identity ? r : A.row_gpos[r];
        if (WANT & W_G) {
          grad[gp] = (double)sgw[r & S.rwin_mask] - (A.rhs ? A.rhs[gp] : 0.0);
          sgw[r & S.rwin_mask] = Real(0);
        }
        if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
      }
      done = c_bd;
      p_done = c_p1;
    }
    __syncthreads();
    cur = nxt;
    c_bd = n_bd;
    c_p1 = n_p1;
  }
  if (done < R1) {
    const int p1 = A.row_ptr[R1];
    if (WANT & W_H)
      for (int q = p_done + threadIdx.x; q < p1; q += NB) hess[q] = (HOut)swin[q & S.win_mask];
    for (int r = done + threadIdx.x; r < R1; r += NB) {
      const int gp = S.gpos_identity ? r : A.row_gpos[r];
      if (WANT & W_G) grad[gp] = (double)sgw[r & S.rwin_mask] - (A.rhs ? A.rhs[gp] : 0.0);
      if ((WANT & W_E) && A.rhs) eacc -= A.rhs[gp] * A.u[A.lo + gp];
    }
  }
  if (WANT & W_E) energy_finalize(eacc, eo);
}

#include "fne_cluster.cuh"

// ---------------------------------------------------------------------------
// energy-only kernels (element-centric, grid-stride)
// ---------------------------------------------------------------------------
constexpr int kElemThreads = 256;

template <typename Real, int FAM>
__global__ void __launch_bounds__(kElemThreads) k_energy_tri(const Chunk* __restrict__ R, int nrec, int n_el,
                                                             const double* __restrict__ u, const double* __restrict__ dir,
                                                             Phys P, const double* __restrict__ rhs, int n_owned,
                                                             long long lo, EnergyOut eo) {
  double acc = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_el; e += stride) {
    TriElem<Real> t;
    load_tri(R, nrec, e, t);
    if (!t.wflag) continue;
    double vd[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) vd[b] = gather(u, dir, t.src[b], 0);
    acc += tri_energy<Real, FAM>(P, vd, t);
  }
  if (rhs)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += stride) acc -= rhs[i] * u[lo + i];
  energy_finalize(acc, eo);
}

template <typename Real>
__global__ void __launch_bounds__(kElemThreads) k_energy_tet(const Chunk* __restrict__ R, int nrec, int n_el,
                                                             const double* __restrict__ u, const double* __restrict__ dir,
                                                             Phys P, const double* __restrict__ rhs, int n_owned,
                                                             long long lo, EnergyOut eo) {
  double acc = 0.0;
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_el; e += stride) {
    TetElem<Real> t;
    load_tet(R, nrec, e, t);
    if (!t.wflag) continue;
    double yd[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int d = 0; d < 3; ++d) yd[b][d] = gather(u, dir, t.src[b], d);
    acc += he_energy<Real>(P, yd, t);
  }
  if (rhs)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += stride) acc -= rhs[i] * u[lo + i];
  energy_finalize(acc, eo);
}

// ---------------------------------------------------------------------------
// No-allocation energy entry point (fne_energy_p1tri_noalloc).
//
// Same FP64 energy reduction as k_energy_tri, reading the caller's float64
// element arrays directly.  Its scratch (the per-CTA partial sums and the
// last-CTA ticket) is this file-scope device array instead of handle-owned
// memory, so the entry point never allocates.  Host code must not use the
// symbol itself as a device pointer: the device address is obtained once per
// device with cudaGetSymbolAddress (noalloc_scratch below).
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxCtas = 1024;  // grid cap = number of partial sums
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxCtas + 1];  // + ticket slot

__global__ void __launch_bounds__(256) k_energy_tri_soa(int fam, long long n_el, const int* __restrict__ codes,
                                                        const double* __restrict__ dvx,
                                                        const double* __restrict__ dvy,
                                                        const double* __restrict__ vol,
                                                        const double* __restrict__ weights,
                                                        const double* __restrict__ u,
                                                        const double* __restrict__ dir, Phys P,
                                                        const double* __restrict__ rhs, long long n_owned,
                                                        long long lo, EnergyOut eo) {
  double acc = 0.0;
  // 64-bit element index: 3 * e exceeds INT32_MAX once n_el passes 715,827,882.
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n_el; e += stride) {
    const double w = weights ? weights[e] : 1.0;
    if (w == 0.0) continue;
    TriElem<double> t;
    const long long b = 3LL * e;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      t.src[k] = codes[b + k];
      t.dvx[k] = dvx[b + k];
      t.dvy[k] = dvy[b + k];
    }
    t.vol = vol[e];
    t.wflag = 1;
    double vd[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) vd[k] = gather(u, dir, t.src[k], 0);
    acc += w * (fam == FAM_PLAP ? tri_energy<double, FAM_PLAP>(P, vd, t) : tri_energy<double, FAM_GL>(P, vd, t));
  }
  if (rhs)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_owned; i += stride)
      acc -= rhs[i] * u[lo + i];
  energy_finalize(acc, eo);
}

namespace {
// Device address of g_noalloc_scratch on the current device.  It is looked up
// on every call (cudaGetSymbolAddress allocates nothing and is cheap), so a
// module reloaded after cudaDeviceReset or a primary-context re-creation is
// picked up instead of a stale cached address.
int noalloc_scratch(double** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return set_error(FNE_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return FNE_OK;
}
}  // namespace

extern "C" int fne_energy_p1tri_noalloc(int32_t family, int64_t n_elem, const int32_t* codes, const double* dvx,
                                        const double* dvy, const double* vol, const double* weights,
                                        const double* u, const double* dirichlet, const double* params,
                                        const double* rhs, int64_t n_owned, int64_t lo, double* energy,
                                        void* stream) {
  if (family != FNE_PLAPLACE && family != FNE_GINZBURG_LANDAU)
    return set_error(FNE_EINVAL, "fne_energy_p1tri_noalloc: family must be FNE_PLAPLACE or FNE_GINZBURG_LANDAU");
  if (n_elem < 0 || n_elem > (int64_t)INT32_MAX || n_owned < 0 || n_owned > (int64_t)INT32_MAX)
    return set_error(FNE_EBOUNDS,
                     "fne_energy_p1tri_noalloc: n_elem and n_owned must be in [0, 2^31-1] (32-bit indexing)");
  if (!energy || !params || (n_elem > 0 && (!codes || !dvx || !dvy || !vol)) || (rhs && n_owned > 0 && !u))
    return set_error(FNE_EINVAL, "fne_energy_p1tri_noalloc: missing array");
  if (family == FNE_PLAPLACE && !(params[0] > 1.0))
    return set_error(FNE_EINVAL, "fne_energy_p1tri_noalloc: p-Laplace needs p > 1");
  double* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  Phys P{};
  P.p = params[0];
  P.eps = params[0];
  if (family == FNE_GINZBURG_LANDAU) {
    for (int i = 0; i < 9; ++i) P.ip[i] = params[1 + i];
    for (int i = 0; i < 3; ++i) P.w[i] = params[10 + i];
  }
  P.p_is3 = family == FNE_PLAPLACE && params[0] == 3.0;
  int dev = 0, sms = 148;
  cudaError_t ae = cudaGetDevice(&dev);
  if (ae == cudaSuccess) ae = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (ae != cudaSuccess)
    return set_error(FNE_ECUDA, std::string("fne_energy_p1tri_noalloc device query: ") + cudaGetErrorString(ae));
  const int64_t work = std::max<int64_t>(n_elem, n_owned);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)kNoAllocMaxCtas, (int64_t)sms * 8,
                                                                (work + 255) / 256}));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxCtas);
  cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), st);  // the ticket must start at zero
  if (e != cudaSuccess)
    return set_error(FNE_ECUDA, std::string("fne_energy_p1tri_noalloc memset: ") + cudaGetErrorString(e));
  EnergyOut eo{scratch, ticket, energy, nullptr};
  k_energy_tri_soa<<<grid, 256, 0, st>>>(family == FNE_PLAPLACE ? FAM_PLAP : FAM_GL, (long long)n_elem, codes, dvx, dvy,
                                         vol, weights, u, dirichlet, P, rhs, (long long)n_owned, (long long)lo, eo);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(FNE_ECUDA, std::string("fne_energy_p1tri_noalloc launch: ") + cudaGetErrorString(e));
  return FNE_OK;
}

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
struct fne_handle {
  McHandle* mc = nullptr;  // Mohr-Coulomb handles delegate to fne_mc.cu
  Mc3dHandle* mc3 = nullptr;  // 3-D Mohr-Coulomb handles delegate to fne_mc3d.cu
  int family = 0, precision = 0, hess_fp32 = 0, npe = 0, bs = 0;
  int64_t n_total = 0, n_free = 0, lo = 0, hi = 0, nnz = 0;
  int n_rows = 0, n_local = 0, n_dir_only = 0, rows_per_cta = 0, grid_rows = 0;
  int tet_lanes = 1;  // lanes per output row of the tet row kernel (1, 2, 4, 8)
  int64_t n_inc = 0;
  int max_row_len = 0;
  size_t smem_bytes = 0;
  int device = 0, num_sms = 148;
  bool use_inc = false;
  bool use_sweep = false;
  bool use_push = false;
  // row-cluster kernel (P1 triangles, default)
  bool use_cluster = false;
  int cl_n_jobs = 0, cl_n_cl = 0, cl_cap_j = 0, cl_cap_r = 0, cl_cap_u = 0, cl_cap_i = 0, cl_cap_w = 0;
  long long cl_wait_limit = kClWaitLimit;
  int4* cl_table = nullptr;
  int* cl_codes = nullptr;
  void* cl_reals = nullptr;
  int4* cl_rows = nullptr;
  int4* cl_runs = nullptr;
  unsigned* cl_incs = nullptr;
  int* err = nullptr;       // status word of the row-cluster kernel
  int* err_host = nullptr;  // pinned copy after each pass
  unsigned long long* sw_eoff = nullptr;
  int* sw_row_of = nullptr;
  int sweep_nb = 0, sweep_win_mask = 0, sweep_rwin_mask = 0;
  int *sw_seg_row = nullptr, *sw_seg_elem = nullptr, *sw_seg_batch = nullptr, *sw_batch_done = nullptr,
      *sw_ent_ptr = nullptr, *sw_inc_base = nullptr, *sw_ent_row = nullptr, *sw_ent_pos = nullptr;
  int sw_gpos_identity = 0;
  unsigned *sw_ent_meta = nullptr, *sw_inc_word = nullptr;
  int inc_max_rank = 0, inc_max_rows = 0, inc_max_len = 0;
  // element-parallel tet pass: per-element blocks + contribution lists
  bool use_elem2 = false;
  int grid_elem2 = 1;
  void *e2_kbuf = nullptr, *e2_gbuf = nullptr;
  int e2_rnodes = 0;
  int *bp_rn_blk = nullptr, *bp_rn_con = nullptr, *bp_rn_row = nullptr, *bp_rn_gpos = nullptr,
      *bp_rn_inc = nullptr, *bp_con = nullptr, *bp_inc = nullptr;
  unsigned* bp_blk = nullptr;
  int64_t e2_contrib = 0;
  Phys phys{};
  // device buffers
  Chunk* rec = nullptr;
  Chunk* rec_dir_only = nullptr;
  int *row_ptr = nullptr, *row_node = nullptr, *row_gpos = nullptr, *inc_ptr = nullptr, *inc_elem = nullptr;
  unsigned char* row_comp = nullptr;
  unsigned* inc_info = nullptr;
  int *cta_row = nullptr, *cta_inc = nullptr, *inc_elem2 = nullptr;
  unsigned* inc_word = nullptr;
  unsigned short* inc_rowl = nullptr;
  double *dir = nullptr, *rhs = nullptr, *partials = nullptr, *dir_const = nullptr;
  unsigned* counter = nullptr;
  int n_partials = 0;
  int64_t device_bytes = 0;
  // device staging for fne_eval_host (allocated on first use)
  double *h_u = nullptr, *h_grad = nullptr, *h_energy = nullptr;
  void* h_hess = nullptr;
};

namespace {

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(FNE_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
int dalloc(fne_handle* h, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return FNE_OK;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return set_error(FNE_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->device_bytes += (int64_t)(count * sizeof(T));
  return FNE_OK;
}

template <typename T>
int upload(fne_handle* h, T** p, const T* src, size_t count) {
  int rc = dalloc(h, p, count);
  if (rc) return rc;
  if (count == 0) return FNE_OK;
  cudaError_t e = cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy H2D");
  return FNE_OK;
}

void free_handle(fne_handle* h) {
  if (!h) return;
  if (h->mc) mc_destroy(h->mc);
  if (h->mc3) mc3d_destroy(h->mc3);
  void* ptrs[] = {h->rec, h->rec_dir_only, h->row_ptr, h->row_node, h->row_gpos, h->inc_ptr, h->inc_elem,
                  h->row_comp, h->inc_info, h->cta_row, h->cta_inc, h->inc_elem2, h->inc_word, h->inc_rowl,
                  h->sw_seg_row, h->sw_seg_elem, h->sw_seg_batch, h->sw_batch_done, h->sw_ent_ptr, h->sw_inc_base,
                  h->sw_ent_row, h->sw_ent_pos, h->sw_ent_meta, h->sw_inc_word, h->sw_eoff, h->sw_row_of,
                  h->dir, h->rhs, h->partials, h->dir_const, h->counter, h->h_u, h->h_grad, h->h_energy,
                  h->h_hess, h->e2_kbuf, h->e2_gbuf, h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row,
                  h->bp_rn_gpos, h->bp_rn_inc, h->bp_con, h->bp_inc, h->bp_blk, h->cl_table,
                  h->cl_codes, h->cl_reals, h->cl_rows, h->cl_runs, h->cl_incs, h->err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->err_host) cudaFreeHost(h->err_host);
  delete h;
}

// ---- packing of the reference's float64 arrays into chunk planes ----------
inline void put_i(Chunk* R, size_t n, int plane, size_t e, int a, int b, int c, int d) {
  int v[4] = {a, b, c, d};
  std::memcpy(R[plane * n + e].w, v, 16);
}
inline void put_f(Chunk* R, size_t n, int plane, size_t e, float a, float b, float c, float d) {
  float v[4] = {a, b, c, d};
  std::memcpy(R[plane * n + e].w, v, 16);
}
inline void put_d(Chunk* R, size_t n, int plane, size_t e, double a, double b) {
  double v[2] = {a, b};
  std::memcpy(R[plane * n + e].w, v, 16);
}
inline double bits_as_double(int lo_word) {
  int v[2] = {lo_word, 0};
  double d;
  std::memcpy(&d, v, 8);
  return d;
}

void pack_tri(const fne_desc* d, bool f32, const std::vector<int64_t>& elems, const std::vector<int32_t>& code,
              const std::vector<uint8_t>* weight, std::vector<Chunk>& out) {
  const size_t n = elems.size();
  out.assign(n * (f32 ? 3 : 5), Chunk{});
  for (size_t i = 0; i < n; ++i) {
    const int64_t e = elems[i];
    const double* dx = d->e0 + e * 3;
    const double* dy = d->e1 + e * 3;
    const double vol = d->e2[e];
    const int w = weight ? (*weight)[i] : 1;
    put_i(out.data(), n, 0, i, code[i * 3], code[i * 3 + 1], code[i * 3 + 2], w);
    if (f32) {
      put_f(out.data(), n, 1, i, (float)dx[0], (float)dx[1], (float)dx[2], (float)vol);
      put_f(out.data(), n, 2, i, (float)dy[0], (float)dy[1], (float)dy[2], 0.f);
    } else {
      put_d(out.data(), n, 1, i, vol, dx[0]);
      put_d(out.data(), n, 2, i, dx[1], dx[2]);
      put_d(out.data(), n, 3, i, dy[0], dy[1]);
      put_d(out.data(), n, 4, i, dy[2], 0.0);
    }
  }
}

void pack_tet(const fne_desc* d, bool f32, const std::vector<int64_t>& elems, const std::vector<int32_t>& code,
              const std::vector<uint8_t>* weight, std::vector<Chunk>& out) {
  const size_t n = elems.size();
  out.assign(n * (f32 ? 5 : 8), Chunk{});
  for (size_t i = 0; i < n; ++i) {
    const int64_t e = elems[i];
    const double* gx = d->e0 + e * 4;
    const double* gy = d->e1 + e * 4;
    const double* gz = d->e2 + e * 4;
    const double vol = d->e3[e];
    const int w = weight ? (*weight)[i] : 1;
    put_i(out.data(), n, 0, i, code[i * 4], code[i * 4 + 1], code[i * 4 + 2], code[i * 4 + 3]);
    if (f32) {
      float wf;
      std::memcpy(&wf, &w, 4);
      put_f(out.data(), n, 1, i, (float)gx[0], (float)gx[1], (float)gx[2], (float)gx[3]);
      put_f(out.data(), n, 2, i, (float)gy[0], (float)gy[1], (float)gy[2], (float)gy[3]);
      put_f(out.data(), n, 3, i, (float)gz[0], (float)gz[1], (float)gz[2], (float)gz[3]);
      put_f(out.data(), n, 4, i, (float)vol, wf, 0.f, 0.f);
    } else {
      put_d(out.data(), n, 1, i, gx[0], gx[1]);
      put_d(out.data(), n, 2, i, gx[2], gx[3]);
      put_d(out.data(), n, 3, i, gy[0], gy[1]);
      put_d(out.data(), n, 4, i, gy[2], gy[3]);
      put_d(out.data(), n, 5, i, gz[0], gz[1]);
      put_d(out.data(), n, 6, i, gz[2], gz[3]);
      put_d(out.data(), n, 7, i, vol, bits_as_double(w));
    }
  }
}

// job records of the row-cluster kernel (layout in fne_cluster.cuh)
template <typename Real>
void pack_cluster_jobs(const fne_desc* d, const RowPlan& P, const ClusterPlan& Q, std::vector<int32_t>& codes,
                       std::vector<Real>& reals) {
  const size_t n = Q.job_elem.size();
  codes.assign(3 * n, -1);  // padding jobs: a valid gather code (the Dirichlet value of DOF 0)
  reals.assign(7 * n, Real(0));
  for (size_t j = 0; j < n; ++j) {
    const int32_t le = Q.job_elem[j];
    if (le < 0) continue;
    const int64_t e = P.local_elems[le];
    reals[j] = (Real)d->e2[e];
    for (int a = 0; a < 3; ++a) {
      codes[a * n + j] = P.elem_code[(size_t)le * 3 + a];
      reals[(1 + a) * n + j] = (Real)d->e0[e * 3 + a];
      reals[(4 + a) * n + j] = (Real)d->e1[e * 3 + a];
    }
  }
}

bool is_tri(int fam) { return fam == FNE_PLAPLACE || fam == FNE_GINZBURG_LANDAU; }

// ---- kernel dispatch -------------------------------------------------------
template <typename Real, int FAM, typename HOut>
cudaError_t launch_tri_t(fne_handle* h, int want, const RowArgs& A, const IncArgs& Q, const SweepArgs& SW,
                         double* grad, void* hess, EnergyOut eo, cudaStream_t st, bool set_attr) {
  HOut* H = static_cast<HOut*>(hess);
  const ClusterArgs CL{h->cl_table,  h->cl_codes, h->cl_reals, h->cl_rows,  h->cl_runs,
                       h->cl_incs,   h->err,      h->cl_wait_limit, h->cl_n_jobs, h->cl_cap_j,
                       h->cl_cap_r,  h->cl_cap_u, h->cl_cap_i, h->cl_cap_w};
  const size_t sm = h->smem_bytes;
  const dim3 grid(h->grid_rows);
  constexpr int NBS = sizeof(Real) == 4 ? 512 : 256;
#define FNE_TRI_CASE(W)                                                                                        \
  case W:                                                                                                      \
    if (h->use_cluster) {                                                                                      \
      if (set_attr)                                                                                            \
        return cudaFuncSetAttribute(k_cluster_tri<Real, FAM, W, HOut>,                                        \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);                     \
      k_cluster_tri<Real, FAM, W, HOut><<<grid, kClThreads, sm, st>>>(A, CL, h->phys, grad, H, eo, h->cl_n_cl); \
    } else if (h->use_push) {                                                                                  \
      if (set_attr)                                                                                            \
        return cudaFuncSetAttribute(k_push_tri<Real, FAM, W, HOut, NBS>,                                      \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);                     \
      k_push_tri<Real, FAM, W, HOut, NBS><<<grid, NBS, sm, st>>>(A, SW, h->rec, h->phys, grad, H, eo);        \
    } else if (h->use_sweep) {                                                                                 \
      if (set_attr)                                                                                            \
        return cudaFuncSetAttribute(k_sweep_tri<Real, FAM, W, HOut, NBS>,                                     \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);                     \
      k_sweep_tri<Real, FAM, W, HOut, NBS><<<grid, NBS, sm, st>>>(A, SW, h->rec, h->phys, grad, H, eo);       \
    } else if (h->use_inc) {                                                                                          \
      if (set_attr)                                                                                            \
        return cudaFuncSetAttribute(k_inc_tri<Real, FAM, W, HOut>,                                            \
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);                     \
      k_inc_tri<Real, FAM, W, HOut><<<grid, kIncThreads, sm, st>>>(A, Q, h->rec, h->phys, grad, H, eo);        \
    } else {                                                                                                   \
      if (set_attr)                                                                                            \
        return cudaFuncSetAttribute(k_rows_tri<Real, FAM, W, HOut>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                    (int)sm);                                                                  \
      k_rows_tri<Real, FAM, W, HOut><<<grid, kTriRows, (W & W_H) ? sm : 0, st>>>(A, h->rec, h->phys, grad, H, eo); \
    }                                                                                                          \
    return cudaGetLastError();
  switch (want) {
    FNE_TRI_CASE(2)
    FNE_TRI_CASE(3)
    FNE_TRI_CASE(4)
    FNE_TRI_CASE(5)
    FNE_TRI_CASE(6)
    FNE_TRI_CASE(7)
  }
#undef FNE_TRI_CASE
  return cudaErrorInvalidValue;
}

template <typename Real, typename HOut, int G>
cudaError_t launch_tet_g(fne_handle* h, int want, const RowArgs& A, double* grad, void* hess, EnergyOut eo,
                         cudaStream_t st, bool set_attr) {
  HOut* H = static_cast<HOut*>(hess);
  const dim3 grid(h->grid_rows), block(kTetRows);
  const size_t sm = (want & W_H) ? h->smem_bytes : 0;
#define FNE_TET_CASE(W)                                                                                       \
  case W:                                                                                                     \
    if (set_attr)                                                                                             \
      return cudaFuncSetAttribute(k_rows_tet<Real, W, HOut, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)h->smem_bytes);                                                        \
    k_rows_tet<Real, W, HOut, G><<<grid, block, sm, st>>>(A, h->rec, h->phys, grad, H, eo);                    \
    return cudaGetLastError();
  switch (want) {
    FNE_TET_CASE(2)
    FNE_TET_CASE(3)
    FNE_TET_CASE(4)
    FNE_TET_CASE(5)
    FNE_TET_CASE(6)
    FNE_TET_CASE(7)
  }
#undef FNE_TET_CASE
  return cudaErrorInvalidValue;
}

template <typename Real, typename HOut>
cudaError_t launch_tet_t(fne_handle* h, int want, const RowArgs& A, double* grad, void* hess, EnergyOut eo,
                         cudaStream_t st, bool set_attr) {
  switch (h->tet_lanes) {
    case 2: return launch_tet_g<Real, HOut, 2>(h, want, A, grad, hess, eo, st, set_attr);
    case 4: return launch_tet_g<Real, HOut, 4>(h, want, A, grad, hess, eo, st, set_attr);
    case 8: return launch_tet_g<Real, HOut, 8>(h, want, A, grad, hess, eo, st, set_attr);
    default: return launch_tet_g<Real, HOut, 1>(h, want, A, grad, hess, eo, st, set_attr);
  }
}

template <typename Real, typename HOut>
cudaError_t launch_elem2_t(fne_handle* h, int want, const double* u, double* grad, void* hess, EnergyOut eo,
                           cudaStream_t st) {
  Real* kb = static_cast<Real*>(h->e2_kbuf);
  Real* gb = static_cast<Real*>(h->e2_gbuf);
  const int n_owned = (int)(h->hi - h->lo);
  const dim3 grid(h->grid_elem2), block(256);
#define FNE_E2_CASE(W)                                                                                      \
  case W:                                                                                                   \
    k_he_elem<Real, W><<<grid, block, 0, st>>>(h->rec, h->n_local, u, h->dir, h->phys, kb, gb, h->rhs,      \
                                               n_owned, h->lo, eo);                                         \
    break;
  switch (want) {
    FNE_E2_CASE(2)
    FNE_E2_CASE(3)
    FNE_E2_CASE(4)
    FNE_E2_CASE(5)
    FNE_E2_CASE(6)
    FNE_E2_CASE(7)
    default:
      return cudaErrorInvalidValue;
  }
#undef FNE_E2_CASE
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (h->e2_rnodes == 0) return cudaSuccess;
  NodeGatherArgs G{h->e2_rnodes, h->bp_rn_blk, h->bp_rn_con, h->bp_rn_row, h->bp_rn_gpos,
                   h->bp_rn_inc, h->bp_blk, h->bp_con, h->bp_inc, h->rhs};
  const int gg = std::max(1, std::min(h->num_sms * 16, (h->e2_rnodes + 7) / 8));
  HOut* H = static_cast<HOut*>(hess);
  if ((want & W_H) && (want & W_G))
    k_node_gather<Real, HOut, 3, 4, true, true><<<gg, 256, 0, st>>>(G, kb, gb, H, grad);
  else if (want & W_H)
    k_node_gather<Real, HOut, 3, 4, true, false><<<gg, 256, 0, st>>>(G, kb, gb, H, grad);
  else if (want & W_G)
    k_node_gather<Real, HOut, 3, 4, false, true><<<gg, 256, 0, st>>>(G, kb, gb, H, grad);
  return cudaGetLastError();
}

cudaError_t launch_elem2(fne_handle* h, int want, const double* u, double* grad, void* hess, EnergyOut eo,
                         cudaStream_t st) {
  if (h->precision == FNE_FP64) return launch_elem2_t<double, double>(h, want, u, grad, hess, eo, st);
  if (h->hess_fp32) return launch_elem2_t<float, float>(h, want, u, grad, hess, eo, st);
  return launch_elem2_t<float, double>(h, want, u, grad, hess, eo, st);
}

cudaError_t launch_rows(fne_handle* h, int want, const RowArgs& A, const IncArgs& Q, const SweepArgs& SW,
                        double* grad, void* hess, EnergyOut eo, cudaStream_t st, bool set_attr) {
  const bool f32 = h->precision == FNE_FP32;
  const bool h32 = f32 && h->hess_fp32;
  if (h->family == FNE_PLAPLACE) {
    if (!f32) return launch_tri_t<double, FAM_PLAP, double>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
    if (h32) return launch_tri_t<float, FAM_PLAP, float>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
    return launch_tri_t<float, FAM_PLAP, double>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
  }
  if (h->family == FNE_GINZBURG_LANDAU) {
    if (!f32) return launch_tri_t<double, FAM_GL, double>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
    if (h32) return launch_tri_t<float, FAM_GL, float>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
    return launch_tri_t<float, FAM_GL, double>(h, want, A, Q, SW, grad, hess, eo, st, set_attr);
  }
  if (h->family == FNE_NEOHOOKEAN) {
    if (!f32) return launch_tet_t<double, double>(h, want, A, grad, hess, eo, st, set_attr);
    if (h32) return launch_tet_t<float, float>(h, want, A, grad, hess, eo, st, set_attr);
    return launch_tet_t<float, double>(h, want, A, grad, hess, eo, st, set_attr);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_energy(fne_handle* h, const Chunk* rec, int n_el, const double* u, const double* rhs, int n_owned,
                          EnergyOut eo, cudaStream_t st) {
  const bool f32 = h->precision == FNE_FP32;
  int grid = std::max(1, std::min(h->num_sms * 8, (std::max(n_el, n_owned) + kElemThreads - 1) / kElemThreads));
  grid = std::min(grid, h->n_partials);
  const long long lo = h->lo;
  if (h->family == FNE_PLAPLACE) {
    if (f32)
      k_energy_tri<float, FAM_PLAP><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs, n_owned,
                                                                   lo, eo);
    else
      k_energy_tri<double, FAM_PLAP><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs,
                                                                    n_owned, lo, eo);
  } else if (h->family == FNE_GINZBURG_LANDAU) {
    if (f32)
      k_energy_tri<float, FAM_GL><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs, n_owned,
                                                                 lo, eo);
    else
      k_energy_tri<double, FAM_GL><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs, n_owned,
                                                                  lo, eo);
  } else if (h->family == FNE_NEOHOOKEAN) {
    if (f32)
      k_energy_tet<float><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs, n_owned, lo, eo);
    else
      k_energy_tet<double><<<grid, kElemThreads, 0, st>>>(rec, n_el, n_el, u, h->dir, h->phys, rhs, n_owned, lo, eo);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// energy of the elements without any free DOF (constant w.r.t. u)
int refresh_dir_const(fne_handle* h) {
  if (!h->dir_const) return FNE_OK;
  cudaError_t e;
  if (h->n_dir_only == 0) {
    e = cudaMemset(h->dir_const, 0, sizeof(double));
  } else {
    EnergyOut eo{h->partials, h->counter, h->dir_const, nullptr};
    // every node of these elements is a Dirichlet node: u is never read
    e = launch_energy(h, h->rec_dir_only, h->n_dir_only, h->dir, nullptr, 0, eo, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) return cuda_fail(e, "Dirichlet-only energy");
  return FNE_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int fne_create(const fne_desc* d, fne_handle** out) {
  if (!d || !out) return set_error(FNE_EINVAL, "fne_create: null argument");
  *out = nullptr;
  if (d->precision != FNE_FP64 && d->precision != FNE_FP32)
    return set_error(FNE_EINVAL, "fne_create: precision must be FNE_FP64 or FNE_FP32");
  int npe_expect = 0, bs_expect = 0;
  if (is_tri(d->family)) {
    npe_expect = 3;
    bs_expect = 1;
  } else if (d->family == FNE_NEOHOOKEAN) {
    npe_expect = 4;
    bs_expect = 3;
  } else if (d->family == FNE_MOHR_COULOMB) {
    if (d->n_elem < 0 || d->n_total < 0 || d->nnz < 0 || (d->n_elem > 0 && !d->elems) || !d->total_to_free_reord ||
        (d->nnz > 0 && (!d->owned_rows || !d->owned_cols)) || (d->n_total > 0 && !d->dirichlet))
      return set_error(FNE_EINVAL, "fne_create: missing array");
    McHandle* mc = nullptr;
    int rc = mc_create(d, &mc);
    if (rc) return rc;
    auto* h = new (std::nothrow) fne_handle();
    if (!h) {
      mc_destroy(mc);
      return set_error(FNE_ENOMEM, "fne_create: out of host memory");
    }
    h->mc = mc;
    h->family = d->family;
    h->precision = d->precision;
    h->hess_fp32 = d->precision == FNE_FP32 && d->hess_fp32;
    h->n_total = d->n_total;
    h->n_free = d->n_free;
    h->lo = d->lo;
    h->hi = d->hi;
    h->nnz = d->nnz;
    *out = h;
    return FNE_OK;
  } else if (d->family == FNE_MOHR_COULOMB_3D) {
    if (d->n_elem < 0 || d->n_total < 0 || d->nnz < 0 || (d->n_elem > 0 && !d->elems) || !d->total_to_free_reord ||
        (d->nnz > 0 && (!d->owned_rows || !d->owned_cols)) || (d->n_total > 0 && !d->dirichlet))
      return set_error(FNE_EINVAL, "fne_create: missing array");
    if (d->precision != FNE_FP64 && d->precision != FNE_FP32)
      return set_error(FNE_EINVAL, "fne_create: precision must be FNE_FP64 or FNE_FP32");
    Mc3dHandle* m3 = nullptr;
    int rc = mc3d_create(d, &m3);
    if (rc) return rc;
    auto* h = new (std::nothrow) fne_handle();
    if (!h) {
      mc3d_destroy(m3);
      return set_error(FNE_ENOMEM, "fne_create: out of host memory");
    }
    h->mc3 = m3;
    h->family = d->family;
    h->precision = d->precision;
    h->hess_fp32 = d->precision == FNE_FP32 && d->hess_fp32;
    h->n_total = d->n_total;
    h->n_free = d->n_free;
    h->lo = d->lo;
    h->hi = d->hi;
    h->nnz = d->nnz;
    *out = h;
    return FNE_OK;
  } else {
    return set_error(FNE_EINVAL, "fne_create: unknown family");
  }
  if (d->npe != npe_expect || d->block_size != bs_expect)
    return set_error(FNE_EINVAL, "fne_create: npe/block_size do not match the family");
  if (d->n_elem < 0 || d->n_total < 0 || d->nnz < 0 || (d->n_elem > 0 && !d->elems) || !d->total_to_free_reord ||
      (d->nnz > 0 && (!d->owned_rows || !d->owned_cols)) || (d->n_total > 0 && !d->dirichlet))
    return set_error(FNE_EINVAL, "fne_create: missing array");
  if (d->n_elem > 0 && (!d->e0 || !d->e1 || !d->e2 || (d->family == FNE_NEOHOOKEAN && !d->e3)))
    return set_error(FNE_EINVAL, "fne_create: missing element data");
  if (d->family == FNE_PLAPLACE && !(d->s[0] > 1.0))
    return set_error(FNE_EINVAL, "fne_create: p-Laplace needs p > 1");

  RowPlan plan;
  int rc = build_row_plan(d, plan);
  if (rc) return rc;
  const bool f32 = d->precision == FNE_FP32;
  const size_t real_size = f32 ? sizeof(float) : sizeof(double);

  int dev_id = 0, n_sms = 148, smem_optin = 227 * 1024;
  cudaGetDevice(&dev_id);
  cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev_id);
  cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev_id);
  if (smem_optin <= 0) smem_optin = 227 * 1024;
  // banded sweep for triangles (default), incidence-parallel on request,
  // else the row-gather kernel
  IncPlan inc;
  SweepPlan sweep;
  bool use_inc = false, use_sweep = false;
  const int sweep_nb = f32 ? 512 : 256;
  if (is_tri(d->family) && plan.n_rows > 0 && d->kernel_variant == 2)
    use_inc = build_inc_plan(plan, kIncThreads, inc);
  const bool want_push = is_tri(d->family) && d->kernel_variant == 3;
  // row clusters for triangles (default): windows of at most 8191 slots, sized
  // for three CTAs per SM, and about as many clusters as a whole number of
  // waves of them
  ClusterPlan cplan;
  bool use_cluster = false;
  if (is_tri(d->family) && plan.n_rows > 0 && d->kernel_variant == 8) {
    // one persistent CTA per SM holding two staging buffers and the window:
    // the buffers (jobs, row / run records, incidence words) and the window
    // share the shared memory in the proportion the mesh needs (jobs per row
    // ~ local elements per row plus the cluster border, incidences per row ~
    // 3 x local elements per row), with 10 % slack for irregular clusters;
    // small meshes get smaller clusters so that every SM has several
    const int64_t budget = (int64_t)smem_optin - 1024;
    const double epr = (double)plan.local_elems.size() / (double)plan.n_rows;
    const double jobs_per_row = 1.15 * epr + 0.05, incs_per_row = 3.0 * epr + 0.5;
    const double vals_per_row = (double)d->nnz / (double)plan.n_rows;
    int64_t rows = 4096;
    rows = std::min<int64_t>(rows, std::max<int64_t>(1, plan.n_rows / (4 * (int64_t)n_sms)));
    ClLayout<double> lay{};
    auto fit = [&](int64_t r) {
      lay.cj = (int)std::min<int64_t>(1 << kClJobBits, ((int64_t)(1.1 * r * jobs_per_row) + 19) / 4 * 4);
      lay.ci = (int)(((int64_t)(1.1 * r * incs_per_row) + 19) / 4 * 4);
      lay.cr = (int)(r + r / 4 + 8);
      lay.cu = 128;
      lay.cw = (int)((int64_t)(1.1 * r * vals_per_row) + 16);
      const size_t b = f32 ? ClLayout<float>{lay.cj, lay.cr, lay.cu, lay.ci, lay.cw}.bytes() : lay.bytes();
      return (int64_t)b <= budget;
    };
    for (int it = 0; it < 80 && rows > 1 && !fit(rows); ++it) rows = std::max<int64_t>(1, rows * 19 / 20);
    const bool gid = [&] {
      for (int32_t k = 0; k < plan.n_rows; ++k)
        if (plan.row_gpos[k] != k) return false;
      return true;
    }();
    if (fit(rows))
      use_cluster = build_cluster_plan(plan, d->lo, d->hi, lay.cr, lay.cj, lay.ci, lay.cw, gid, cplan);
    if (use_cluster && cplan.max_runs > lay.cu) use_cluster = false;
  }
  if (is_tri(d->family) && plan.n_rows > 0 &&
      (d->kernel_variant == 0 || (d->kernel_variant == 8 && !use_cluster) || d->kernel_variant == 7 || want_push)) {
    // shared memory per CTA: 12*nb element quantities (pull sweep only) +
    // entry window + row window, sized so that two CTAs fit on one SM
    const int64_t budget = std::min<int64_t>(smem_optin, (228 * 1024) / 2 - 1024) / (int64_t)real_size;
    const int64_t avail = budget - (want_push ? 0 : 12 * (int64_t)sweep_nb);
    // two CTAs per SM when the mesh allows; small meshes get one batch per
    // segment (more re-evaluated boundary strips, but every SM busy)
    const int n_seg = (int)std::max<int64_t>(
        1, std::min<int64_t>(2 * n_sms, (int64_t)plan.local_elems.size() / sweep_nb));
    if (avail > 0)
      use_sweep = build_sweep_plan(plan, sweep_nb, n_seg, (int)(avail * 3 / 4), (int)(avail / 4), sweep);
    if (use_sweep && (want_push ? 0 : 12 * (int64_t)sweep_nb) + sweep.win_entries + sweep.win_rows > budget)
      use_sweep = false;
  }
  // push variant: per-element column offsets and the row index of every owned DOF
  std::vector<unsigned long long> eoff;
  std::vector<int32_t> row_of;
  const bool use_push = use_sweep && want_push;
  if (use_push) {
    eoff.assign(plan.local_elems.size(), ~0ull);
    for (int32_t k = 0; k < plan.n_rows; ++k) {
      const int32_t nd = plan.row_node[k];
      for (int32_t i = plan.inc_ptr[nd]; i < plan.inc_ptr[nd + 1]; ++i) {
        const uint32_t info = plan.inc_info[i];
        const int a = (int)(info & 7u);
        const unsigned long long bits = (info >> kOffShift) & ((1u << (3 * kOffBits)) - 1u);
        unsigned long long& w = eoff[plan.inc_elem[i]];
        w = (w & ~(0x1FFFFFull << (21 * a))) | (bits << (21 * a));
      }
    }
    row_of.assign((size_t)(d->hi - d->lo), -1);
    for (int32_t k = 0; k < plan.n_rows; ++k) row_of[plan.row_gpos[k]] = k;
  }

  auto* h = new (std::nothrow) fne_handle();
  if (!h) return set_error(FNE_ENOMEM, "fne_create: out of host memory");
  h->family = d->family;
  h->precision = d->precision;
  h->hess_fp32 = f32 ? (d->hess_fp32 ? 1 : 0) : 0;
  h->npe = d->npe;
  h->bs = d->block_size;
  h->n_total = d->n_total;
  h->n_free = d->n_free;
  h->lo = d->lo;
  h->hi = d->hi;
  h->nnz = d->nnz;
  h->n_rows = plan.n_rows;
  h->n_local = (int)plan.local_elems.size();
  h->n_dir_only = (int)plan.dir_only.size();
  h->n_inc = (int64_t)plan.inc_elem.size();
  h->max_row_len = plan.max_row_len;
  h->use_inc = use_inc;
  h->use_cluster = use_cluster;
  h->use_sweep = use_sweep && !use_cluster;
  h->use_push = use_push;
  h->phys.p = d->s[0];
  h->phys.eps = d->s[0];
  for (int i = 0; i < 9; ++i) h->phys.ip[i] = d->s[1 + i];
  for (int i = 0; i < 3; ++i) h->phys.w[i] = d->s[10 + i];
  h->phys.C1 = d->s[0];
  h->phys.D1 = d->s[1];
  h->phys.absdet = d->family == FNE_NEOHOOKEAN && d->s[2] != 0.0;
  h->phys.p_is3 = d->family == FNE_PLAPLACE && d->s[0] == 3.0;
  h->phys.pf = (float)h->phys.p;
  h->phys.epsf = (float)h->phys.eps;
  for (int i = 0; i < 9; ++i) h->phys.ipf[i] = (float)h->phys.ip[i];
  for (int i = 0; i < 3; ++i) h->phys.wf[i] = (float)h->phys.w[i];
  h->phys.C1f = (float)h->phys.C1;
  h->phys.D1f = (float)h->phys.D1;
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);

  if (use_cluster) {
    h->cl_n_cl = cplan.n_cl;
    h->grid_rows = std::min(cplan.n_cl, n_sms);
    h->cl_n_jobs = (int)cplan.job_elem.size();
    h->cl_cap_j = cplan.max_jobs;
    h->cl_cap_r = cplan.max_rows;
    h->cl_cap_i = cplan.max_incs;
    h->cl_cap_u = cplan.max_runs;
    h->cl_cap_w = cplan.max_win;
    h->smem_bytes = f32 ? ClLayout<float>{h->cl_cap_j, h->cl_cap_r, h->cl_cap_u, h->cl_cap_i, h->cl_cap_w}.bytes()
                        : ClLayout<double>{h->cl_cap_j, h->cl_cap_r, h->cl_cap_u, h->cl_cap_i, h->cl_cap_w}.bytes();
  } else if (use_sweep) {
    h->grid_rows = sweep.n_seg;
    h->sweep_nb = sweep.nb;
    h->sweep_win_mask = sweep.win_entries - 1;
    h->sweep_rwin_mask = sweep.win_rows - 1;
    h->smem_bytes = ((size_t)(use_push ? 0 : 12 * sweep.nb) + sweep.win_entries + sweep.win_rows) * real_size;
  } else if (use_inc) {
    h->grid_rows = inc.n_cta;
    h->inc_max_rank = inc.max_rank;
    h->inc_max_rows = std::max(1, inc.max_rows);
    h->inc_max_len = inc.max_len;
    h->smem_bytes = (size_t)h->inc_max_rows * (sizeof(int) + real_size) + (size_t)inc.max_len * real_size;
  } else {
    // tets: G lanes per row (kernel_variant 1 = one lane, 4 / 5 / 6 = 2 / 4 / 8
    // lanes; automatic: the fewest lanes giving at least 1024 (FP64) or 512
    // (FP32) row lanes per SM -- measured on the 61,440- and 491,520-tet beams)
    h->tet_lanes = 1;
    if (!is_tri(d->family)) {
      if (d->kernel_variant >= 4 && d->kernel_variant <= 6) {
        h->tet_lanes = 1 << (d->kernel_variant - 3);
      } else if (d->kernel_variant != 1) {
        const int64_t want = (int64_t)h->num_sms * (f32 ? 512 : 1024);
        while (h->tet_lanes < 8 && (int64_t)plan.n_rows * h->tet_lanes < want) h->tet_lanes *= 2;
      }
    }
    h->rows_per_cta = is_tri(d->family) ? kTriRows : kTetRows / h->tet_lanes;
    h->grid_rows = (h->n_rows + h->rows_per_cta - 1) / h->rows_per_cta;
    int64_t max_cta = 0;
    for (int c = 0; c < h->grid_rows; ++c) {
      const int a = c * h->rows_per_cta, b = std::min(h->n_rows, a + h->rows_per_cta);
      max_cta = std::max<int64_t>(max_cta, plan.row_ptr[b] - plan.row_ptr[a]);
    }
    h->smem_bytes = (size_t)max_cta * h->tet_lanes * real_size;
  }
  if (h->smem_bytes > 227 * 1024) {
    free_handle(h);
    return set_error(FNE_EBOUNDS, "fne_create: a CTA's rows exceed shared memory");
  }
  h->n_partials = std::max({h->grid_rows, h->num_sms * 8, 1});

#define FNE_TRY(x)      \
  do {                  \
    rc = (x);           \
    if (rc) {           \
      free_handle(h);   \
      return rc;        \
    }                   \
  } while (0)

  {
    std::vector<Chunk> recs, dro;
    if (is_tri(d->family)) {
      pack_tri(d, f32, plan.local_elems, plan.elem_code, &plan.elem_weight, recs);
      if (d->dirichlet_only_energy) pack_tri(d, f32, plan.dir_only, plan.dir_only_code, nullptr, dro);
    } else {
      pack_tet(d, f32, plan.local_elems, plan.elem_code, &plan.elem_weight, recs);
      if (d->dirichlet_only_energy) pack_tet(d, f32, plan.dir_only, plan.dir_only_code, nullptr, dro);
    }
    FNE_TRY(upload(h, &h->rec, recs.data(), recs.size()));
    FNE_TRY(upload(h, &h->rec_dir_only, dro.data(), dro.size()));
  }
  FNE_TRY(upload(h, &h->row_ptr, plan.row_ptr.data(), plan.row_ptr.size()));
  FNE_TRY(upload(h, &h->row_node, plan.row_node.data(), plan.row_node.size()));
  FNE_TRY(upload(h, &h->row_comp, plan.row_comp.data(), plan.row_comp.size()));
  FNE_TRY(upload(h, &h->row_gpos, plan.row_gpos.data(), plan.row_gpos.size()));
  FNE_TRY(upload(h, &h->inc_ptr, plan.inc_ptr.data(), plan.inc_ptr.size()));
  if (use_cluster) {
    std::vector<int32_t> codes;
    if (f32) {
      std::vector<float> reals;
      pack_cluster_jobs(d, plan, cplan, codes, reals);
      float* dr = nullptr;
      FNE_TRY(upload(h, &dr, reals.data(), reals.size()));
      h->cl_reals = dr;
    } else {
      std::vector<double> reals;
      pack_cluster_jobs(d, plan, cplan, codes, reals);
      double* dr = nullptr;
      FNE_TRY(upload(h, &dr, reals.data(), reals.size()));
      h->cl_reals = dr;
    }
    FNE_TRY(upload(h, &h->cl_codes, codes.data(), codes.size()));
    FNE_TRY(upload(h, &h->cl_table, reinterpret_cast<const int4*>(cplan.table.data()), cplan.table.size() / 4));
    FNE_TRY(upload(h, &h->cl_rows, reinterpret_cast<const int4*>(cplan.rows.data()), cplan.rows.size() / 4));
    FNE_TRY(upload(h, &h->cl_runs, reinterpret_cast<const int4*>(cplan.runs.data()), cplan.runs.size() / 4));
    FNE_TRY(upload(h, &h->cl_incs, cplan.incs.data(), cplan.incs.size()));
    FNE_TRY(dalloc(h, &h->err, 1));
    if (cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess ||
        cudaHostAlloc((void**)&h->err_host, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
      free_handle(h);
      return set_error(FNE_ECUDA, "fne_create: status word");
    }
    *h->err_host = 0;
  }
  if (use_sweep && !use_cluster) {
    FNE_TRY(upload(h, &h->sw_seg_row, sweep.seg_row.data(), sweep.seg_row.size()));
    FNE_TRY(upload(h, &h->sw_seg_elem, sweep.seg_elem.data(), sweep.seg_elem.size()));
    FNE_TRY(upload(h, &h->sw_seg_batch, sweep.seg_batch.data(), sweep.seg_batch.size()));
    FNE_TRY(upload(h, &h->sw_batch_done, sweep.batch_done.data(), sweep.batch_done.size()));
    FNE_TRY(upload(h, &h->sw_ent_ptr, sweep.ent_ptr.data(), sweep.ent_ptr.size()));
    FNE_TRY(upload(h, &h->sw_inc_base, sweep.inc_base.data(), sweep.inc_base.size()));
    FNE_TRY(upload(h, &h->sw_ent_row, sweep.ent_row.data(), sweep.ent_row.size()));
    FNE_TRY(upload(h, &h->sw_ent_pos, sweep.ent_pos.data(), sweep.ent_pos.size()));
    h->sw_gpos_identity = sweep.gpos_identity ? 1 : 0;
    FNE_TRY(upload(h, &h->sw_ent_meta, sweep.ent_meta.data(), sweep.ent_meta.size()));
    FNE_TRY(upload(h, &h->sw_inc_word, sweep.inc_word.data(), sweep.inc_word.size()));
    if (use_push) {
      FNE_TRY(upload(h, &h->sw_eoff, eoff.data(), eoff.size()));
      FNE_TRY(upload(h, &h->sw_row_of, row_of.data(), row_of.size()));
    }
  } else if (use_inc) {
    FNE_TRY(upload(h, &h->cta_row, inc.cta_row.data(), inc.cta_row.size()));
    FNE_TRY(upload(h, &h->cta_inc, inc.cta_inc.data(), inc.cta_inc.size()));
    FNE_TRY(upload(h, &h->inc_elem2, inc.inc_elem.data(), inc.inc_elem.size()));
    FNE_TRY(upload(h, &h->inc_word, inc.inc_word.data(), inc.inc_word.size()));
    FNE_TRY(upload(h, &h->inc_rowl, inc.inc_rowl.data(), inc.inc_rowl.size()));
  } else {
    FNE_TRY(upload(h, &h->inc_elem, plan.inc_elem.data(), plan.inc_elem.size()));
    FNE_TRY(upload(h, &h->inc_info, plan.inc_info.data(), plan.inc_info.size()));
  }
  if (d->family == FNE_NEOHOOKEAN && d->kernel_variant == 2 && plan.n_rows > 0) {
    // element-parallel pass + node-block gather on request (falls back to the
    // row-gather kernel when the pattern is not node-blocked)
    BlockPlan bp;
    std::vector<int64_t> edofs((size_t)h->n_local * 12);
    for (int32_t le = 0; le < h->n_local; ++le)
      for (int i = 0; i < 12; ++i) edofs[(size_t)le * 12 + i] = d->elems[plan.local_elems[le] * 12 + i];
    if (build_block_plan(h->n_local, 4, 3, edofs.data(), d, bp) == FNE_OK &&
        (int64_t)h->n_local * kHeSlots < (int64_t)INT32_MAX) {
      h->use_elem2 = true;
      h->e2_rnodes = bp.n_rnodes;
      h->e2_contrib = (int64_t)bp.con.size();
      h->grid_elem2 = std::max(1, std::min(h->num_sms * 8, (h->n_local + 255) / 256));
      h->n_partials = std::max(h->n_partials, h->grid_elem2);
      FNE_TRY(upload(h, &h->bp_rn_blk, bp.rn_blk.data(), bp.rn_blk.size()));
      FNE_TRY(upload(h, &h->bp_rn_con, bp.rn_con.data(), bp.rn_con.size()));
      FNE_TRY(upload(h, &h->bp_rn_row, bp.rn_row.data(), bp.rn_row.size()));
      FNE_TRY(upload(h, &h->bp_rn_gpos, bp.rn_gpos.data(), bp.rn_gpos.size()));
      FNE_TRY(upload(h, &h->bp_rn_inc, bp.rn_inc.data(), bp.rn_inc.size()));
      FNE_TRY(upload(h, &h->bp_blk, bp.blk.data(), bp.blk.size()));
      FNE_TRY(upload(h, &h->bp_con, bp.con.data(), bp.con.size()));
      FNE_TRY(upload(h, &h->bp_inc, bp.inc.data(), bp.inc.size()));
      unsigned char* kb = nullptr;
      FNE_TRY(dalloc(h, &kb, (size_t)h->n_local * kHeSlots * real_size));
      h->e2_kbuf = kb;
      unsigned char* gb = nullptr;
      FNE_TRY(dalloc(h, &gb, (size_t)h->n_local * 12 * real_size));
      h->e2_gbuf = gb;
    }
  }
  FNE_TRY(upload(h, &h->dir, d->dirichlet, (size_t)d->n_total));
  if (d->rhs_owned) FNE_TRY(upload(h, &h->rhs, d->rhs_owned, (size_t)(d->hi - d->lo)));
  FNE_TRY(dalloc(h, &h->partials, (size_t)h->n_partials));
  FNE_TRY(dalloc(h, &h->counter, 1));
  {
    cudaError_t e = cudaMemset(h->counter, 0, sizeof(unsigned));
    if (e != cudaSuccess) {
      free_handle(h);
      return cuda_fail(e, "cudaMemset");
    }
  }
  if (d->dirichlet_only_energy) {
    FNE_TRY(dalloc(h, &h->dir_const, 1));
    FNE_TRY(refresh_dir_const(h));
  }
  if (h->smem_bytes > 48 * 1024) {
    RowArgs ra{};
    IncArgs pa{};
    SweepArgs sa{};
    for (int want = 2; want <= 7; ++want) {
      cudaError_t e = launch_rows(h, want, ra, pa, sa, nullptr, nullptr, EnergyOut{}, 0, true);
      if (e != cudaSuccess) {
        free_handle(h);
        return cuda_fail(e, "cudaFuncSetAttribute");
      }
    }
  }
#undef FNE_TRY
  *out = h;
  return FNE_OK;
}

extern "C" int fne_info_get(const fne_handle* h, fne_info* info) {
  if (!h || !info) return set_error(FNE_EINVAL, "fne_info_get: null argument");
  if (h->mc) {
    mc_info(h->mc, info);
    return FNE_OK;
  }
  if (h->mc3) {
    mc3d_info(h->mc3, info);
    return FNE_OK;
  }
  info->n_rows = h->n_rows;
  info->nnz = h->nnz;
  info->n_elem = h->n_local;
  info->n_incidences = h->n_inc;
  info->device_bytes = h->device_bytes;
  info->max_row_len = h->max_row_len;
  info->kernel_variant = is_tri(h->family) ? (h->use_cluster ? 10 : h->use_push ? 8 : (h->use_sweep ? 4 : (h->use_inc ? 3 : 1)))
                                           : (h->use_elem2 ? 7 : 2);
  if (h->use_elem2) info->n_incidences = h->e2_contrib;
  info->row_lanes = h->tet_lanes;
  return FNE_OK;
}

extern "C" int fne_hvp_prepare(fne_handle* h, const double* u, void* stream) {
  if (!h || (!u && h->n_free > 0)) return set_error(FNE_EINVAL, "fne_hvp_prepare: null argument");
  if (!h->mc) return set_error(FNE_EINVAL, "fne_hvp_prepare: matrix-free products exist for the Mohr-Coulomb family");
  return mc_hvp_prepare(h->mc, u, stream);
}

extern "C" int fne_hvp(fne_handle* h, const double* x, double* y, void* stream) {
  if (!h || (!x && h->n_free > 0) || (!y && h->hi > h->lo)) return set_error(FNE_EINVAL, "fne_hvp: null argument");
  if (!h->mc) return set_error(FNE_EINVAL, "fne_hvp: matrix-free products exist for the Mohr-Coulomb family");
  return mc_hvp(h->mc, x, y, stream);
}

extern "C" int fne_hvp_diagonal(fne_handle* h, double* diag, void* stream) {
  if (!h || (!diag && h->hi > h->lo)) return set_error(FNE_EINVAL, "fne_hvp_diagonal: null argument");
  if (!h->mc) return set_error(FNE_EINVAL, "fne_hvp_diagonal: matrix-free products exist for the Mohr-Coulomb family");
  return mc_hvp_diagonal(h->mc, diag, stream);
}

extern "C" int fne_check_device_status(fne_handle* h) {
  if (!h) return set_error(FNE_EINVAL, "fne_check_device_status: null handle");
  if (h->mc) return mc_check_status(h->mc);
  if (!h->err) return FNE_OK;
  int v = 0;
  cudaError_t e = cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "fne_check_device_status");
  if (v == 0) return FNE_OK;
  cudaMemset(h->err, 0, sizeof(int));
  if (h->err_host) *h->err_host = 0;
  return set_error(FNE_ETIMEOUT, "row-cluster kernel: a wait for its staging copies gave up");
}

extern "C" int fne_poll_device_status(fne_handle* h) {
  if (!h) return set_error(FNE_EINVAL, "fne_poll_device_status: null handle");
  if (h->mc) return mc_poll_status(h->mc);
  if (!h->err_host || *(volatile int*)h->err_host == 0) return FNE_OK;
  *h->err_host = 0;
  cudaMemset(h->err, 0, sizeof(int));
  return set_error(FNE_ETIMEOUT, "row-cluster kernel: a wait for its staging copies gave up");
}

extern "C" int fne_set_wait_limit(fne_handle* h, int64_t polls) {
  if (!h) return set_error(FNE_EINVAL, "fne_set_wait_limit: null handle");
  if (h->use_cluster) {
    h->cl_wait_limit = polls < 0 ? kClWaitLimit : (long long)polls;
    return FNE_OK;
  }
  if (!h->mc) return set_error(FNE_EINVAL, "fne_set_wait_limit: the handle runs no kernel with a bounded wait");
  return mc_set_wait_limit(h->mc, (long long)polls);
}

extern "C" int fne_set_dirichlet(fne_handle* h, const double* dirichlet) {
  if (!h || (!dirichlet && h->n_total > 0)) return set_error(FNE_EINVAL, "fne_set_dirichlet: null argument");
  if (h->n_total == 0) return FNE_OK;
  if (h->mc) return mc_set_dirichlet(h->mc, dirichlet);
  if (h->mc3) return mc3d_set_dirichlet(h->mc3, dirichlet);
  cudaError_t e = cudaMemcpy(h->dir, dirichlet, h->n_total * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "fne_set_dirichlet");
  return refresh_dir_const(h);
}

extern "C" int fne_eval(fne_handle* h, const double* u, int flags, double* energy, double* grad, void* hess,
                        void* stream) {
  if (!h) return set_error(FNE_EINVAL, "fne_eval: null handle");
  if (flags <= 0 || flags > 7) return set_error(FNE_EINVAL, "fne_eval: flags must combine FNE_ENERGY|GRAD|HESS");
  if ((flags & FNE_ENERGY) && !energy) return set_error(FNE_EINVAL, "fne_eval: energy output missing");
  if ((flags & FNE_GRAD) && !grad && h->hi > h->lo) return set_error(FNE_EINVAL, "fne_eval: grad output missing");
  if ((flags & FNE_HESS) && !hess && h->nnz > 0) return set_error(FNE_EINVAL, "fne_eval: hess output missing");
  if (!u && h->n_free > 0) return set_error(FNE_EINVAL, "fne_eval: u missing");
  if (h->mc) return mc_eval(h->mc, u, flags, energy, grad, hess, stream);
  if (h->mc3) return mc3d_eval(h->mc3, u, flags, energy, grad, hess, stream);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  EnergyOut eo{h->partials, h->counter, energy, h->dir_const};
  cudaError_t e = cudaSuccess;
  const int n_owned = (int)(h->hi - h->lo);
  if (flags == FNE_ENERGY || h->n_rows == 0) {
    if (flags & FNE_ENERGY) e = launch_energy(h, h->rec, h->n_local, u, h->rhs, n_owned, eo, st);
  } else {
    RowArgs A;
    A.n_rows = h->n_rows;
    A.row_ptr = h->row_ptr;
    A.row_node = h->row_node;
    A.row_comp = h->row_comp;
    A.row_gpos = h->row_gpos;
    A.inc_ptr = h->inc_ptr;
    A.inc_elem = h->inc_elem;
    A.inc_info = h->inc_info;
    A.u = u;
    A.dir = h->dir;
    A.rhs = h->rhs;
    A.lo = h->lo;
    A.nrec = h->n_local;
    IncArgs Q{h->cta_row, h->cta_inc, h->inc_elem2, h->inc_word, h->inc_rowl, h->inc_max_rank, h->inc_max_rows,
              h->inc_max_len};
    SweepArgs SW{h->sw_seg_row,  h->sw_seg_elem,  h->sw_seg_batch,  h->sw_batch_done,
                 h->sw_ent_ptr,  h->sw_inc_base,  h->sw_ent_row,    h->sw_ent_pos,
                 h->sw_ent_meta, h->sw_inc_word,  h->sweep_win_mask, h->sweep_rwin_mask,
                 h->sw_gpos_identity, h->sw_eoff, h->sw_row_of};
    e = h->use_elem2 ? launch_elem2(h, flags, u, grad, hess, eo, st)
                     : launch_rows(h, flags, A, Q, SW, grad, hess, eo, st, false);
    // stream-ordered copy of the status word for fne_poll_device_status
    if (e == cudaSuccess && h->use_cluster)
      e = cudaMemcpyAsync(h->err_host, h->err, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (e != cudaSuccess) return cuda_fail(e, "fne_eval launch");
  return FNE_OK;
}

extern "C" int fne_eval_host(fne_handle* h, const double* u_host, int flags, double* energy_host, double* grad_host,
                             void* hess_host) {
  if (!h) return set_error(FNE_EINVAL, "fne_eval_host: null handle");
  const size_t n_owned = (size_t)(h->hi - h->lo);
  const size_t hsz = (h->precision == FNE_FP32 && h->hess_fp32) ? sizeof(float) : sizeof(double);
  if (!h->h_energy) {  // staging buffers, allocated once per handle
    int rc = dalloc(h, &h->h_u, std::max<size_t>(1, (size_t)h->n_free));
    if (!rc) rc = dalloc(h, &h->h_grad, std::max<size_t>(1, n_owned));
    if (!rc) rc = dalloc(h, &h->h_energy, 1);
    if (!rc) rc = dalloc(h, (unsigned char**)&h->h_hess, std::max<size_t>(1, (size_t)h->nnz * hsz));
    if (rc) return rc;
  }
  cudaError_t e = cudaSuccess;
  if (h->n_free) e = cudaMemcpy(h->h_u, u_host, h->n_free * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "fne_eval_host H2D");
  int rc = fne_eval(h, h->h_u, flags, h->h_energy, h->h_grad, h->h_hess, nullptr);
  if (rc) return rc;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "fne_eval_host kernel");
  if ((flags & FNE_ENERGY) && energy_host) e = cudaMemcpy(energy_host, h->h_energy, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && (flags & FNE_GRAD) && grad_host && n_owned)
    e = cudaMemcpy(grad_host, h->h_grad, n_owned * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && (flags & FNE_HESS) && hess_host && h->nnz)
    e = cudaMemcpy(hess_host, h->h_hess, h->nnz * hsz, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "fne_eval_host D2H");
  return FNE_OK;
}

extern "C" int fne_destroy(fne_handle* h) {
  free_handle(h);
  return FNE_OK;
}

extern "C" const char* fne_last_error(void) { return g_err.c_str(); }
extern "C" const char* fne_version(void) { return "fne_asm 0.2 (sm_100a)"; }
