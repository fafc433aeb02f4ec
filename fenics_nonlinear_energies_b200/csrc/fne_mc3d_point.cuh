// One quadrature point of the 3-D Mohr-Coulomb density: energy, stress and
// consistent tangent in strain space, as host/device code (the reference
// density is src/problems/slope_stability_3d/jax/jax_energy_3d.py:38-191;
// its derivatives there come from JAX autodiff through eigvalsh).
//
// Strain eps = [xx, yy, zz, xy, yz, xz] with engineering shears.  With
// A = tensor(eps) + tiny diag(0, 1, 2), lambda_1 >= lambda_2 >= lambda_3 its
// eigenvalues, I1 = eps_xx + eps_yy + eps_zz and
// Q = eps_xx^2 + eps_yy^2 + eps_zz^2 + (xy^2 + yz^2 + xz^2) / 2, every
// branch potential is a quadratic form in z = (lambda_1, lambda_2,
// lambda_3, I1) plus mu Q (elastic and smooth branches), built from terms
// -d/2 (n / ds)^2 with n = a.z - c linear, d a constant denominator and ds
// = d through the reference's signed tiny guard:
//   elastic  lame/2 I1^2 + mu Q
//   smooth   lame/2 I1^2 + mu Q - d_s/2 (f / ds_s)^2,  f = 2mu((1+s)l1 - (1-s)l3) + 2 lame s I1 - c
//   left     lame/2 I1^2 + mu(l3^2 + (l1+l2)^2/2) - d_l/2 (n_l / ds_l)^2
//   right    lame/2 I1^2 + mu(l1^2 + (l2+l3)^2/2) - d_r/2 (n_r / ds_r)^2
//   apex     K/2 I1^2 - d_a/2 (n_a / ds_a)^2
// The branch is picked from the primal values in the reference's order.  Stress and tangent
// follow by the chain rule with the eigenvalue derivatives
//   d lambda_k / dA = v_k v_k^T,
//   d2 lambda_k / dA dA[X, Y] = 2 sum_{j != k} (v_k^T X v_j)(v_j^T Y v_k) / (lambda_k - lambda_j)
// (summed per eigenvalue pair),
// eigenvectors from a fixed six-sweep cyclic Jacobi solve.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define FNE_HD __host__ __device__ __forceinline__
#else
#define FNE_HD inline
#endif

namespace fne {
namespace mc3d {

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (at most 6
// sweeps); w descending, V columns the eigenvectors.
FNE_HD void eigh3(const double A0[3][3], double w[3], double V[3][3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      a[i][j] = A0[i][j];
      V[i][j] = i == j ? 1.0 : 0.0;
    }
  const int P[3] = {0, 0, 1}, Qi[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 6; ++sweep) {
    bool rotated = false;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int p = P[r], q = Qi[r];
      const double apq = a[p][q];
      // a rotation by less than one ulp of angle (|t| ~ |apq / (aqq - app)|)
      // changes nothing beyond rounding: skipped; a sweep without rotations
      // ends the solve (3 to 4 sweeps for almost every strain)
      if (apq == 0.0 || fabs(apq) <= 2.220446049250313e-16 * fabs(a[q][q] - a[p][p])) continue;
      rotated = true;
      const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      const double t = fabs(theta) > 1e100 ? 0.5 / theta
                                            : (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      // a <- R^T a R with R = identity except R_pp = R_qq = c, R_pq = s, R_qp = -s
      for (int k = 0; k < 3; ++k) {  // columns p, q
        const double akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
      }
      for (int k = 0; k < 3; ++k) {  // rows p, q
        const double apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
      for (int k = 0; k < 3; ++k) {
        const double vkp = V[k][p], vkq = V[k][q];
        V[k][p] = c * vkp - s * vkq;
        V[k][q] = s * vkp + c * vkq;
      }
    }
    if (!rotated) break;
  }
  // sort descending: compare-swaps (0, 1), (1, 2), (0, 1) on the diagonal
  // and the eigenvector columns (constant indices, so everything stays in
  // registers)
  double d[3] = {a[0][0], a[1][1], a[2][2]};
  auto cswap = [&](int i, int j) {
    if (d[i] < d[j]) {
      const double t = d[i];
      d[i] = d[j];
      d[j] = t;
      for (int k = 0; k < 3; ++k) {
        const double v = V[k][i];
        V[k][i] = V[k][j];
        V[k][j] = v;
      }
    }
  };
  cswap(0, 1);
  cswap(1, 2);
  cswap(0, 1);
  for (int k = 0; k < 3; ++k) w[k] = d[k];
}

FNE_HD double safe_denom(double x, double tiny) {
  return fabs(x) < tiny ? (x >= 0.0 ? tiny : -tiny) : x;
}

// psi, sigma[6], D[6][6] at strain e[6].  Returns the branch (0 elastic,
// 1 smooth, 2 left edge, 3 right edge, 4 apex).
FNE_HD int point(const double e[6], double c_bar, double sp, double mu, double K, double lame, double tiny,
                 double& psi, double sig[6], double D[6][6]) {
  // dA / d eps_m: (i, j) entries with weight (1 for normals, 1/2 for the shears)
  const double A[3][3] = {{e[0] + 0.0 * tiny, 0.5 * e[3], 0.5 * e[5]},
                          {0.5 * e[3], e[1] + tiny, 0.5 * e[4]},
                          {0.5 * e[5], 0.5 * e[4], e[2] + 2.0 * tiny}};
  double lam[3], V[3][3];
  eigh3(A, lam, V);
  const double l1 = lam[0], l2 = lam[1], l3 = lam[2];
  const double I1 = e[0] + e[1] + e[2];
  const double Qv = e[0] * e[0] + e[1] * e[1] + e[2] * e[2] + 0.5 * (e[3] * e[3] + e[4] * e[4] + e[5] * e[5]);
  // branch tests (primal values, the reference's order)
  const double f_tr = 2.0 * mu * ((1.0 + sp) * l1 - (1.0 - sp) * l3) + 2.0 * lame * sp * I1 - c_bar;
  const double g_sl = (l1 - l2) / fmax(tiny, 1.0 + sp), g_sr = (l2 - l3) / fmax(tiny, 1.0 - sp);
  const double g_la = (l1 + l2 - 2.0 * l3) / fmax(tiny, 3.0 - sp), g_ra = (2.0 * l1 - l2 - l3) / fmax(tiny, 3.0 + sp);
  // raw denominators (they weight the return terms) and their signed-tiny
  // guarded copies (they divide)
  const double r_s = 4.0 * lame * sp * sp + 4.0 * mu * (1.0 + sp * sp);
  const double r_l = 4.0 * lame * sp * sp + mu * (1.0 + sp) * (1.0 + sp) + 2.0 * mu * (1.0 - sp) * (1.0 - sp);
  const double r_r = 4.0 * lame * sp * sp + 2.0 * mu * (1.0 + sp) * (1.0 + sp) + mu * (1.0 - sp) * (1.0 - sp);
  const double r_a = 4.0 * K * sp * sp;
  const double d_s = safe_denom(r_s, tiny), d_l = safe_denom(r_l, tiny), d_r = safe_denom(r_r, tiny),
               d_a = safe_denom(r_a, tiny);
  // linear forms n = a.z - c over z = (l1, l2, l3, I1)
  const double as[4] = {2.0 * mu * (1.0 + sp), 0.0, -2.0 * mu * (1.0 - sp), 2.0 * lame * sp};
  const double al[4] = {mu * (1.0 + sp), mu * (1.0 + sp), -2.0 * mu * (1.0 - sp), 2.0 * lame * sp};
  const double ar[4] = {2.0 * mu * (1.0 + sp), -mu * (1.0 - sp), -mu * (1.0 - sp), 2.0 * lame * sp};
  const double aa[4] = {0.0, 0.0, 0.0, 2.0 * K * sp};
  auto lin = [&](const double a[4]) { return a[0] * l1 + a[1] * l2 + a[2] * l3 + a[3] * I1 - c_bar; };
  const double lam_s = f_tr / d_s, lam_l = lin(al) / d_l, lam_r = lin(ar) / d_r;
  int br;
  if (f_tr <= 0.0) br = 0;
  else if (lam_s <= fmin(g_sl, g_sr)) br = 1;
  else if (g_sl < g_sr && lam_l >= g_sl && lam_l <= g_la) br = 2;
  else if (g_sl > g_sr && lam_r >= g_sr && lam_r <= g_ra) br = 3;
  else br = 4;
  // F(z) = 1/2 z^T M z + q^T z (+ const) + wQ Q: value, gradient Fz[4], Hessian Fzz[4][4]
  double Fz[4] = {0, 0, 0, 0}, Fzz[4][4] = {{0}};
  double wQ = 0.0;
  psi = 0.0;
  auto add_quad = [&](int i, int j, double coef) {  // + coef/2 (z_i + z_j)^2 style terms via M entries
    Fzz[i][j] += coef;
    if (i != j) Fzz[j][i] += coef;
  };
  const double z[4] = {l1, l2, l3, I1};
  // - d/2 (n / ds)^2 with n = a.z - c, d the raw denominator and ds its
  // guarded copy (the reference's form: where |d| < tiny the term is
  // d/2 (n/tiny)^2, vanishing with d, not n^2 / (2 tiny))
  auto add_neg_sq = [&](const double a[4], double d, double ds) {
    const double n = lin(a), r = d / (ds * ds);
    psi -= 0.5 * r * n * n;
    for (int i = 0; i < 4; ++i) {
      Fz[i] -= r * n * a[i];
      for (int j = 0; j < 4; ++j) Fzz[i][j] -= r * a[i] * a[j];
    }
  };
  if (br == 4) {
    psi = 0.5 * K * I1 * I1;
    Fz[3] += K * I1;
    add_quad(3, 3, K);
    add_neg_sq(aa, r_a, d_a);
  } else {
    psi = 0.5 * lame * I1 * I1;
    Fz[3] += lame * I1;
    add_quad(3, 3, lame);
    if (br <= 1) {
      psi += mu * Qv;
      wQ = mu;
      if (br == 1) add_neg_sq(as, r_s, d_s);
    } else if (br == 2) {  // mu (l3^2 + (l1 + l2)^2 / 2)
      psi += mu * (l3 * l3 + 0.5 * (l1 + l2) * (l1 + l2));
      Fz[2] += 2.0 * mu * l3;
      Fz[0] += mu * (l1 + l2);
      Fz[1] += mu * (l1 + l2);
      add_quad(2, 2, 2.0 * mu);
      add_quad(0, 0, mu);
      add_quad(1, 1, mu);
      add_quad(0, 1, mu);
      add_neg_sq(al, r_l, d_l);
    } else {  // mu (l1^2 + (l2 + l3)^2 / 2)
      psi += mu * (l1 * l1 + 0.5 * (l2 + l3) * (l2 + l3));
      Fz[0] += 2.0 * mu * l1;
      Fz[1] += mu * (l2 + l3);
      Fz[2] += mu * (l2 + l3);
      add_quad(0, 0, 2.0 * mu);
      add_quad(1, 1, mu);
      add_quad(2, 2, mu);
      add_quad(1, 2, mu);
      add_neg_sq(ar, r_r, d_r);
    }
  }
  (void)z;
  // d z / d eps: eigenvalues g_k[m] = v_k^T dA_m v_k, I1 = (1, 1, 1, 0, 0, 0)
  const int mi[6] = {0, 1, 2, 0, 1, 0}, mj[6] = {0, 1, 2, 1, 2, 2};
  const double mw[6] = {1.0, 1.0, 1.0, 0.5, 0.5, 0.5};
  // dz[k][m] = v_k^T dA_m v_k (eigenvalue k), dz[3] = d I1; Xp[r][m] =
  // v_k^T dA_m v_j for the pairs (k, j) = (0, 1), (0, 2), (1, 2)
  const int pk[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
  double dz[4][6], Xp[3][6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const int i = mi[m], j = mj[m];
#pragma unroll
    for (int k = 0; k < 3; ++k) dz[k][m] = i == j ? V[i][k] * V[i][k] : 2.0 * mw[m] * V[i][k] * V[j][k];
    dz[3][m] = m < 3 ? 1.0 : 0.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int k = pk[r], l = pj[r];
      Xp[r][m] = i == j ? V[i][k] * V[i][l] : mw[m] * (V[i][k] * V[j][l] + V[j][k] * V[i][l]);
    }
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    double s = wQ * (m < 3 ? 2.0 * e[m] : e[m]);
    for (int a = 0; a < 4; ++a) s += Fz[a] * dz[a][m];
    sig[m] = s;
  }
  // eigenvalue curvature, one term per pair k < j:
  // 2 (Fz_k - Fz_j) / (lambda_k - lambda_j) Xp[m] Xp[n].  Summing the pair
  // once avoids the cancellation of two ~1/(lambda_k - lambda_j) terms; a
  // pair with Fz_k == Fz_j, or with coincident eigenvalues (tie-break
  // absorbed), contributes 0 instead of 0/0.
  double cp[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double dF = Fz[pk[r]] - Fz[pj[r]], dl = lam[pk[r]] - lam[pj[r]];
    cp[r] = (dF != 0.0 && dl != 0.0) ? 2.0 * dF / dl : 0.0;
  }
  // D = dz^T Fzz dz + wQ diag(2, 2, 2, 1, 1, 1) + curvature, through
  // G = Fzz dz; the upper triangle, mirrored
  double G[4][6];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int n = 0; n < 6; ++n) G[a][n] = Fzz[a][0] * dz[0][n] + Fzz[a][1] * dz[1][n] + Fzz[a][2] * dz[2][n] +
                                          Fzz[a][3] * dz[3][n];
#pragma unroll
  for (int m = 0; m < 6; ++m)
#pragma unroll
    for (int n = m; n < 6; ++n) {
      double s = (m == n) ? wQ * (m < 3 ? 2.0 : 1.0) : 0.0;
      s += dz[0][m] * G[0][n] + dz[1][m] * G[1][n] + dz[2][m] * G[2][n] + dz[3][m] * G[3][n];
      s += cp[0] * Xp[0][m] * Xp[0][n] + cp[1] * Xp[1][m] * Xp[1][n] + cp[2] * Xp[2][m] * Xp[2][n];
      D[m][n] = s;
      D[n][m] = s;
    }
  return br;
}

// One element with NP nodes (DOFs (x, y, z) per node) and nq points:
// energy sum_q w_q psi_q, gradient g = sum_q w_q B_q^T sigma_q and Hessian
// K = sum_q w_q B_q^T D_q B_q (dense 3NP x 3NP).  gx/gy/gz [nq][NP] are the
// physical basis gradients, prm [nq][5] = (c_bar, sin_phi, shear, bulk, lame).
template <int NP>
FNE_HD double element(const double* u, const double* gx, const double* gy, const double* gz, const double* w,
                      const double* prm, int nq, double tiny, double* g, double* K) {
  constexpr int N = 3 * NP;
  double e_tot = 0.0;
  for (int i = 0; i < N; ++i) g[i] = 0.0;
  for (int i = 0; i < N * N; ++i) K[i] = 0.0;
  for (int q = 0; q < nq; ++q) {
    const double* px = gx + q * NP;
    const double* py = gy + q * NP;
    const double* pz = gz + q * NP;
    double e[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < NP; ++a) {
      const double ux = u[3 * a], uy = u[3 * a + 1], uz = u[3 * a + 2];
      e[0] += px[a] * ux;
      e[1] += py[a] * uy;
      e[2] += pz[a] * uz;
      e[3] += py[a] * ux + px[a] * uy;
      e[4] += pz[a] * uy + py[a] * uz;
      e[5] += pz[a] * ux + px[a] * uz;
    }
    const double* m = prm + 5 * q;
    double psi, sig[6], D[6][6];
    point(e, m[0], m[1], m[2], m[3], m[4], tiny, psi, sig, D);
    e_tot += w[q] * psi;
    // B_q columns of DOF (a, c): the strain components it feeds
    for (int a = 0; a < NP; ++a) {
      const double b[3][6] = {{px[a], 0, 0, py[a], 0, pz[a]}, {0, py[a], 0, px[a], pz[a], 0}, {0, 0, pz[a], 0, py[a], px[a]}};
      for (int c = 0; c < 3; ++c) {
        double s = 0.0, Db[6];
        for (int i = 0; i < 6; ++i) {
          s += b[c][i] * sig[i];
          Db[i] = 0.0;
          for (int j = 0; j < 6; ++j) Db[i] += D[i][j] * b[c][j];
        }
        g[3 * a + c] += w[q] * s;
        for (int a2 = 0; a2 < NP; ++a2) {
          const double b2[3][6] = {{px[a2], 0, 0, py[a2], 0, pz[a2]}, {0, py[a2], 0, px[a2], pz[a2], 0},
                                   {0, 0, pz[a2], 0, py[a2], px[a2]}};
          for (int c2 = 0; c2 < 3; ++c2) {
            double t = 0.0;
            for (int i = 0; i < 6; ++i) t += b2[c2][i] * Db[i];
            K[(3 * a2 + c2) * N + 3 * a + c] += w[q] * t;
          }
        }
      }
    }
  }
  return e_tot;
}

}  // namespace mc3d
}  // namespace fne
