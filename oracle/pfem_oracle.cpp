// pfem_oracle.cpp -- CPU FP64 restatement of the reference's finite-strain
// F-bar J2 path (vinaysrao1/plasticity, lagrangian/src).
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle: it is linked by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the
// checker / timed CPU baseline, never by the product library.  It restates the
// reference algorithm literally (dense 9x9 dP/dF, dense G^T A Geff products,
// binary-search CSC scatter) so that its cost and its arithmetic follow the
// reference's own code.  Each function cites the reference lines it follows.
//
// Conventions (lagrangian/src/Materials.jl:18-19): Voigt order
// [xx,yy,zz,xy,yz,zx]; strain Voigt carries engineering shear, stress Voigt
// physical shear.  3x3 matrices are stored row-major m[i][j] here; the
// reference's 9-vectors of F/P/G are column-major (index (j)*3+i), and every
// place that forms such a 9-vector below uses that column-major index.
//
// Parity notes: the reference's symmetric 3x3 eigensolver is StaticArrays'
// closed form (third-party, version unpinned); this oracle uses cyclic Jacobi.
// Both return an orthonormal eigenbasis, and every quantity built from it is an
// isotropic tensor function, so results agree to rounding.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <thread>
#include <atomic>

namespace {

// Minimal parallel-for over [0, n) with `nt` std::threads pulling chunks of
// `grain` indices from a shared counter (the image has no OpenMP runtime).
template <class Fn>
void parallel_for(int64_t n, int nt, int64_t grain, Fn fn) {
  if (nt <= 1 || n <= grain) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next(0);
  auto work = [&]() {
    for (;;) {
      const int64_t b = next.fetch_add(grain);
      if (b >= n) break;
      const int64_t e = std::min(n, b + grain);
      for (int64_t i = b; i < e; ++i) fn(i);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

struct Mat {
  double E, nu, sigy0, Hiso, Hkin, sigsat, delta, G, K, lam;
  bool voce;  // saturation branch active (Materials.jl:201)
};

// J2Material constructor moduli, lagrangian/src/Materials.jl:82-108.  m7 =
// (E, nu, sigy0, Hiso, Hkin, sigsat, delta); sigsat <= 0 stands for the
// keyword default sigsat = sigy0.
Mat make_mat(const double* m7) {
  Mat m;
  m.E = m7[0]; m.nu = m7[1]; m.sigy0 = m7[2]; m.Hiso = m7[3]; m.Hkin = m7[4];
  m.sigsat = m7[5] > 0 ? m7[5] : m7[2];
  m.delta = m7[6];
  m.voce = m.delta > 0 && m.sigsat > m.sigy0;
  m.G = m.E / (2.0 * (1.0 + m.nu));
  m.K = m.E / (3.0 * (1.0 - 2.0 * m.nu));
  m.lam = m.E * m.nu / ((1.0 + m.nu) * (1.0 - 2.0 * m.nu));
  return m;
}

// elastic_matrix, Materials.jl:27-35 (row-major 6x6).
void cmat(const Mat& m, double C[36]) {
  std::memset(C, 0, 36 * sizeof(double));
  const double a = m.lam + 2.0 * m.G;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C[i * 6 + j] = (i == j) ? a : m.lam;
  for (int i = 3; i < 6; ++i) C[i * 6 + i] = m.G;
}

// devnorm, Materials.jl:144-146.
double devnorm(const double s[6]) {
  return std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2] +
                   2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// yield_stress, Materials.jl:117-118.  sy0 is the element's initial yield
// stress (the material's unless a per-element value is given); the saturation
// amplitude is the material's sigsat - sigy0.
double yield_stress(const Mat& m, double sy0, double a) {
  return sy0 + (m.sigsat - m.sigy0) * (1.0 - std::exp(-m.delta * a)) + m.Hiso * a;
}
// yield_slope, Materials.jl:126-127.
double yield_slope(const Mat& m, double a) {
  return m.delta * (m.sigsat - m.sigy0) * std::exp(-m.delta * a) + m.Hiso;
}

// return_map, Materials.jl:159-250: linear branch (closed-form dgamma, :218)
// or the saturation branch (scalar local Newton on dgamma, :201-213).
// Returns 1 for the plastic branch (f_tr > 0), 0 for elastic.
int return_map(const Mat& m, double sigy0, const double eps[6], const double epsp_n[6],
               const double beta_n[6], double alpha_n, double sig[6], double epsp_new[6],
               double beta_new[6], double* alpha_new, double D[36], double* ftr_out) {
  double C[36];
  cmat(m, C);
  double de[6];
  for (int i = 0; i < 6; ++i) de[i] = eps[i] - epsp_n[i];
  double st[6];
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += C[i * 6 + j] * de[j];
    st[i] = s;
  }
  const double p = (st[0] + st[1] + st[2]) / 3.0;
  double xi[6];
  for (int i = 0; i < 6; ++i) xi[i] = st[i] - (i < 3 ? p : 0.0) - beta_n[i];
  const double nrm = devnorm(xi);
  const double q = std::sqrt(1.5) * nrm;
  const double ftr = m.voce ? q - yield_stress(m, sigy0, alpha_n) : q - (sigy0 + m.Hiso * alpha_n);
  if (ftr_out) *ftr_out = ftr;
  if (ftr <= 0.0) {
    for (int i = 0; i < 6; ++i) {
      sig[i] = st[i]; epsp_new[i] = epsp_n[i]; beta_new[i] = beta_n[i];
    }
    *alpha_new = alpha_n;
    std::memcpy(D, C, sizeof(C));
    return 0;
  }
  const double s32 = std::sqrt(1.5);
  double nh[6];
  for (int i = 0; i < 6; ++i) nh[i] = xi[i] / nrm;
  const double G = m.G;
  double dg;
  if (m.voce) {
    dg = ftr / (3.0 * G + m.Hkin + yield_slope(m, alpha_n));
    for (int it = 0; it < 50; ++it) {
      const double Hp = yield_slope(m, alpha_n + dg);
      const double r = q - (3.0 * G + m.Hkin) * dg - yield_stress(m, sigy0, alpha_n + dg);
      const double d = r / (3.0 * G + m.Hkin + Hp);
      dg += d;
      if (std::fabs(d) <= 1e-13 * (dg + 1e-14)) break;
    }
  } else {
    dg = ftr / (3.0 * G + m.Hiso + m.Hkin);
  }
  for (int i = 0; i < 6; ++i) sig[i] = st[i] - (2.0 * G * dg * s32) * nh[i];
  for (int i = 0; i < 6; ++i)
    epsp_new[i] = epsp_n[i] + (dg * s32) * (i < 3 ? nh[i] : 2.0 * nh[i]);
  for (int i = 0; i < 6; ++i) beta_new[i] = beta_n[i] + (2.0 / 3.0) * m.Hkin * (dg * s32) * nh[i];
  *alpha_new = alpha_n + dg;
  const double Hp = m.voce ? yield_slope(m, *alpha_new) : m.Hiso;
  const double b0 = 2.0 * G * dg / q;
  const double g0 = 2.0 * G / (3.0 * G + m.Hkin + Hp);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      const double isym = (i == j) ? (i < 3 ? 1.0 : 0.5) : 0.0;
      const double one = (i < 3 && j < 3) ? 1.0 : 0.0;
      const double idev = isym - one / 3.0;
      D[i * 6 + j] = C[i * 6 + j] - (3.0 * G * b0) * idev + (3.0 * G * (b0 - g0)) * nh[i] * nh[j];
    }
  return 1;
}

// ---- 3x3 helpers (row-major) ----
inline double det3(const double a[3][3]) {
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
         a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
         a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}
inline void inv3(const double a[3][3], double r[3][3]) {
  const double d = det3(a);
  r[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / d;
  r[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / d;
  r[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / d;
  r[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / d;
  r[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / d;
  r[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / d;
  r[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / d;
  r[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / d;
  r[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / d;
}
inline void mul3(const double a[3][3], const double b[3][3], double c[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      c[i][j] = s;
    }
}
inline void tr3(const double a[3][3], double t[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) t[i][j] = a[j][i];
}
// voigt_to_sym3 (physical shear), FiniteStrain.jl:83-87.
inline void v2s(const double v[6], double m[3][3]) {
  m[0][0] = v[0]; m[1][1] = v[1]; m[2][2] = v[2];
  m[0][1] = m[1][0] = v[3];
  m[1][2] = m[2][1] = v[4];
  m[0][2] = m[2][0] = v[5];
}
// sym3_to_voigt, FiniteStrain.jl:94-96.
inline void s2v(const double m[3][3], double v[6]) {
  v[0] = m[0][0]; v[1] = m[1][1]; v[2] = m[2][2];
  v[3] = m[0][1]; v[4] = m[1][2]; v[5] = m[0][2];
}

// Symmetric 3x3 eigendecomposition by cyclic Jacobi rotations.  Stand-in for
// StaticArrays `eigen(Symmetric(...))` (FiniteStrain.jl:158, :338).  Returns
// eigenvalues ascending in w and eigenvectors as the columns of V.
void eig3(const double Ain[3][3], double w[3], double V[3][3]) {
  double a[3][3];
  std::memcpy(a, Ain, sizeof(a));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  static const int PQ[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 60; ++sweep) {
    const double off = std::fabs(a[0][1]) + std::fabs(a[0][2]) + std::fabs(a[1][2]);
    const double dia = std::fabs(a[0][0]) + std::fabs(a[1][1]) + std::fabs(a[2][2]);
    if (off == 0.0 || off <= 1e-300 || off < 1e-18 * dia) break;
    for (int r = 0; r < 3; ++r) {
      const int p = PQ[r][0], q = PQ[r][1];
      const double apq = a[p][q];
      if (apq == 0.0) continue;
      const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
      double t;
      if (std::fabs(theta) > 1e150) t = 0.5 / theta;
      else t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
      const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
      a[p][p] -= t * apq;
      a[q][q] += t * apq;
      a[p][q] = a[q][p] = 0.0;
      const int o = 3 - p - q;
      const double arp = a[o][p], arq = a[o][q];
      a[o][p] = a[p][o] = c * arp - s * arq;
      a[o][q] = a[q][o] = s * arp + c * arq;
      for (int k = 0; k < 3; ++k) {
        const double vp = V[k][p], vq = V[k][q];
        V[k][p] = c * vp - s * vq;
        V[k][q] = s * vp + c * vq;
      }
    }
  }
  int idx[3] = {0, 1, 2};
  std::sort(idx, idx + 3, [&](int x, int y) { return a[x][x] < a[y][y]; });
  double W[3][3];
  for (int c = 0; c < 3; ++c) {
    w[c] = a[idx[c]][idx[c]];
    for (int k = 0; k < 3; ++k) W[k][c] = V[k][idx[c]];
  }
  std::memcpy(V, W, sizeof(W));
}

const double EIG_TOL = 1e-9;  // FiniteStrain.jl:69

struct Kin {
  double eps_tr[6];  // engineering-shear Voigt
  double b[3];
  double n[3][3];    // eigenvectors as columns
  double Finv[3][3];
  double J;
  bool ok;
};

// finite_kinematics, FiniteStrain.jl:148-170.
Kin finite_kinematics(const double F[3][3], const double cpi_v[6]) {
  Kin k;
  k.J = det3(F);
  if (k.J <= 0) {
    k.ok = false;
    return k;
  }
  k.ok = true;
  double Cpi[3][3], T[3][3], Ft[3][3], be[3][3];
  v2s(cpi_v, Cpi);
  mul3(F, Cpi, T);
  tr3(F, Ft);
  mul3(T, Ft, be);
  eig3(be, k.b, k.n);
  double lnl[3];
  for (int A = 0; A < 3; ++A) lnl[A] = 0.5 * std::log(k.b[A]);
  double em[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      em[i][j] = lnl[0] * k.n[i][0] * k.n[j][0] + lnl[1] * k.n[i][1] * k.n[j][1] +
                 lnl[2] * k.n[i][2] * k.n[j][2];
  k.eps_tr[0] = em[0][0]; k.eps_tr[1] = em[1][1]; k.eps_tr[2] = em[2][2];
  k.eps_tr[3] = 2 * em[0][1]; k.eps_tr[4] = 2 * em[1][2]; k.eps_tr[5] = 2 * em[0][2];
  inv3(F, k.Finv);
  return k;
}

// Right polar decomposition F = R U, polar_RU (FiniteStrain.jl:194-210):
// U = (F^T F)^(1/2) through the eigenbasis V of F^T F (eigenvalues floored at
// 0), R = F U^-1.  mu receives U's eigenvalues, V its eigenvectors (columns),
// which dR_polar reuses (the reference decomposes U again; it has the same
// eigenbasis and eigenvalues).
void polar_RU(const double F[3][3], double R[3][3], double Um[3][3], double V[3][3], double mu[3]) {
  double Ft[3][3], C[3][3];
  tr3(F, Ft);
  mul3(Ft, F, C);
  double w[3];
  eig3(C, w, V);
  double isq[3];
  for (int A = 0; A < 3; ++A) {
    mu[A] = std::sqrt(std::max(w[A], 0.0));
    isq[A] = mu[A] > 0 ? 1.0 / mu[A] : 0.0;
  }
  double Ui[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double u = 0.0, ui = 0.0;
      for (int A = 0; A < 3; ++A) {
        u += V[i][A] * mu[A] * V[j][A];
        ui += V[i][A] * isq[A] * V[j][A];
      }
      Um[i][j] = u;
      Ui[i][j] = ui;
    }
  mul3(F, Ui, R);
}

// dR_polar (FiniteStrain.jl:220-233): Omega U + U Omega = R^T dF - dF^T R solved
// in U's eigenbasis, dR = R Omega.
void dR_polar(const double R[3][3], const double V[3][3], const double mu[3], const double dF[3][3],
              double dR[3][3]) {
  double Rt[3][3], A[3][3], rhs[3][3];
  tr3(R, Rt);
  mul3(Rt, dF, A);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) rhs[i][j] = A[i][j] - A[j][i];
  double Vt[3][3], T[3][3], rb[3][3];
  tr3(V, Vt);
  mul3(Vt, rhs, T);
  mul3(T, V, rb);
  double Ob[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Ob[i][j] = rb[i][j] / (mu[i] + mu[j]);
  double O[3][3];
  mul3(V, Ob, T);
  mul3(T, Vt, O);
  mul3(R, O, dR);
}

// dtau_dbeta (FiniteStrain.jl:250-268), row-major 6x6: zero in the elastic
// branch, else a I + xi (x) g with g = (da/dnrm / nrm) W xi.
void dtau_dbeta(const Mat& m, double sy0, const double eps_tr[6], const double beta_sp[6], double alpha_n,
                double out[36]) {
  std::memset(out, 0, 36 * sizeof(double));
  const double G = m.G, H = m.Hiso + m.Hkin, s32 = std::sqrt(1.5);
  double C[36];
  cmat(m, C);
  double st[6];
  for (int i = 0; i < 6; ++i) {
    double t = 0.0;
    for (int j = 0; j < 6; ++j) t += C[i * 6 + j] * eps_tr[j];
    st[i] = t;
  }
  const double p = (st[0] + st[1] + st[2]) / 3.0;
  double xi[6];
  for (int i = 0; i < 6; ++i) xi[i] = st[i] - (i < 3 ? p : 0.0) - beta_sp[i];
  const double nrm = devnorm(xi);
  const double Y = sy0 + m.Hiso * alpha_n;
  const double f = s32 * nrm - Y;
  if (f <= 0.0) return;
  const double dg = f / (3.0 * G + H);
  const double a = 2.0 * G * s32 * dg / nrm;
  const double da = 2.0 * G * s32 / (3.0 * G + H) * (Y / (nrm * nrm));
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j)
      out[i * 6 + j] = (i == j ? a : 0.0) + xi[i] * (da / nrm) * (j < 3 ? 1.0 : 2.0) * xi[j];
}

struct Upd {
  double tau[6], epsp_inc[6], alpha_new, D[36], cpi_new[6], ftr;
  double beta_ref_new[6], beta_sp[6], R[3][3], Um[3][3], V[3][3], mu[3];
  int plastic;
};

// finite_stress_update (FiniteStrain.jl:292-346).  With Hkin > 0 the back
// stress is stored in the reference configuration: beta_sp = R beta_ref R^T
// enters the return map and the update is pulled back, beta_ref_new =
// R^T beta_sp_new R (:316-324).  With Hkin = 0, R = U = I and beta_sp = 0.
Upd finite_stress_update(const Mat& m, double sigy0, const Kin& k, const double F[3][3], double alpha_n,
                         const double* beta_ref_n) {
  Upd u;
  const double Z6[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) u.R[i][j] = u.Um[i][j] = u.V[i][j] = (i == j) ? 1.0 : 0.0;
  u.mu[0] = u.mu[1] = u.mu[2] = 1.0;
  std::memset(u.beta_sp, 0, sizeof(u.beta_sp));
  const bool kin = m.Hkin > 0;
  if (kin) {
    polar_RU(F, u.R, u.Um, u.V, u.mu);
    double B[3][3], T[3][3], Rt[3][3], S[3][3];
    v2s(beta_ref_n, B);
    tr3(u.R, Rt);
    mul3(u.R, B, T);
    mul3(T, Rt, S);
    s2v(S, u.beta_sp);
  }
  double beta_new[6];
  u.plastic = return_map(m, sigy0, k.eps_tr, Z6, u.beta_sp, alpha_n, u.tau, u.epsp_inc, beta_new,
                         &u.alpha_new, u.D, &u.ftr);
  if (kin) {
    double B[3][3], T[3][3], Rt[3][3], S[3][3];
    v2s(beta_new, B);
    tr3(u.R, Rt);
    mul3(Rt, B, T);
    mul3(T, u.R, S);
    s2v(S, u.beta_ref_new);
  } else {
    std::memcpy(u.beta_ref_new, beta_new, sizeof(beta_new));
  }
  double ee[6];
  for (int i = 0; i < 6; ++i) ee[i] = k.eps_tr[i] - u.epsp_inc[i];
  double E2[3][3] = {{2 * ee[0], ee[3], ee[5]}, {ee[3], 2 * ee[1], ee[4]}, {ee[5], ee[4], 2 * ee[2]}};
  double w[3], V[3][3];
  eig3(E2, w, V);
  double be[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      be[i][j] = std::exp(w[0]) * V[i][0] * V[j][0] + std::exp(w[1]) * V[i][1] * V[j][1] +
                 std::exp(w[2]) * V[i][2] * V[j][2];
  double T[3][3], FinvT[3][3], C[3][3];
  mul3(k.Finv, be, T);
  tr3(k.Finv, FinvT);
  mul3(T, FinvT, C);
  s2v(C, u.cpi_new);
  return u;
}

// _dhalflog_contract, FiniteStrain.jl:463-482.
void dhalflog_contract(const double Q[3][3], const double b[3], const double H[3][3],
                       double out[3][3]) {
  double Qt[3][3], T[3][3], Hp[3][3];
  tr3(Q, Qt);
  mul3(Qt, H, T);
  mul3(T, Q, Hp);
  double ly[3];
  for (int A = 0; A < 3; ++A) ly[A] = 0.5 * std::log(b[A]);
  double Yp[3][3];
  for (int A = 0; A < 3; ++A)
    for (int B = 0; B < 3; ++B) {
      double g;
      if (A == B) g = 1.0 / (2.0 * b[A]);
      else if (std::fabs(b[A] - b[B]) < EIG_TOL * (std::fabs(b[A]) + std::fabs(b[B]) + 1.0))
        g = 1.0 / (b[A] + b[B]);
      else g = (ly[A] - ly[B]) / (b[A] - b[B]);
      Yp[A][B] = g * Hp[A][B];
    }
  mul3(Q, Yp, T);
  mul3(T, Qt, out);
}

// dPdF (FiniteStrain.jl:503-547).  A9 is 9x9 row-major with both indices
// column-major F/P order.  kin (non-null) carries the kinematic-hardening
// coupling dtau/dbeta_sp . dbeta_sp/dF through the polar rotation (:532-536).
struct KinTerm {
  double Bref[3][3], R[3][3], V[3][3], mu[3], dtdb[36];
};
void dPdF(const Kin& k, const double cpi_v[6], const double D[36], const double tau_v[6],
          const double F[3][3], double A9[81], const KinTerm* kin = nullptr) {
  double Cpi[3][3], tau[3][3], FinvT[3][3], Ft[3][3];
  v2s(cpi_v, Cpi);
  v2s(tau_v, tau);
  tr3(k.Finv, FinvT);
  tr3(F, Ft);
  double CpiFt[3][3], FCpi[3][3];
  mul3(Cpi, Ft, CpiFt);
  mul3(F, Cpi, FCpi);
  for (int col = 0; col < 9; ++col) {
    const int p = col % 3, q = col / 3;
    double dF[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    dF[p][q] = 1.0;
    double dFt[3][3], t1[3][3], t2[3][3], dbe[3][3];
    tr3(dF, dFt);
    mul3(dF, CpiFt, t1);
    mul3(FCpi, dFt, t2);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dbe[i][j] = t1[i][j] + t2[i][j];
    double de[3][3];
    dhalflog_contract(k.n, k.b, dbe, de);
    const double dev[6] = {de[0][0], de[1][1], de[2][2], 2 * de[0][1], 2 * de[1][2], 2 * de[0][2]};
    double dtv[6];
    for (int i = 0; i < 6; ++i) {
      double s = 0.0;
      for (int j = 0; j < 6; ++j) s += D[i * 6 + j] * dev[j];
      dtv[i] = s;
    }
    if (kin) {
      double dR[3][3], Rt[3][3], dRt[3][3], T1[3][3], T2[3][3], T3[3][3], T4[3][3], db[3][3];
      dR_polar(kin->R, kin->V, kin->mu, dF, dR);
      tr3(kin->R, Rt);
      tr3(dR, dRt);
      mul3(dR, kin->Bref, T1);
      mul3(T1, Rt, T2);
      mul3(kin->R, kin->Bref, T3);
      mul3(T3, dRt, T4);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) db[i][j] = T2[i][j] + T4[i][j];
      double dbv[6];
      s2v(db, dbv);
      for (int i = 0; i < 6; ++i) {
        double s = 0.0;
        for (int j = 0; j < 6; ++j) s += kin->dtdb[i * 6 + j] * dbv[j];
        dtv[i] += s;
      }
    }
    double dt[3][3];
    v2s(dtv, dt);
    double a1[3][3], a2[3][3], dFinvT[3][3];
    mul3(FinvT, dFt, a1);
    mul3(a1, FinvT, a2);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dFinvT[i][j] = -a2[i][j];
    double p1[3][3], p2[3][3];
    mul3(dt, FinvT, p1);
    mul3(tau, dFinvT, p2);
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) A9[(c * 3 + r) * 9 + col] = p1[r][c] + p2[r][c];
  }
}

// Hex8 natural node coordinates and Gauss points, Elements.jl:26-43.
const double NODE_NAT[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                               {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
const double GSGN[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// hex8_dshape, Elements.jl:62-75.
void dshape(const double xi[3], double dN[8][3]) {
  for (int a = 0; a < 8; ++a) {
    const double xa = NODE_NAT[a][0], ya = NODE_NAT[a][1], za = NODE_NAT[a][2];
    dN[a][0] = 0.125 * xa * (1 + ya * xi[1]) * (1 + za * xi[2]);
    dN[a][1] = 0.125 * ya * (1 + xa * xi[0]) * (1 + za * xi[2]);
    dN[a][2] = 0.125 * za * (1 + xa * xi[0]) * (1 + ya * xi[1]);
  }
}

// Reference gradients dN/dX = dN * inv(J), J = Xe' * dN (Elements.jl:89,
// :155-161); returns det(J) (times weight 1, Elements.jl:43, :139).
double ref_grads(const double Xe[8][3], const double xi[3], double dNdX[8][3]) {
  double dN[8][3];
  dshape(xi, dN);
  double J[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int a = 0; a < 8; ++a) s += Xe[a][i] * dN[a][j];
      J[i][j] = s;
    }
  double Ji[3][3];
  inv3(J, Ji);
  for (int a = 0; a < 8; ++a)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int m = 0; m < 3; ++m) s += dN[a][m] * Ji[m][j];
      dNdX[a][j] = s;
    }
  return det3(J);
}

// deformation_gradient, FiniteStrain.jl:107-119.
void defgrad(const double ue[24], const double dNdX[8][3], double F[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int a = 0; a < 8; ++a) s += ue[3 * a + i] * dNdX[a][j];
      F[i][j] = s;
    }
}

// _Gmatrix, Elements.jl:500-510 (9x24 row-major, rows column-major F index).
void Gmatrix(const double dNdX[8][3], double G[9 * 24]) {
  for (int r = 0; r < 9; ++r) {
    const int i = r % 3, j = r / 3;
    for (int c = 0; c < 24; ++c) {
      const int a = c / 3, k = c % 3;
      G[r * 24 + c] = (i == k) ? dNdX[a][j] : 0.0;
    }
  }
}

inline void p9(const double P[3][3], double v[9]) {  // _p9, Elements.jl:513-514
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) v[c * 3 + r] = P[r][c];
}

}  // namespace

extern "C" {

// ---- material / kinematics entry points (reference tests T1-T7, F3-F5) ----

int or_return_map(const double* mat7, const double* eps6, const double* epsp6,
                  const double* beta6, double alpha_n, double* sig6, double* epsp_new6,
                  double* beta_new6, double* alpha_new, double* D36) {
  Mat m = make_mat(mat7);
  return return_map(m, m.sigy0, eps6, epsp6, beta6, alpha_n, sig6, epsp_new6, beta_new6,
                    alpha_new, D36, nullptr);
}

// F given column-major 9 (F[j*3+i] = F_ij).  beta6: committed back stress in
// the reference configuration (null = 0).  Returns -1 when det F <= 0, else
// the plastic flag.
int or_finite_update(const double* mat7, const double* F9, const double* cpi6, double alpha_n,
                     const double* beta6, double* tau6, double* cpi_new6, double* alpha_new,
                     double* beta_new6, double* epsp_inc6, double* D36, double* A81) {
  Mat m = make_mat(mat7);
  double F[3][3];
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) F[i][j] = F9[j * 3 + i];
  Kin k = finite_kinematics(F, cpi6);
  if (!k.ok) return -1;
  const double Z6[6] = {0, 0, 0, 0, 0, 0};
  const double* bn = beta6 ? beta6 : Z6;
  Upd u = finite_stress_update(m, m.sigy0, k, F, alpha_n, bn);
  std::memcpy(tau6, u.tau, sizeof(u.tau));
  std::memcpy(cpi_new6, u.cpi_new, sizeof(u.cpi_new));
  *alpha_new = u.alpha_new;
  if (beta_new6) std::memcpy(beta_new6, u.beta_ref_new, sizeof(u.beta_ref_new));
  if (epsp_inc6) std::memcpy(epsp_inc6, u.epsp_inc, sizeof(u.epsp_inc));
  if (D36) std::memcpy(D36, u.D, sizeof(u.D));
  if (A81) {
    if (m.Hkin > 0) {
      KinTerm kt;
      v2s(bn, kt.Bref);
      std::memcpy(kt.R, u.R, sizeof(kt.R));
      std::memcpy(kt.V, u.V, sizeof(kt.V));
      std::memcpy(kt.mu, u.mu, sizeof(kt.mu));
      dtau_dbeta(m, m.sigy0, k.eps_tr, u.beta_sp, alpha_n, kt.dtdb);
      dPdF(k, cpi6, u.D, u.tau, F, A81, &kt);
    } else {
      dPdF(k, cpi6, u.D, u.tau, F, A81);
    }
  }
  return u.plastic;
}

// Element force / tangent for one Hex8 element,
// fbar = 0: element_force_tangent_finite!, Elements.jl:405-494 (Hkin = 0);
// fbar = 1: the same with the
// F-bar chain of _fbar_Geff, Elements.jl:524-531; fbar = 2: the small-strain
// element_force_tangent!, Elements.jl:323-360 (state slot = eps_p, tau = sigma).
//   Xe24: node-major coordinates (a*3 + d); ue24 node-major displacements.
//   cpi48 / alpha8 / beta48: committed state per Gauss point (g*6 + c, g);
//   beta48 (null = 0) is the back stress (reference configuration for the
//   finite kinds), beta_new48 (nullable) receives its update.
//   Ke576 row-major 24x24.  tau48 Kirchhoff stress per GP.  flags8 = f_tr>0.
// Returns 0, or -(g+1) for the first inverted Gauss point g (J in *badJ).
int or_element(int fbar, const double* mat7, double sigy0, const double* Xe24,
               const double* ue24, const double* cpi48, const double* alpha8, const double* beta48,
               double* Fe24, double* Ke576, double* tau48, double* cpi_new48, double* alpha_new8,
               double* beta_new48, double* epsp_inc48, unsigned char* flags8, double* badJ) {
  Mat m = make_mat(mat7);
  static const double Z48[48] = {0};
  if (!beta48) beta48 = Z48;
  double Xe[8][3];
  for (int a = 0; a < 8; ++a)
    for (int d = 0; d < 3; ++d) Xe[a][d] = Xe24[a * 3 + d];
  if (fbar == 2) {
    // Small strain: element_force_tangent!, Elements.jl:323-360, with bmatrix
    // :97-117 and return_map.  The state slot cpi48 carries eps_p (6 per GP,
    // engineering shear), tau48 receives sigma.
    const double g = 1.0 / std::sqrt(3.0);
    std::memset(Fe24, 0, 24 * sizeof(double));
    std::memset(Ke576, 0, 576 * sizeof(double));
    for (int gp = 0; gp < 8; ++gp) {
      const double xi[3] = {GSGN[gp][0] * g, GSGN[gp][1] * g, GSGN[gp][2] * g};
      double dNdX[8][3];
      const double w = ref_grads(Xe, xi, dNdX);
      double B[6 * 24];
      std::memset(B, 0, sizeof(B));
      for (int a = 0; a < 8; ++a) {
        const double Nx = dNdX[a][0], Ny = dNdX[a][1], Nz = dNdX[a][2];
        B[0 * 24 + 3 * a + 0] = Nx;
        B[1 * 24 + 3 * a + 1] = Ny;
        B[2 * 24 + 3 * a + 2] = Nz;
        B[3 * 24 + 3 * a + 0] = Ny; B[3 * 24 + 3 * a + 1] = Nx;
        B[4 * 24 + 3 * a + 1] = Nz; B[4 * 24 + 3 * a + 2] = Ny;
        B[5 * 24 + 3 * a + 0] = Nz; B[5 * 24 + 3 * a + 2] = Nx;
      }
      double eps[6];
      for (int r = 0; r < 6; ++r) {
        double t = 0.0;
        for (int c = 0; c < 24; ++c) t += B[r * 24 + c] * ue24[c];
        eps[r] = t;
      }
      double sig[6], ep_new[6], b_new[6], a_new, D[36];
      const int pl = return_map(m, sigy0, eps, cpi48 + gp * 6, beta48 + gp * 6, alpha8[gp], sig, ep_new, b_new,
                                &a_new, D, nullptr);
      if (beta_new48) std::memcpy(beta_new48 + gp * 6, b_new, sizeof(b_new));
      for (int c = 0; c < 24; ++c) {
        double t = 0.0;
        for (int r = 0; r < 6; ++r) t += B[r * 24 + c] * sig[r];
        Fe24[c] += t * w;
      }
      double DB[6 * 24];
      for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 24; ++c) {
          double t = 0.0;
          for (int q = 0; q < 6; ++q) t += D[r * 6 + q] * B[q * 24 + c];
          DB[r * 24 + c] = t;
        }
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
          double t = 0.0;
          for (int r = 0; r < 6; ++r) t += B[r * 24 + i] * DB[r * 24 + j];
          Ke576[i * 24 + j] += t * w;
        }
      for (int c = 0; c < 6; ++c) {
        if (tau48) tau48[gp * 6 + c] = sig[c];
        if (cpi_new48) cpi_new48[gp * 6 + c] = ep_new[c];
        if (epsp_inc48) epsp_inc48[gp * 6 + c] = ep_new[c] - cpi48[gp * 6 + c];
      }
      if (alpha_new8) alpha_new8[gp] = a_new;
      if (flags8) flags8[gp] = (unsigned char)pl;
    }
    return 0;
  }
  const double g = 1.0 / std::sqrt(3.0);
  double dNdX0[8][3], F0[3][3], J0 = 1.0, g0[24];
  if (fbar) {
    const double c0[3] = {0, 0, 0};
    ref_grads(Xe, c0, dNdX0);
    defgrad(ue24, dNdX0, F0);
    J0 = det3(F0);
    double F0i[3][3];
    inv3(F0, F0i);
    // g0 = G0' * vec(F0^{-T}) :  g0_(a,k) = sum_j F0^{-T}_kj dNdX0_aj
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s += F0i[j][k] * dNdX0[a][j];
        g0[a * 3 + k] = s;
      }
  }
  std::memset(Fe24, 0, 24 * sizeof(double));
  std::memset(Ke576, 0, 576 * sizeof(double));
  for (int gp = 0; gp < 8; ++gp) {
    const double xi[3] = {GSGN[gp][0] * g, GSGN[gp][1] * g, GSGN[gp][2] * g};
    double dNdX[8][3];
    const double w = ref_grads(Xe, xi, dNdX);
    double F[3][3];
    defgrad(ue24, dNdX, F);
    const double Jg = det3(F);
    const double scale = fbar ? std::cbrt(J0 / Jg) : 1.0;
    double Fb[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Fb[i][j] = scale * F[i][j];
    Kin k = finite_kinematics(Fb, cpi48 + gp * 6);
    if (!k.ok) {
      if (badJ) *badJ = k.J;
      return -(gp + 1);
    }
    Upd u = finite_stress_update(m, sigy0, k, Fb, alpha8[gp], beta48 + gp * 6);
    double Gm[9 * 24];
    Gmatrix(dNdX, Gm);
    double tau[3][3], FinvT[3][3], P[3][3];
    v2s(u.tau, tau);
    tr3(k.Finv, FinvT);
    mul3(tau, FinvT, P);  // first_piola, FiniteStrain.jl:560-561
    double Pv[9];
    p9(P, Pv);
    double A[81];
    if (m.Hkin > 0) {
      KinTerm kt;
      v2s(beta48 + gp * 6, kt.Bref);
      std::memcpy(kt.R, u.R, sizeof(kt.R));
      std::memcpy(kt.V, u.V, sizeof(kt.V));
      std::memcpy(kt.mu, u.mu, sizeof(kt.mu));
      dtau_dbeta(m, sigy0, k.eps_tr, u.beta_sp, alpha8[gp], kt.dtdb);
      dPdF(k, cpi48 + gp * 6, u.D, u.tau, Fb, A, &kt);
    } else {
      dPdF(k, cpi48 + gp * 6, u.D, u.tau, Fb, A);
    }
    for (int c = 0; c < 24; ++c) {
      double s = 0.0;
      for (int r = 0; r < 9; ++r) s += Gm[r * 24 + c] * Pv[r];
      Fe24[c] += s * w;
    }
    double Geff[9 * 24];
    if (fbar) {
      double Fi[3][3], FiT[3][3];
      inv3(F, Fi);
      tr3(Fi, FiT);
      double vFiT[9], vF[9];
      p9(FiT, vFiT);
      p9(F, vF);
      double gJ[24];
      for (int c = 0; c < 24; ++c) {
        double s = 0.0;
        for (int r = 0; r < 9; ++r) s += Gm[r * 24 + c] * vFiT[r];
        gJ[c] = s;
      }
      for (int r = 0; r < 9; ++r)
        for (int c = 0; c < 24; ++c)
          Geff[r * 24 + c] = scale * Gm[r * 24 + c] + (scale / 3.0) * vF[r] * (g0[c] - gJ[c]);
    } else {
      std::memcpy(Geff, Gm, sizeof(Geff));
    }
    double AG[9 * 24];
    for (int r = 0; r < 9; ++r)
      for (int c = 0; c < 24; ++c) {
        double s = 0.0;
        for (int t = 0; t < 9; ++t) s += A[r * 9 + t] * Geff[t * 24 + c];
        AG[r * 24 + c] = s;
      }
    for (int r = 0; r < 24; ++r)
      for (int c = 0; c < 24; ++c) {
        double s = 0.0;
        for (int t = 0; t < 9; ++t) s += Gm[t * 24 + r] * AG[t * 24 + c];
        Ke576[r * 24 + c] += s * w;
      }
    if (tau48) std::memcpy(tau48 + gp * 6, u.tau, 6 * sizeof(double));
    if (cpi_new48) std::memcpy(cpi_new48 + gp * 6, u.cpi_new, 6 * sizeof(double));
    if (alpha_new8) alpha_new8[gp] = u.alpha_new;
    if (beta_new48) std::memcpy(beta_new48 + gp * 6, u.beta_ref_new, 6 * sizeof(double));
    if (epsp_inc48) std::memcpy(epsp_inc48 + gp * 6, u.epsp_inc, 6 * sizeof(double));
    if (flags8) flags8[gp] = (unsigned char)u.plastic;
  }
  return 0;
}

// ---- mesh topology: sparsity pattern, element colors ----

// Number of stored entries of the CSC pattern, build_sparsity,
// Assembly.jl:99-111 (node adjacency :62-82).  elem is 8 x ne, 1-based,
// column-major (elem[e*8 + a]).
int64_t or_pattern_nnz(int64_t nn, int64_t ne, const int64_t* elem) {
  std::vector<std::vector<int64_t>> adj(nn);
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) adj[elem[e * 8 + a] - 1].push_back(elem[e * 8 + b]);
  int64_t tot = 0;
  for (int64_t n = 0; n < nn; ++n) {
    auto& v = adj[n];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    tot += 3 * (int64_t)v.size();
  }
  return tot * 3;
}

// Fill colptr (3nn+1) / rowval (nnz), 1-based, count-then-fill,
// Assembly.jl:119-146.
void or_pattern_fill(int64_t nn, int64_t ne, const int64_t* elem, int64_t* colptr,
                     int64_t* rowval) {
  std::vector<std::vector<int64_t>> adj(nn);
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) adj[elem[e * 8 + a] - 1].push_back(elem[e * 8 + b]);
  for (auto& v : adj) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  colptr[0] = 1;
  for (int64_t j = 0; j < nn; ++j) {
    const int64_t ncol = 3 * (int64_t)adj[j].size();
    for (int c = 0; c < 3; ++c) colptr[3 * j + c + 1] = colptr[3 * j + c] + ncol;
  }
  for (int64_t j = 0; j < nn; ++j)
    for (int c = 0; c < 3; ++c) {
      int64_t p = colptr[3 * j + c] - 1;
      for (int64_t nb : adj[j]) {
        const int64_t r0 = 3 * (nb - 1);
        rowval[p] = r0 + 1; rowval[p + 1] = r0 + 2; rowval[p + 2] = r0 + 3;
        p += 3;
      }
    }
}

// element_colors + _box_dims, Assembly.jl:172-206.  nodes 3 x nn
// column-major.  Writes the 0-based color of every element (colors renumbered
// after dropping empty ones, as the reference does) and returns the count.
int or_element_colors(int64_t nn, int64_t ne, const double* nodes, int64_t* color) {
  if (ne == 0) return 0;
  // round(x; digits=12) then unique, Assembly.jl:197-199
  int64_t dims[3];
  for (int d = 0; d < 3; ++d) {
    std::vector<double> v(nn);
    for (int64_t n = 0; n < nn; ++n) v[n] = std::round(nodes[n * 3 + d] * 1e12) / 1e12;
    std::sort(v.begin(), v.end());
    dims[d] = (int64_t)(std::unique(v.begin(), v.end()) - v.begin()) - 1;
  }
  const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
  if (!(nx >= 1 && ny >= 1 && nz >= 1 && nx * ny * nz == ne &&
        (nx + 1) * (ny + 1) * (nz + 1) == nn)) {
    for (int64_t e = 0; e < ne; ++e) color[e] = 0;
    return 1;
  }
  int64_t raw[8] = {0};
  std::vector<int> c8(ne);
  int64_t e = 0;
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        const int c = (int)((i & 1) + 2 * (j & 1) + 4 * (k & 1));
        c8[e++] = c;
        raw[c]++;
      }
  int remap[8], nc = 0;
  for (int c = 0; c < 8; ++c) remap[c] = raw[c] ? nc++ : -1;
  for (int64_t q = 0; q < ne; ++q) color[q] = remap[c8[q]];
  return nc;
}

// ---- global assembly (Assembly.jl:238-331) ----
//
// Serial-order scatter (element order 1..ne, the reference `assemble!`) of
// element contributions into the CSC nzval and R; elements are evaluated in
// parallel chunks, the scatter itself runs in element order so the result is
// independent of the thread count.  State arrays are 6 x ngp column-major.
// commit != 0 writes cpi/alpha/epsp in place (Elements.jl:483-491).
// Returns 0, or -1 on an inverted element (bad_e 1-based, bad_g 1-based, badJ).
int or_assemble(int fbar, const double* mat7, const double* sigy0_e, int64_t nn, int64_t ne,
                const double* nodes, const int64_t* elem, const int64_t* colptr,
                const int64_t* rowval, const double* U, double* cpi, double* alpha,
                double* epsp, double* beta, int commit, double* nzval, double* R, double* tau,
                unsigned char* flags, int nthreads, int64_t* bad_e, int* bad_g, double* badJ) {
  const int64_t ndof = 3 * nn;
  const int64_t nnz = colptr[ndof] - 1;
  std::fill(nzval, nzval + nnz, 0.0);
  std::fill(R, R + ndof, 0.0);
  const int64_t CH = 2048;
  std::vector<double> Fe(CH * 24), Ke(CH * 576);
  std::vector<double> cnew(CH * 48), anew(CH * 8), pinc(CH * 48), bnew(beta ? CH * 48 : 0);
  std::vector<int> st(CH);
  std::vector<double> sJ(CH);
  const int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  for (int64_t e0 = 0; e0 < ne; e0 += CH) {
    const int64_t e1 = std::min(ne, e0 + CH);
    parallel_for(e1 - e0, nt, 16, [&](int64_t q) {
      const int64_t e = e0 + q;
      double Xe[24], ue[24];
      for (int a = 0; a < 8; ++a) {
        const int64_t nd = elem[e * 8 + a] - 1;
        for (int d = 0; d < 3; ++d) {
          Xe[a * 3 + d] = nodes[nd * 3 + d];
          ue[a * 3 + d] = U[nd * 3 + d];
        }
      }
      const double sy = sigy0_e ? sigy0_e[e] : mat7[2];
      st[q] = or_element(fbar, mat7, sy, Xe, ue, cpi + e * 48, alpha + e * 8, beta ? beta + e * 48 : nullptr,
                         &Fe[q * 24], &Ke[q * 576], tau ? tau + e * 48 : nullptr, &cnew[q * 48],
                         &anew[q * 8], beta ? &bnew[q * 48] : nullptr, &pinc[q * 48],
                         flags ? flags + e * 8 : nullptr, &sJ[q]);
    });
    for (int64_t e = e0; e < e1; ++e) {
      const int64_t q = e - e0;
      if (st[q] != 0) {
        if (bad_e) *bad_e = e + 1;
        if (bad_g) *bad_g = -st[q];
        if (badJ) *badJ = sJ[q];
        return -1;
      }
      int64_t ed[24];
      for (int c = 0; c < 24; ++c) ed[c] = 3 * (elem[e * 8 + c / 3] - 1) + (c % 3) + 1;
      for (int c = 0; c < 24; ++c) {
        const int64_t gc = ed[c];
        for (int r = 0; r < 24; ++r) {
          // _find_nz binary search, Assembly.jl:210-224
          int64_t lo = colptr[gc - 1], hi = colptr[gc] - 1, idx = 0;
          const int64_t gr = ed[r];
          while (lo <= hi) {
            const int64_t mid = (lo + hi) >> 1;
            const int64_t rv = rowval[mid - 1];
            if (rv == gr) { idx = mid; break; }
            if (rv < gr) lo = mid + 1; else hi = mid - 1;
          }
          nzval[idx - 1] += Ke[q * 576 + r * 24 + c];
        }
      }
      for (int i = 0; i < 24; ++i) R[ed[i] - 1] += Fe[q * 24 + i];
      if (commit) {
        std::memcpy(cpi + e * 48, &cnew[q * 48], 48 * sizeof(double));
        std::memcpy(alpha + e * 8, &anew[q * 8], 8 * sizeof(double));
        if (beta) std::memcpy(beta + e * 48, &bnew[q * 48], 48 * sizeof(double));
        if (epsp)
          for (int i = 0; i < 48; ++i) epsp[e * 48 + i] += pinc[q * 48 + i];
      }
    }
  }
  return 0;
}

// impose_dirichlet!, BoundaryConditions.jl:62-109, on a 1-based CSC matrix.
void or_impose_dirichlet(int64_t n, const int64_t* colptr, const int64_t* rowval, double* nzval,
                         double* R, int64_t nbc, const int64_t* dofs, const double* vals,
                         int ramp, double lam, const double* U) {
  std::vector<char> isbc(n, 0);
  std::vector<double> dg(n, 0.0);
  for (int64_t i = 0; i < nbc; ++i) {
    const int64_t d = dofs[i] - 1;
    const double g = ramp ? lam * vals[i] : vals[i];
    isbc[d] = 1;
    dg[d] = g - U[d];
  }
  for (int64_t col = 0; col < n; ++col)
    for (int64_t k = colptr[col] - 1; k < colptr[col + 1] - 1; ++k) {
      const int64_t row = rowval[k] - 1;
      if (isbc[col] && !isbc[row]) R[row] += nzval[k] * dg[col];
    }
  for (int64_t col = 0; col < n; ++col)
    for (int64_t k = colptr[col] - 1; k < colptr[col + 1] - 1; ++k) {
      const int64_t row = rowval[k] - 1;
      if (isbc[col] || isbc[row]) nzval[k] = (row == col && isbc[row]) ? 1.0 : 0.0;
    }
  for (int64_t i = 0; i < nbc; ++i) {
    const int64_t d = dofs[i] - 1;
    R[d] = -dg[d];
  }
}

}  // extern "C"
