// element.cu -- K1: fused per-color F-bar Hex8 element kernel + colored scatter.
//
// One warp owns four elements of one color.  Phase A: lane (slot, g) evaluates
// Gauss point g of element `slot`: geometry, F / F-bar, trial b^e and its
// eigenbasis, the J2 radial return in principal stresses, P = tau F^-T and the
// two-point tangent A = dP/dFbar built column by column in the eigenbasis of
// b^e.  The internal force is summed over the element's eight Gauss-point
// lanes node by node with warp shuffles (FP64) and added into R; the tangent
// records (dN/dX, w s A, w s/3 A vec(F), F^-1) go to shared memory in the
// tangent's type TT (FP32 on the mixed-precision path, where only the tangent
// is FP32).  The Kirchhoff stress and the elastic/plastic flag are written,
// and on the commit pass the exponential-map plastic update.  Phase B: the
// 4 x 24 columns (b,k) of the warp's four element tangents are spread over the
// 32 lanes; each sums the eight Gauss-point contributions
//   Ke[:,(b,k)] = sum_g G_g^T (w s A G_g + (w s/3) A vec(F) (g0 - gJ)^T)[:,(b,k)]
// (lagrangian/src/Elements.jl:470-478 with _fbar_Geff :524-531) and adds them
// into the 3x3-block CSR tangent in place.  Elements of one color share no
// node, so the adds need no atomics (lagrangian/src/Assembly.jl:167-188,
// :370-385).
//
// Arithmetic follows the reference kernel element_force_tangent_finite!
// (Elements.jl:405-494), finite_kinematics (FiniteStrain.jl:148-170),
// return_map (Materials.jl:159-250; linear or saturation isotropic hardening,
// or linear kinematic hardening through the polar rotation, HARD),
// finite_stress_update (FiniteStrain.jl:292-346) and dPdF with
// _dhalflog_contract (FiniteStrain.jl:463-547).  The return map is evaluated
// on principal values: the trial stress is an isotropic function of b^e, so
// its deviator and the flow direction share b^e's eigenbasis, and the
// reference's global-Voigt formulas reduce to these principal ones exactly.
#include <type_traits>

#include "common.cuh"
#include "pfem_internal.h"

namespace pfem {

constexpr int EPW = 4;                     // elements per warp
constexpr int GPREC = 24 + 81 + 9 + 9;     // dNdX, w s A, w s/3 A vec(F), F^-1 (TT each)
constexpr int SLOT_TT = 24 + 8 * GPREC;    // g0, then the 8 Gauss-point records
constexpr int WPB = 1;                     // warps per block
// Shared memory per warp (bytes).  The element's nodal coordinates and
// displacements (48 doubles) live at the start of the record area until the
// geometry is formed, then the records overwrite them.
template <typename TT>
constexpr int warp_smem_bytes(bool commit) {
  return commit ? EPW * 48 * 8 : EPW * SLOT_TT * (int)sizeof(TT);
}
static_assert(8 * GPREC * 4 >= 48 * 8, "coordinate scratch must fit in the record area");

__device__ __forceinline__ double nsgn_x(int a) { return (((a + 1) >> 1) & 1) ? 1.0 : -1.0; }
__device__ __forceinline__ double nsgn_y(int a) { return ((a >> 1) & 1) ? 1.0 : -1.0; }
__device__ __forceinline__ double nsgn_z(int a) { return (a >> 2) ? 1.0 : -1.0; }

// hex8_dshape (Elements.jl:62-75) at natural point (x, y, z) for node a.
__device__ __forceinline__ void dshape_a(int a, double x, double y, double z, double* d) {
  const double xa = nsgn_x(a), ya = nsgn_y(a), za = nsgn_z(a);
  d[0] = 0.125 * xa * (1.0 + ya * y) * (1.0 + za * z);
  d[1] = 0.125 * ya * (1.0 + xa * x) * (1.0 + za * z);
  d[2] = 0.125 * za * (1.0 + xa * x) * (1.0 + ya * y);
}

// ---- saturation (Voce) hardening: yield_stress / yield_slope (Materials.jl:117-127)
// and the scalar local Newton on dgamma of the plastic corrector (:201-213).
// sy0 is the element's initial yield stress; m.sat = sigsat - sigy0.
__device__ __forceinline__ double voce_ys(const MatParams& m, double sy0, double a) {
  return sy0 + m.sat * (1.0 - exp(-m.delta * a)) + m.Hiso * a;
}
__device__ __forceinline__ double voce_slope(const MatParams& m, double a) {
  return m.delta * m.sat * exp(-m.delta * a) + m.Hiso;
}
// Returns dgamma; *Hp receives the plastic modulus at alpha_n + dgamma.
__device__ __forceinline__ double voce_dgamma(const MatParams& m, double sy0, double qtr, double an, double ftr,
                                              double* Hp) {
  const double c = 3.0 * m.G + m.Hkin;
  double dg = ftr / (c + voce_slope(m, an));
  for (int it = 0; it < 50; ++it) {
    const double r = qtr - c * dg - voce_ys(m, sy0, an + dg);
    const double d = r / (c + voce_slope(m, an + dg));
    dg += d;
    if (fabs(d) <= 1e-13 * (dg + 1e-14)) break;
  }
  *Hp = voce_slope(m, an + dg);
  return dg;
}

// ---- symmetric 3x3 tensors packed as [00, 11, 22, 01, 12, 02] (physical shear) ----
template <typename T>
__device__ __forceinline__ void unpack_sym(const T* s, T* M) {
  M[0] = s[0]; M[4] = s[1]; M[8] = s[2];
  M[1] = s[3]; M[3] = s[3];
  M[5] = s[4]; M[7] = s[4];
  M[2] = s[5]; M[6] = s[5];
}
// out = A S A^T (S full symmetric), packed
template <typename T>
__device__ __forceinline__ void congruence(const T* A, const T* S, T* out) {
  T AS[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) AS[3 * i + j] = A[3 * i] * S[j] + A[3 * i + 1] * S[3 + j] + A[3 * i + 2] * S[6 + j];
  constexpr int I[6] = {0, 1, 2, 0, 1, 0}, J[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int c = 0; c < 6; ++c)
    out[c] = AS[3 * I[c]] * A[3 * J[c]] + AS[3 * I[c] + 1] * A[3 * J[c] + 1] + AS[3 * I[c] + 2] * A[3 * J[c] + 2];
}
// out = A^T S A (S full symmetric), packed
template <typename T>
__device__ __forceinline__ void congruence_t(const T* A, const T* S, T* out) {
  T At[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) At[3 * i + j] = A[3 * j + i];
  congruence(At, S, out);
}
// Full contraction a : b of two packed symmetric tensors.
template <typename T>
__device__ __forceinline__ T sym_dot(const T* a, const T* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + T(2) * (a[3] * b[3] + a[4] * b[4] + a[5] * b[5]);
}

// With FP32 tangent records the kernel is occupancy-bound: capping registers
// for 11 resident one-warp blocks per SM (a little spilling to L1) measured
// 14 % faster at 64^3 than the unconstrained 222 registers (9 blocks); the
// FP64 variants lose from the same cap and keep the compiler's choice.
// The kinematic variant carries more live state and keeps the compiler's choice.
template <typename KT, bool COMMIT, bool FBAR, int HARD>
__global__ void __launch_bounds__(32 * WPB, (std::is_same<KT, float>::value && !COMMIT && HARD != HARD_KIN) ? 11 : 1)
element_color_kernel(ElemArgs<KT> p, const int* __restrict__ elist, int nlist) {
  using TT = KT;  // type of the tangent records and of the phase-B arithmetic
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane >> 3, g = lane & 7;
  const long long li = ((long long)blockIdx.x * WPB + warp) * EPW + slot;
  const bool valid = li < nlist;
  // Lanes of a slot past the end of the list evaluate a duplicate of the
  // first element (so every lane takes part in the warp shuffles) and write
  // nothing to global memory.
  const int e = elist[valid ? li : 0];
  TT* const wbase = reinterpret_cast<TT*>(smem_raw) + warp * EPW * SLOT_TT;
  TT* const S = wbase + slot * SLOT_TT;
  TT* const g0s = S;                      // [a*3+k]
  TT* const Rg = S + 24 + g * GPREC;      // this lane's Gauss-point record
  double* const XU = COMMIT ? reinterpret_cast<double*>(smem_raw) + (warp * EPW + slot) * 48
                            : reinterpret_cast<double*>(S + 24);
  double* const Xe = XU;                  // [a*3+d]
  double* const ue = XU + 24;             // [a*3+d]

  __shared__ int nodes_s[WPB][EPW][8];
  {
    const int nd = p.elem[(long long)e * 8 + g];
    nodes_s[warp][slot][g] = nd;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Xe[g * 3 + d] = p.X[(long long)nd * 3 + d];
      ue[g * 3 + d] = p.U[(long long)nd * 3 + d];
    }
  }
  __syncwarp();

  const MatParams m = p.mat;
  const long long gp = (long long)e * 8 + g;
  const double gc = 0.57735026918962576451;  // 1/sqrt(3)
  const double xg = nsgn_x(g) * gc, yg = nsgn_y(g) * gc, zg = nsgn_z(g) * gc;
  // ---- F-bar centroid quantities (Elements.jl:418-424) ----
  double J0 = 1.0;
  if (FBAR) {
    double J0m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, UC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      double dc[3];
      dshape_a(a, 0.0, 0.0, 0.0, dc);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          J0m[3 * i + j] += Xe[a * 3 + i] * dc[j];
          UC[3 * i + j] += ue[a * 3 + i] * dc[j];
        }
    }
    double J0i[9], F0[9], F0i[9];
    inv3(J0m, J0i);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) s += UC[3 * i + q] * J0i[3 * q + j];
        F0[3 * i + j] = s;
      }
    J0 = det3(F0);
    if (!COMMIT && g == 0) {
      // g0_(a,k) = sum_m dN_a/dxi_m(0) H0[m][k], H0 = J0mat^-1 F0^-1
      inv3(F0, F0i);
      double H0[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double s = 0.0;
#pragma unroll
          for (int q = 0; q < 3; ++q) s += J0i[3 * i + q] * F0i[3 * q + j];
          H0[3 * i + j] = s;
        }
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        double dc[3];
        dshape_a(a, 0.0, 0.0, 0.0, dc);
#pragma unroll
        for (int k = 0; k < 3; ++k) g0s[a * 3 + k] = (TT)(dc[0] * H0[k] + dc[1] * H0[3 + k] + dc[2] * H0[6 + k]);
      }
    }
  }
  // ---- Gauss-point geometry: J = Xe' dN (Elements.jl:89,155-161) ----
  double Jm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Ug[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double d[3];
    dshape_a(a, xg, yg, zg, d);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Jm[3 * i + j] += Xe[a * 3 + i] * d[j];
        Ug[3 * i + j] += ue[a * 3 + i] * d[j];
      }
  }
  // The nodal coordinates are dead from here on; the records may overwrite them.
  __syncwarp();
  const double w = det3(Jm);  // detJ * weight (weights are 1, Elements.jl:43)
  double Ji[9];
  inv3(Jm, Ji);
  // F = I + sum_a u_a (x) dN_a/dX  (FiniteStrain.jl:107-119)
  double F[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
      for (int q = 0; q < 3; ++q) s += Ug[3 * i + q] * Ji[3 * q + j];
      F[3 * i + j] = s;
    }
  const double Jg = det3(F);
  const double scale = FBAR ? cbrt(J0 / Jg) : 1.0;  // Elements.jl:437
  double Fb[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) Fb[i] = scale * F[i];
  // ---- finite_kinematics (FiniteStrain.jl:148-170) ----
  const double Jb = det3(Fb);
  double c6[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) c6[c] = p.cpi[(long long)c * p.ngp + gp];
  const double Cp[9] = {c6[0], c6[3], c6[5], c6[3], c6[1], c6[4], c6[5], c6[4], c6[2]};
  double M[9];  // Cp Fb^T
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) M[3 * i + j] = Cp[3 * i] * Fb[3 * j] + Cp[3 * i + 1] * Fb[3 * j + 1] + Cp[3 * i + 2] * Fb[3 * j + 2];
  double be[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) be[3 * i + j] = Fb[3 * i] * M[j] + Fb[3 * i + 1] * M[3 + j] + Fb[3 * i + 2] * M[6 + j];
  be[1] = be[3] = 0.5 * (be[1] + be[3]);
  be[2] = be[6] = 0.5 * (be[2] + be[6]);
  be[5] = be[7] = 0.5 * (be[5] + be[7]);
  double bv[3], Q[9];
  const bool ok = Jb > 0.0;
  if (!ok) {
    if (valid && atomicCAS(&p.status->code, 0, 1) == 0) {
      p.status->e = (long long)e + 1;
      p.status->g = g + 1;
      p.status->J = Jb;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) Q[i] = (i % 4 == 0) ? 1.0 : 0.0;
    bv[0] = bv[1] = bv[2] = 1.0;
  } else {
    eig3_jacobi(be, bv, Q);
  }
  // ---- return_map on principal values (Materials.jl:159-250) ----
  const double G = m.G, lam = m.lam, H = m.Hiso;
  const double sy0 = p.sigy0_e ? p.sigy0_e[e] : m.sigy0;
  const double an = p.alpha[gp];
  const double e0 = 0.5 * log(bv[0]), e1 = 0.5 * log(bv[1]), e2 = 0.5 * log(bv[2]);
  const double tre = e0 + e1 + e2;
  const double t0 = lam * tre + 2.0 * G * e0, t1 = lam * tre + 2.0 * G * e1, t2 = lam * tre + 2.0 * G * e2;
  const double pm = (t0 + t1 + t2) / 3.0;
  const double s0 = t0 - pm, s1 = t1 - pm, s2 = t2 - pm;
  const double s32 = 1.22474487139158904910;  // sqrt(1.5)
  // Kinematic hardening (finite_stress_update, FiniteStrain.jl:316-324): the
  // back stress is stored in the reference configuration and pushed forward
  // with the polar rotation of Fbar = R U (polar_RU, :194-210).  Everything
  // below runs in b^e's eigenbasis Q: beta' = (Q^T R) beta_ref (Q^T R)^T, and
  // the shifted stress xi' = diag(s) - beta' is no longer diagonal there, so
  // the flow direction nh' is a full symmetric tensor.
  double Rp[9], Vu[9], mu[3], QR[9], Bp[6], xi6[6], nh6[6];
  double nrm;
  if constexpr (HARD == HARD_KIN) {
    double Cm[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Cm[3 * i + j] = Fb[i] * Fb[j] + Fb[3 + i] * Fb[3 + j] + Fb[6 + i] * Fb[6 + j];
    double lc[3];
    eig3_jacobi(Cm, lc, Vu);
    double imu[3];
#pragma unroll
    for (int A = 0; A < 3; ++A) {
      mu[A] = sqrt(fmax(lc[A], 0.0));
      imu[A] = mu[A] > 0.0 ? 1.0 / mu[A] : 0.0;
    }
    double Ui[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Ui[3 * i + j] = Vu[3 * i] * imu[0] * Vu[3 * j] + Vu[3 * i + 1] * imu[1] * Vu[3 * j + 1] + Vu[3 * i + 2] * imu[2] * Vu[3 * j + 2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Rp[3 * i + j] = Fb[3 * i] * Ui[j] + Fb[3 * i + 1] * Ui[3 + j] + Fb[3 * i + 2] * Ui[6 + j];
#pragma unroll
    for (int A = 0; A < 3; ++A)
#pragma unroll
      for (int k = 0; k < 3; ++k) QR[3 * A + k] = Q[A] * Rp[k] + Q[3 + A] * Rp[3 + k] + Q[6 + A] * Rp[6 + k];
    double b6[6], Bf[9];
#pragma unroll
    for (int c = 0; c < 6; ++c) b6[c] = p.beta[(long long)c * p.ngp + gp];
    unpack_sym(b6, Bf);
    congruence(QR, Bf, Bp);
    xi6[0] = s0 - Bp[0]; xi6[1] = s1 - Bp[1]; xi6[2] = s2 - Bp[2];
    xi6[3] = -Bp[3]; xi6[4] = -Bp[4]; xi6[5] = -Bp[5];
    nrm = sqrt(sym_dot(xi6, xi6));
  } else {
    nrm = sqrt(s0 * s0 + s1 * s1 + s2 * s2);
  }
  const double qtr = s32 * nrm;
  const double ftr = (HARD == HARD_VOCE) ? qtr - voce_ys(m, sy0, an) : qtr - (sy0 + H * an);
  const bool plastic = ftr > 0.0;
  double n0 = 0.0, n1 = 0.0, n2 = 0.0, dg = 0.0, b0 = 0.0, g0c = 0.0;
  double ta0 = t0, ta1 = t1, ta2 = t2;
  if (plastic) {
    if constexpr (HARD == HARD_KIN) {
#pragma unroll
      for (int c = 0; c < 6; ++c) nh6[c] = xi6[c] / nrm;
      dg = ftr / (3.0 * G + H + m.Hkin);
      g0c = 2.0 * G / (3.0 * G + m.Hkin + H);
    } else {
      n0 = s0 / nrm; n1 = s1 / nrm; n2 = s2 / nrm;
      if constexpr (HARD == HARD_VOCE) {
        double Hp;
        dg = voce_dgamma(m, sy0, qtr, an, ftr, &Hp);
        g0c = 2.0 * G / (3.0 * G + Hp);
      } else {
        dg = ftr / (3.0 * G + H);
        g0c = 2.0 * G / (3.0 * G + H);
      }
      const double c = 2.0 * G * dg * s32;
      ta0 = t0 - c * n0; ta1 = t1 - c * n1; ta2 = t2 - c * n2;
    }
    b0 = 2.0 * G * dg / qtr;
  } else if constexpr (HARD == HARD_KIN) {
#pragma unroll
    for (int c = 0; c < 6; ++c) nh6[c] = 0.0;
  }
  // tau = Q tau' Q^T  (Kirchhoff, physical-shear Voigt); tau' is diagonal
  // unless kinematic hardening tilts the flow direction.
  double tau[9];
  if constexpr (HARD == HARD_KIN) {
    const double c = 2.0 * G * dg * s32;
    const double tp[6] = {t0 - c * nh6[0], t1 - c * nh6[1], t2 - c * nh6[2], -c * nh6[3], -c * nh6[4], -c * nh6[5]};
    double Tf[9], t6[6];
    unpack_sym(tp, Tf);
    congruence(Q, Tf, t6);
    unpack_sym(t6, tau);
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i; j < 3; ++j) {
        const double v = Q[3 * i] * ta0 * Q[3 * j] + Q[3 * i + 1] * ta1 * Q[3 * j + 1] + Q[3 * i + 2] * ta2 * Q[3 * j + 2];
        tau[3 * i + j] = v;
        tau[3 * j + i] = v;
      }
  }
  if (valid) {
    p.tau[0 * p.ngp + gp] = tau[0];
    p.tau[1 * p.ngp + gp] = tau[4];
    p.tau[2 * p.ngp + gp] = tau[8];
    p.tau[3 * p.ngp + gp] = tau[1];
    p.tau[4 * p.ngp + gp] = tau[5];
    p.tau[5 * p.ngp + gp] = tau[2];
    p.flags[gp] = plastic ? 1 : 0;
  }
  double Fbi[9];
  inv3(Fb, Fbi);
  if constexpr (COMMIT && HARD == HARD_KIN) {
    if (!valid) return;
    const double c = dg * s32;
    // back stress: beta_sp' + (2/3) Hkin dgamma sqrt(3/2) nh', pulled back to the
    // reference configuration, beta_ref = R^T beta_sp R (FiniteStrain.jl:324)
    double bn[6], Bf[9], b6n[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) bn[k] = Bp[k] + (2.0 / 3.0) * m.Hkin * c * nh6[k];
    unpack_sym(bn, Bf);
    congruence_t(QR, Bf, b6n);
#pragma unroll
    for (int k = 0; k < 6; ++k) p.beta[(long long)k * p.ngp + gp] = b6n[k];
    // exponential map with a flow direction that is not coaxial with b^e:
    // b^e_{n+1} = exp(2 eps^e'), eps^e' = diag(e) - dgamma sqrt(3/2) nh'
    // (FiniteStrain.jl:331-343), Cp^-1 = Fbar^-1 Q b^e' Q^T Fbar^-T.
    const double ee[6] = {2.0 * (e0 - c * nh6[0]), 2.0 * (e1 - c * nh6[1]), 2.0 * (e2 - c * nh6[2]),
                          -2.0 * c * nh6[3], -2.0 * c * nh6[4], -2.0 * c * nh6[5]};
    double E2[9], w2[3], V2[9];
    unpack_sym(ee, E2);
    eig3_jacobi(E2, w2, V2);
    double FQ[9], T[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int A = 0; A < 3; ++A) FQ[3 * i + A] = Fbi[3 * i] * Q[A] + Fbi[3 * i + 1] * Q[3 + A] + Fbi[3 * i + 2] * Q[6 + A];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int A = 0; A < 3; ++A) T[3 * i + A] = FQ[3 * i] * V2[A] + FQ[3 * i + 1] * V2[3 + A] + FQ[3 * i + 2] * V2[6 + A];
    const double l0 = exp(w2[0]), l1 = exp(w2[1]), l2 = exp(w2[2]);
    constexpr int I6[6] = {0, 1, 2, 0, 1, 0}, J6[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const int i = I6[k], j = J6[k];
      p.cpi[(long long)k * p.ngp + gp] = T[3 * i] * l0 * T[3 * j] + T[3 * i + 1] * l1 * T[3 * j + 1] + T[3 * i + 2] * l2 * T[3 * j + 2];
    }
    p.alpha[gp] = an + dg;
    // accumulated plastic strain Q (c nh') Q^T (diagnostic; engineering-shear Voigt)
    double cn6[6], Nf[9], d6[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) cn6[k] = c * nh6[k];
    unpack_sym(cn6, Nf);
    congruence(Q, Nf, d6);
#pragma unroll
    for (int k = 0; k < 6; ++k) p.epsp[(long long)k * p.ngp + gp] += (k < 3 ? 1.0 : 2.0) * d6[k];
  } else if constexpr (COMMIT) {
    if (!valid) return;
    // exponential-map update b^e_{n+1} = exp(2 eps^e), Cp^-1 = F^-1 b^e F^-T
    // (FiniteStrain.jl:331-343); eps^e shares the trial eigenbasis.
    const double c = dg * s32;
    const double l0 = exp(2.0 * (e0 - c * n0)), l1 = exp(2.0 * (e1 - c * n1)), l2 = exp(2.0 * (e2 - c * n2));
    double T[9];  // Fbi Q
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int A = 0; A < 3; ++A) T[3 * i + A] = Fbi[3 * i] * Q[A] + Fbi[3 * i + 1] * Q[3 + A] + Fbi[3 * i + 2] * Q[6 + A];
    double cn[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i; j < 3; ++j) {
        const double v = T[3 * i] * l0 * T[3 * j] + T[3 * i + 1] * l1 * T[3 * j + 1] + T[3 * i + 2] * l2 * T[3 * j + 2];
        cn[3 * i + j] = v;
        cn[3 * j + i] = v;
      }
    p.cpi[0 * p.ngp + gp] = cn[0];
    p.cpi[1 * p.ngp + gp] = cn[4];
    p.cpi[2 * p.ngp + gp] = cn[8];
    p.cpi[3 * p.ngp + gp] = cn[1];
    p.cpi[4 * p.ngp + gp] = cn[5];
    p.cpi[5 * p.ngp + gp] = cn[2];
    p.alpha[gp] = an + dg;
    // accumulated plastic strain (diagnostic; engineering-shear Voigt)
    double nn_[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        nn_[3 * i + j] = c * (Q[3 * i] * n0 * Q[3 * j] + Q[3 * i + 1] * n1 * Q[3 * j + 1] + Q[3 * i + 2] * n2 * Q[3 * j + 2]);
    p.epsp[0 * p.ngp + gp] += nn_[0];
    p.epsp[1 * p.ngp + gp] += nn_[4];
    p.epsp[2 * p.ngp + gp] += nn_[8];
    p.epsp[3 * p.ngp + gp] += 2.0 * nn_[1];
    p.epsp[4 * p.ngp + gp] += 2.0 * nn_[5];
    p.epsp[5 * p.ngp + gp] += 2.0 * nn_[2];
  } else {
    // ---- P = tau Fb^-T (FiniteStrain.jl:560-561) ----
    double P[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) P[3 * i + j] = tau[3 * i] * Fbi[3 * j] + tau[3 * i + 1] * Fbi[3 * j + 1] + tau[3 * i + 2] * Fbi[3 * j + 2];
    // ---- internal force, node by node: dN_a/dX = dN_a/dxi J^-1, then
    // Fe_a = sum over the element's 8 Gauss-point lanes of w P dN_a/dX (FP64);
    // lane g keeps node a = g and adds it into R (colored: no atomics).
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      double d[3];
      dshape_a(a, xg, yg, zg, d);
      const double x0 = d[0] * Ji[0] + d[1] * Ji[3] + d[2] * Ji[6];
      const double x1 = d[0] * Ji[1] + d[1] * Ji[4] + d[2] * Ji[7];
      const double x2 = d[0] * Ji[2] + d[1] * Ji[5] + d[2] * Ji[8];
      Rg[a * 3 + 0] = (TT)x0;
      Rg[a * 3 + 1] = (TT)x1;
      Rg[a * 3 + 2] = (TT)x2;
      double v0 = w * (P[0] * x0 + P[1] * x1 + P[2] * x2);
      double v1 = w * (P[3] * x0 + P[4] * x1 + P[5] * x2);
      double v2 = w * (P[6] * x0 + P[7] * x1 + P[8] * x2);
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        v2 += __shfl_xor_sync(0xffffffffu, v2, o);
      }
      if (a == g) { f0 = v0; f1 = v1; f2 = v2; }
    }
    if (valid) {
      if (p.Fbuf) {
        double* fb = p.Fbuf + (long long)e * 24 + g * 3;
        fb[0] = f0; fb[1] = f1; fb[2] = f2;
      } else {
        const int nd = nodes_s[warp][slot][g];
        p.R[(long long)nd * 3 + 0] += f0;
        p.R[(long long)nd * 3 + 1] += f1;
        p.R[(long long)nd * 3 + 2] += f2;
      }
    }
    // ---- A = dP/dFbar in the eigenbasis of b^e (dPdF, FiniteStrain.jl:503-547) ----
    // gamma_AB of _dhalflog_contract (FiniteStrain.jl:463-482)
    const double lyv[3] = {e0, e1, e2};
    TT gam[9];
#pragma unroll
    for (int A = 0; A < 3; ++A)
#pragma unroll
      for (int B = 0; B < 3; ++B) {
        double v;
        if (A == B) v = 1.0 / (2.0 * bv[A]);
        else if (fabs(bv[A] - bv[B]) < 1e-9 * (fabs(bv[A]) + fabs(bv[B]) + 1.0)) v = 1.0 / (bv[A] + bv[B]);
        else v = (lyv[A] - lyv[B]) / (bv[A] - bv[B]);
        gam[3 * A + B] = (TT)v;
      }
    TT Qt[9], MQ[9], NN[9], FbiT[9], Pt[9], Ft[9];  // MQ = (Cp Fb^T) Q, NN = Q^T Fb^-T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        FbiT[3 * i + j] = (TT)Fbi[3 * j + i];
        Qt[3 * i + j] = (TT)Q[3 * i + j];
        Pt[3 * i + j] = (TT)P[3 * i + j];
        Ft[3 * i + j] = (TT)F[3 * i + j];
      }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int B = 0; B < 3; ++B) {
        MQ[3 * i + B] = (TT)(M[3 * i] * Q[B] + M[3 * i + 1] * Q[3 + B] + M[3 * i + 2] * Q[6 + B]);
        NN[3 * i + B] = (TT)(Q[i] * Fbi[3 * B] + Q[3 + i] * Fbi[3 * B + 1] + Q[6 + i] * Fbi[3 * B + 2]);
      }
    // tangent modulus D in principal form:
    //   dtau' = c2 Y + c1 tr(Y) I + c3 (n . diag Y) diag(n)
    const TT c2 = (TT)(2.0 * G - 3.0 * G * b0);
    const TT c1 = (TT)(lam + G * b0);
    const TT c3 = (TT)(3.0 * G * (b0 - g0c));
    const TT nv[3] = {(TT)n0, (TT)n1, (TT)n2};
    // Kinematic hardening: the flow direction nh' (full in the eigenbasis) and
    // the back-stress rotation coupling dtau/dbeta_sp . dbeta_sp/dFbar of dPdF
    // (FiniteStrain.jl:532-536) with dtau/dbeta = a I + kd xi (x) xi
    // (dtau_dbeta, :250-268; zero in the elastic branch).  Per column the polar
    // spin follows from Omega U + U Omega = R^T dF - dF^T R in U's eigenbasis V
    // (dR_polar, :220-233): dbeta' = W' beta' + (W' beta')^T, W' = M Ob M^T,
    // M = Q^T R V.
    TT nhk[6], xik[6], Bk[9], M3[9], RV[9], Vk[9], muk[3], ask = TT(0), kdk = TT(0);
    if constexpr (HARD == HARD_KIN) {
      double Bf[9];
      unpack_sym(Bp, Bf);
#pragma unroll
      for (int k = 0; k < 6; ++k) { nhk[k] = (TT)nh6[k]; xik[k] = (TT)xi6[k]; }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          Bk[3 * i + j] = (TT)Bf[3 * i + j];
          Vk[3 * i + j] = (TT)Vu[3 * i + j];
          M3[3 * i + j] = (TT)(QR[3 * i] * Vu[j] + QR[3 * i + 1] * Vu[3 + j] + QR[3 * i + 2] * Vu[6 + j]);
          RV[3 * i + j] = (TT)(Rp[3 * i] * Vu[j] + Rp[3 * i + 1] * Vu[3 + j] + Rp[3 * i + 2] * Vu[6 + j]);
        }
#pragma unroll
      for (int A = 0; A < 3; ++A) muk[A] = (TT)mu[A];
      if (plastic) {
        const double Yy = sy0 + H * an;
        ask = (TT)(2.0 * G * s32 * dg / nrm);
        kdk = (TT)(2.0 * G * s32 / (3.0 * G + H + m.Hkin) * (Yy / (nrm * nrm)) / nrm);
      }
    }
    const TT ws_ = (TT)(w * scale);
    TT* const As = Rg + 24;  // [(j*3+i)*9 + (q*3+p)]
    TT uacc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int col = 0; col < 9; ++col) {
      const int pp = col % 3, qq = col / 3;
      TT Y[9];
#pragma unroll
      for (int A = 0; A < 3; ++A)
#pragma unroll
        for (int B = A; B < 3; ++B) {
          const TT h = Qt[3 * pp + A] * MQ[3 * qq + B] + MQ[3 * qq + A] * Qt[3 * pp + B];
          const TT v = gam[3 * A + B] * h;
          Y[3 * A + B] = v;
          Y[3 * B + A] = v;
        }
      const TT trY = Y[0] + Y[4] + Y[8];
      TT dt[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) dt[i] = c2 * Y[i];
      if constexpr (HARD == HARD_KIN) {
        const TT Ys[6] = {Y[0], Y[4], Y[8], Y[1], Y[5], Y[2]};
        const TT nd = sym_dot(nhk, Ys);
        TT add[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) add[k] = c3 * nd * nhk[k];
        add[0] += c1 * trY; add[1] += c1 * trY; add[2] += c1 * trY;
        if (ask != TT(0)) {
          const TT* av = RV + 3 * pp;  // row pp of R V
          const TT* cv = Vk + 3 * qq;  // row qq of V
          const TT w01 = (av[0] * cv[1] - cv[0] * av[1]) / (muk[0] + muk[1]);
          const TT w02 = (av[0] * cv[2] - cv[0] * av[2]) / (muk[0] + muk[2]);
          const TT w12 = (av[1] * cv[2] - cv[1] * av[2]) / (muk[1] + muk[2]);
          const TT Ob[9] = {TT(0), w01, w02, -w01, TT(0), w12, -w02, -w12, TT(0)};
          TT MO[9], Wp[9], X[9];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) MO[3 * i + j] = M3[3 * i] * Ob[j] + M3[3 * i + 1] * Ob[3 + j] + M3[3 * i + 2] * Ob[6 + j];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Wp[3 * i + j] = MO[3 * i] * M3[3 * j] + MO[3 * i + 1] * M3[3 * j + 1] + MO[3 * i + 2] * M3[3 * j + 2];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) X[3 * i + j] = Wp[3 * i] * Bk[j] + Wp[3 * i + 1] * Bk[3 + j] + Wp[3 * i + 2] * Bk[6 + j];
          const TT db[6] = {TT(2) * X[0], TT(2) * X[4], TT(2) * X[8], X[1] + X[3], X[5] + X[7], X[2] + X[6]};
          const TT xd = kdk * sym_dot(xik, db);
#pragma unroll
          for (int k = 0; k < 6; ++k) add[k] += ask * db[k] + xd * xik[k];
        }
        dt[0] += add[0]; dt[4] += add[1]; dt[8] += add[2];
        dt[1] += add[3]; dt[3] += add[3];
        dt[5] += add[4]; dt[7] += add[4];
        dt[2] += add[5]; dt[6] += add[5];
      } else {
        const TT nd = nv[0] * Y[0] + nv[1] * Y[4] + nv[2] * Y[8];
        dt[0] += c1 * trY + c3 * nd * nv[0];
        dt[4] += c1 * trY + c3 * nd * nv[1];
        dt[8] += c1 * trY + c3 * nd * nv[2];
      }
      TT T[9];  // dt' N
#pragma unroll
      for (int A = 0; A < 3; ++A)
#pragma unroll
        for (int j = 0; j < 3; ++j) T[3 * A + j] = dt[3 * A] * NN[j] + dt[3 * A + 1] * NN[3 + j] + dt[3 * A + 2] * NN[6 + j];
      const TT Fq = Ft[3 * pp + qq];  // standard F for the F-bar vec(F)
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const TT dP = Qt[3 * i] * T[j] + Qt[3 * i + 1] * T[3 + j] + Qt[3 * i + 2] * T[6 + j] - Pt[3 * i + qq] * FbiT[3 * pp + j];
          As[(j * 3 + i) * 9 + col] = ws_ * dP;
          uacc[j * 3 + i] += dP * Fq;
        }
    }
    const TT uf = (TT)(w * scale / 3.0);
#pragma unroll
    for (int r = 0; r < 9; ++r) Rg[105 + r] = FBAR ? uf * uacc[r] : TT(0);
    // F^-1 of the standard F = scale * Fb^-1 (for gJ = G^T vec(F^-T))
#pragma unroll
    for (int i = 0; i < 9; ++i) Rg[114 + i] = (TT)(scale * Fbi[i]);
    __syncwarp();

  // ---- Phase B: the warp's 4 x 24 Ke columns over 32 lanes, scatter into
  // the block-CSR tangent ----
#pragma unroll 1
  for (int t = lane; t < EPW * 24; t += 32) {
    const int s = t / 24, col = t - 24 * s;
    const long long ls = ((long long)blockIdx.x * WPB + warp) * EPW + s;
    if (ls >= nlist) continue;
    const int es = elist[ls];
    const TT* Ss = wbase + s * SLOT_TT;
    const int b = col / 3, k = col - 3 * b;
    TT acc[24];
#pragma unroll
    for (int r = 0; r < 24; ++r) acc[r] = TT(0);
    const TT g0bk = FBAR ? Ss[col] : TT(0);
#pragma unroll 1
    for (int gg = 0; gg < 8; ++gg) {
      const TT* Rr = Ss + 24 + gg * GPREC;
      const TT* dX = Rr;
      const TT* A = Rr + 24;
      const TT* u = Rr + 105;
      const TT* Fi = Rr + 114;
      const TT db0 = dX[b * 3], db1 = dX[b * 3 + 1], db2 = dX[b * 3 + 2];
      // dg_(b,k) = g0_(b,k) - gJ_(b,k),  gJ_(b,k) = sum_j F^-1[j][k] dNdX[b][j]
      const TT dgbk = FBAR ? (g0bk - (Fi[k] * db0 + Fi[3 + k] * db1 + Fi[6 + k] * db2)) : TT(0);
      TT T[9];
#pragma unroll
      for (int r = 0; r < 9; ++r)
        T[r] = A[r * 9 + k] * db0 + A[r * 9 + 3 + k] * db1 + A[r * 9 + 6 + k] * db2 + u[r] * dgbk;
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const TT x0 = dX[a * 3], x1 = dX[a * 3 + 1], x2 = dX[a * 3 + 2];
#pragma unroll
        for (int i = 0; i < 3; ++i) acc[a * 3 + i] += x0 * T[i] + x1 * T[3 + i] + x2 * T[6 + i];
      }
    }
    if (p.Kbuf) {
      // element-ordered: column (b,k) of rows (a,i) at [es][a][i][col]; the 24
      // lanes of an element write 24 consecutive values per (a,i)
      KT* kb = p.Kbuf + (long long)es * 576 + col;
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i) __stcs(kb + a * 72 + i * 24, (KT)acc[a * 3 + i]);
      continue;
    }
    // The eight target blocks lie in eight different block rows, so nothing
    // aliases: all 24 loads are issued before any store (one memory latency
    // per column instead of a chain of eight).
    const int* nds = nodes_s[warp][s];
    KT* vp[8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
      vp[a] = p.Kval + ((long long)p.browptr[nds[a]] + p.rank[(long long)es * 64 + a * 8 + b]) * 9 + k;
    KT old[24];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      old[a * 3 + 0] = vp[a][0];
      old[a * 3 + 1] = vp[a][3];
      old[a * 3 + 2] = vp[a][6];
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      vp[a][0] = old[a * 3 + 0] + (KT)acc[a * 3 + 0];
      vp[a][3] = old[a * 3 + 1] + (KT)acc[a * 3 + 1];
      vp[a][6] = old[a * 3 + 2] + (KT)acc[a * 3 + 2];
    }
  }
  }  // !COMMIT
}

template <typename KT, bool COMMIT, bool FBAR, int HARD>
static void launch_t(const ElemArgs<KT>& a, const int* elist, int n, cudaStream_t st) {
  if (n <= 0) return;
  const int warps = (n + EPW - 1) / EPW;
  const int blocks = (warps + WPB - 1) / WPB;
  const size_t sm = (size_t)WPB * warp_smem_bytes<KT>(COMMIT);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(element_color_kernel<KT, COMMIT, FBAR, HARD>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  pfem::count_launch(); element_color_kernel<KT, COMMIT, FBAR, HARD><<<blocks, 32 * WPB, sm, st>>>(a, elist, n);
}

// ---------------------------------------------------------------- small strain
// The small-strain kind, element_force_tangent! (Elements.jl:323-360) with
// bmatrix (:97-117) and the Voigt return map (Materials.jl:159-250; linear or
// saturation isotropic hardening, or linear kinematic hardening with the back
// stress in p.beta, HARD).  Same warp
// organisation as the finite kernel: a lane evaluates one Gauss point
// (strain, return map, stress, consistent tangent D in FP64), the forces are
// shuffle-reduced node by node, the records (dN/dX, w D) go to shared memory in
// the tangent's type and the warp's 4 x 24 K_e columns are summed over the
// eight Gauss points by all 32 lanes and added into the tangent.  The state
// array epsp holds the committed plastic strain, tau receives sigma.
constexpr int SREC = 24 + 36;                 // dN/dX, w D (row-major 6 x 6)
constexpr int SSLOT = 8 * SREC;
template <typename TT>
constexpr int warp_smem_small(bool commit) {
  return commit ? EPW * 48 * 8 : EPW * SSLOT * (int)sizeof(TT);
}
static_assert(8 * SREC * 4 >= 48 * 8, "coordinate scratch must fit in the record area");

template <typename KT, bool COMMIT, int HARD>
__global__ void __launch_bounds__(32 * WPB)
element_small_kernel(ElemArgs<KT> p, const int* __restrict__ elist, int nlist) {
  using TT = KT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane >> 3, g = lane & 7;
  const long long li = ((long long)blockIdx.x * WPB + warp) * EPW + slot;
  const bool valid = li < nlist;
  const int e = elist[valid ? li : 0];
  TT* const wbase = reinterpret_cast<TT*>(smem_raw) + warp * EPW * SSLOT;
  TT* const S = wbase + slot * SSLOT;
  TT* const Rg = S + g * SREC;
  double* const XU = COMMIT ? reinterpret_cast<double*>(smem_raw) + (warp * EPW + slot) * 48
                            : reinterpret_cast<double*>(S);
  double* const Xe = XU;
  double* const ue = XU + 24;
  __shared__ int nodes_s[WPB][EPW][8];
  {
    const int nd = p.elem[(long long)e * 8 + g];
    nodes_s[warp][slot][g] = nd;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Xe[g * 3 + d] = p.X[(long long)nd * 3 + d];
      ue[g * 3 + d] = p.U[(long long)nd * 3 + d];
    }
  }
  __syncwarp();
  const MatParams m = p.mat;
  const long long gp = (long long)e * 8 + g;
  const double gc = 0.57735026918962576451;
  const double xg = nsgn_x(g) * gc, yg = nsgn_y(g) * gc, zg = nsgn_z(g) * gc;
  double Jm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double d[3];
    dshape_a(a, xg, yg, zg, d);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Jm[3 * i + j] += Xe[a * 3 + i] * d[j];
  }
  const double w = det3(Jm);
  double Ji[9];
  inv3(Jm, Ji);
  // strain eps = B u (engineering shear), bmatrix Elements.jl:97-117
  double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double d[3];
    dshape_a(a, xg, yg, zg, d);
    const double nx = d[0] * Ji[0] + d[1] * Ji[3] + d[2] * Ji[6];
    const double ny = d[0] * Ji[1] + d[1] * Ji[4] + d[2] * Ji[7];
    const double nz = d[0] * Ji[2] + d[1] * Ji[5] + d[2] * Ji[8];
    const double ux = ue[a * 3], uy = ue[a * 3 + 1], uz = ue[a * 3 + 2];
    eps[0] += nx * ux;
    eps[1] += ny * uy;
    eps[2] += nz * uz;
    eps[3] += ny * ux + nx * uy;
    eps[4] += nz * uy + ny * uz;
    eps[5] += nz * ux + nx * uz;
  }
  __syncwarp();  // the nodal coordinates are dead; the records may overwrite them
  // ---- return_map, Materials.jl:159-250 ----
  const double G = m.G, lam = m.lam, H = m.Hiso;
  const double sy0 = p.sigy0_e ? p.sigy0_e[e] : m.sigy0;
  const double an = p.alpha[gp];
  double de[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) de[c] = eps[c] - p.epsp[(long long)c * p.ngp + gp];
  const double tr = de[0] + de[1] + de[2];
  double st[6];
#pragma unroll
  for (int c = 0; c < 3; ++c) st[c] = lam * tr + 2.0 * G * de[c];
#pragma unroll
  for (int c = 3; c < 6; ++c) st[c] = G * de[c];
  const double pm = (st[0] + st[1] + st[2]) / 3.0;
  double xi[6], bn[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    bn[c] = (HARD == HARD_KIN) ? p.beta[(long long)c * p.ngp + gp] : 0.0;
    xi[c] = st[c] - (c < 3 ? pm : 0.0) - bn[c];
  }
  const double nrm = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2] +
                          2.0 * (xi[3] * xi[3] + xi[4] * xi[4] + xi[5] * xi[5]));
  const double s32 = 1.22474487139158904910;
  const double qtr = s32 * nrm;
  const double ftr = (HARD == HARD_VOCE) ? qtr - voce_ys(m, sy0, an) : qtr - (sy0 + H * an);
  const bool plastic = ftr > 0.0;
  double nh[6] = {0, 0, 0, 0, 0, 0}, sig[6], dg = 0.0, b0 = 0.0, g0c = 0.0;
  if (plastic) {
#pragma unroll
    for (int c = 0; c < 6; ++c) nh[c] = xi[c] / nrm;
    if constexpr (HARD == HARD_VOCE) {
      double Hp;
      dg = voce_dgamma(m, sy0, qtr, an, ftr, &Hp);
      g0c = 2.0 * G / (3.0 * G + Hp);
    } else if constexpr (HARD == HARD_KIN) {
      dg = ftr / (3.0 * G + H + m.Hkin);
      g0c = 2.0 * G / (3.0 * G + m.Hkin + H);
    } else {
      dg = ftr / (3.0 * G + H);
      g0c = 2.0 * G / (3.0 * G + H);
    }
    b0 = 2.0 * G * dg / qtr;
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) sig[c] = st[c] - (2.0 * G * dg * s32) * nh[c];
  if (valid) {
#pragma unroll
    for (int c = 0; c < 6; ++c) p.tau[(long long)c * p.ngp + gp] = sig[c];
    p.flags[gp] = plastic ? 1 : 0;
  }
  if constexpr (COMMIT) {
    if (!valid) return;
#pragma unroll
    for (int c = 0; c < 6; ++c)
      p.epsp[(long long)c * p.ngp + gp] += (dg * s32) * (c < 3 ? nh[c] : 2.0 * nh[c]);
    if constexpr (HARD == HARD_KIN) {
#pragma unroll
      for (int c = 0; c < 6; ++c) p.beta[(long long)c * p.ngp + gp] = bn[c] + (2.0 / 3.0) * m.Hkin * (dg * s32) * nh[c];
    }
    p.alpha[gp] = an + dg;
  } else {
    // ---- internal force, node by node (FP64), lane g keeps node g ----
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      double d[3];
      dshape_a(a, xg, yg, zg, d);
      const double nx = d[0] * Ji[0] + d[1] * Ji[3] + d[2] * Ji[6];
      const double ny = d[0] * Ji[1] + d[1] * Ji[4] + d[2] * Ji[7];
      const double nz = d[0] * Ji[2] + d[1] * Ji[5] + d[2] * Ji[8];
      Rg[a * 3 + 0] = (TT)nx;
      Rg[a * 3 + 1] = (TT)ny;
      Rg[a * 3 + 2] = (TT)nz;
      double v0 = w * (nx * sig[0] + ny * sig[3] + nz * sig[5]);
      double v1 = w * (ny * sig[1] + nx * sig[3] + nz * sig[4]);
      double v2 = w * (nz * sig[2] + ny * sig[4] + nx * sig[5]);
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        v2 += __shfl_xor_sync(0xffffffffu, v2, o);
      }
      if (a == g) { f0 = v0; f1 = v1; f2 = v2; }
    }
    if (valid) {
      if (p.Fbuf) {
        double* fb = p.Fbuf + (long long)e * 24 + g * 3;
        fb[0] = f0; fb[1] = f1; fb[2] = f2;
      } else {
        const int nd = nodes_s[warp][slot][g];
        p.R[(long long)nd * 3 + 0] += f0;
        p.R[(long long)nd * 3 + 1] += f1;
        p.R[(long long)nd * 3 + 2] += f2;
      }
    }
    // ---- w D: D = C - 3G b0 Idev + 3G (b0 - g0) n n^T (Materials.jl:245-247) ----
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const double c = (i < 3 && j < 3) ? (i == j ? lam + 2.0 * G : lam) : (i == j ? G : 0.0);
        const double isym = (i == j) ? (i < 3 ? 1.0 : 0.5) : 0.0;
        const double idev = isym - ((i < 3 && j < 3) ? 1.0 / 3.0 : 0.0);
        const double dv = c - (3.0 * G * b0) * idev + (3.0 * G * (b0 - g0c)) * nh[i] * nh[j];
        Rg[24 + i * 6 + j] = (TT)(w * dv);
      }
    __syncwarp();
    // ---- K_e columns over all 32 lanes, colored scatter ----
#pragma unroll 1
    for (int t = lane; t < EPW * 24; t += 32) {
      const int s2 = t / 24, col = t - 24 * s2;
      const long long ls = ((long long)blockIdx.x * WPB + warp) * EPW + s2;
      if (ls >= nlist) continue;
      const int es = elist[ls];
      const TT* Ss = wbase + s2 * SSLOT;
      const int b = col / 3, k = col - 3 * b;
      TT acc[24];
#pragma unroll
      for (int r = 0; r < 24; ++r) acc[r] = TT(0);
#pragma unroll 1
      for (int gg = 0; gg < 8; ++gg) {
        const TT* Rr = Ss + gg * SREC;
        const TT* dX = Rr;
        const TT* D = Rr + 24;
        const TT bx = dX[b * 3], by = dX[b * 3 + 1], bz = dX[b * 3 + 2];
        TT bc[6];  // column (b,k) of B
        bc[0] = k == 0 ? bx : TT(0);
        bc[1] = k == 1 ? by : TT(0);
        bc[2] = k == 2 ? bz : TT(0);
        bc[3] = k == 0 ? by : (k == 1 ? bx : TT(0));
        bc[4] = k == 1 ? bz : (k == 2 ? by : TT(0));
        bc[5] = k == 0 ? bz : (k == 2 ? bx : TT(0));
        TT T[6];
#pragma unroll
        for (int r = 0; r < 6; ++r) {
          TT v = TT(0);
#pragma unroll
          for (int q = 0; q < 6; ++q) v += D[r * 6 + q] * bc[q];
          T[r] = v;
        }
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          const TT x0 = dX[a * 3], x1 = dX[a * 3 + 1], x2 = dX[a * 3 + 2];
          acc[a * 3 + 0] += x0 * T[0] + x1 * T[3] + x2 * T[5];
          acc[a * 3 + 1] += x1 * T[1] + x0 * T[3] + x2 * T[4];
          acc[a * 3 + 2] += x2 * T[2] + x1 * T[4] + x0 * T[5];
        }
      }
      if (p.Kbuf) {
        KT* kb = p.Kbuf + (long long)es * 576 + col;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int i = 0; i < 3; ++i) __stcs(kb + a * 72 + i * 24, (KT)acc[a * 3 + i]);
        continue;
      }
      const int* nds = nodes_s[warp][s2];
      KT* vp[8];
#pragma unroll
      for (int a = 0; a < 8; ++a)
        vp[a] = p.Kval + ((long long)p.browptr[nds[a]] + p.rank[(long long)es * 64 + a * 8 + b]) * 9 + k;
      KT old[24];
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        old[a * 3 + 0] = vp[a][0];
        old[a * 3 + 1] = vp[a][3];
        old[a * 3 + 2] = vp[a][6];
      }
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        vp[a][0] = old[a * 3 + 0] + (KT)acc[a * 3 + 0];
        vp[a][3] = old[a * 3 + 1] + (KT)acc[a * 3 + 1];
        vp[a][6] = old[a * 3 + 2] + (KT)acc[a * 3 + 2];
      }
    }
  }
}

template <typename KT, bool COMMIT, int HARD>
static void launch_small_t(const ElemArgs<KT>& a, const int* elist, int n, cudaStream_t st) {
  if (n <= 0) return;
  const int warps = (n + EPW - 1) / EPW;
  const int blocks = (warps + WPB - 1) / WPB;
  const size_t sm = (size_t)WPB * warp_smem_small<KT>(COMMIT);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(element_small_kernel<KT, COMMIT, HARD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    attr = true;
  }
  pfem::count_launch();
  element_small_kernel<KT, COMMIT, HARD><<<blocks, 32 * WPB, sm, st>>>(a, elist, n);
}

template <typename KT, int HARD>
static void launch_small_h(const ElemArgs<KT>& a, const int* elist, int n, bool commit, cudaStream_t st) {
  if (commit) launch_small_t<KT, true, HARD>(a, elist, n, st);
  else launch_small_t<KT, false, HARD>(a, elist, n, st);
}

template <typename KT>
void launch_element_small(const ElemArgs<KT>& a, const int* elist, int n, bool commit, int hard, cudaStream_t st) {
  if (hard == HARD_KIN) launch_small_h<KT, HARD_KIN>(a, elist, n, commit, st);
  else if (hard == HARD_VOCE) launch_small_h<KT, HARD_VOCE>(a, elist, n, commit, st);
  else launch_small_h<KT, HARD_LINEAR>(a, elist, n, commit, st);
}
template void launch_element_small<double>(const ElemArgs<double>&, const int*, int, bool, int, cudaStream_t);
template void launch_element_small<float>(const ElemArgs<float>&, const int*, int, bool, int, cudaStream_t);

template <typename KT, int HARD>
static void launch_color_h(const ElemArgs<KT>& a, const int* elist, int n, bool commit, bool fbar, cudaStream_t st) {
  if (commit) {
    if (fbar) launch_t<KT, true, true, HARD>(a, elist, n, st);
    else launch_t<KT, true, false, HARD>(a, elist, n, st);
  } else {
    if (fbar) launch_t<KT, false, true, HARD>(a, elist, n, st);
    else launch_t<KT, false, false, HARD>(a, elist, n, st);
  }
}

template <typename KT>
void launch_element_color(const ElemArgs<KT>& a, const int* elist, int n, bool commit,
                          bool fbar, int hard, cudaStream_t st) {
  if (hard == HARD_KIN) launch_color_h<KT, HARD_KIN>(a, elist, n, commit, fbar, st);
  else if (hard == HARD_VOCE) launch_color_h<KT, HARD_VOCE>(a, elist, n, commit, fbar, st);
  else launch_color_h<KT, HARD_LINEAR>(a, elist, n, commit, fbar, st);
}

// ---------------------------------------------------------------- row gather
// One warp per node a: the row's blocks accumulate in shared memory, element by
// element in increasing element order (a fixed order: deterministic sums).
// Within one element the 72 values go to 72 distinct entries (eight distinct
// column nodes), so the lanes never add into the same entry at once.
template <typename KT>
__global__ void __launch_bounds__(256) gather_rows_kernel(int nn, const int* __restrict__ nptr,
                                                          const int* __restrict__ nel,
                                                          const uint8_t* __restrict__ nloc,
                                                          const int* __restrict__ browptr,
                                                          const uint8_t* __restrict__ rank,
                                                          const KT* __restrict__ Kbuf,
                                                          const double* __restrict__ Fbuf, KT* __restrict__ Kval,
                                                          double* __restrict__ R, int maxlen) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = (int)blockIdx.x * (int)(blockDim.x >> 5) + warp;
  if (a >= nn) return;  // whole warps; no block-wide barrier below
  KT* acc = reinterpret_cast<KT*>(gsm) + (size_t)warp * maxlen * 9;
  const int r0 = browptr[a], len9 = (browptr[a + 1] - r0) * 9;
  for (int v = lane; v < len9; v += 32) acc[v] = KT(0);
  double fr = 0.0;
  __syncwarp();
  const int q1 = nptr[a + 1];
  for (int q = nptr[a]; q < q1; ++q) {
    const int e = nel[q];
    const int al = nloc[q];
    const KT* src = Kbuf + (long long)e * 576 + al * 72;
    const uint8_t* rk = rank + (long long)e * 64 + al * 8;
    for (int v = lane; v < 72; v += 32) {
      const int i = v / 24, col = v - 24 * i, b = col / 3, k = col - 3 * b;
      acc[rk[b] * 9 + i * 3 + k] += __ldcs(src + v);
    }
    if (lane < 3) fr += Fbuf[(long long)e * 24 + al * 3 + lane];
    __syncwarp();
  }
  KT* dst = Kval + (long long)r0 * 9;
  for (int v = lane; v < len9; v += 32) dst[v] = acc[v];
  if (lane < 3) R[(long long)a * 3 + lane] = fr;
}

// Rows of at most 32 blocks (every hex mesh: 27): lane p of the node's warp owns
// block p of the row in registers.  The node's element ids, positions and rank
// bytes are loaded once, one element per lane; then, element by element in
// increasing order, the lane whose position appears among the element's eight
// rank bytes (at most one does, per column node b) adds that 3 x 3 block.  The
// value loads of different elements do not depend on each other, nothing goes
// through shared memory, and each lane sums in the same element order as the
// shared-memory gather above.
template <typename KT>
__global__ void __launch_bounds__(256) gather_rows_lane_kernel(int nn, const int* __restrict__ nptr,
                                                               const int* __restrict__ nel,
                                                               const uint8_t* __restrict__ nloc,
                                                               const int* __restrict__ browptr,
                                                               const uint8_t* __restrict__ rank,
                                                               const KT* __restrict__ Kbuf,
                                                               const double* __restrict__ Fbuf,
                                                               KT* __restrict__ Kval, double* __restrict__ R) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int a = (int)blockIdx.x * (int)(blockDim.x >> 5) + warp;
  if (a >= nn) return;  // whole warps
  const int r0 = browptr[a], len = browptr[a + 1] - r0;
  const int q0 = nptr[a], nq = nptr[a + 1] - q0;
  const unsigned key = (unsigned)lane * 0x01010101u;
  KT acc[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) acc[v] = KT(0);
  double fr = 0.0;
  for (int base = 0; base < nq; base += 32) {
    const int cnt = min(32, nq - base);
    int e_l = 0, al_l = 0;
    unsigned lo_l = 0xFFFFFFFFu, hi_l = 0xFFFFFFFFu;
    if (lane < cnt) {
      e_l = nel[q0 + base + lane];
      al_l = nloc[q0 + base + lane];
      const uint2 rk = *reinterpret_cast<const uint2*>(rank + (long long)e_l * 64 + al_l * 8);
      lo_l = rk.x;
      hi_l = rk.y;
    }
#pragma unroll 4
    for (int j = 0; j < cnt; ++j) {
      const int e = __shfl_sync(0xffffffffu, e_l, j), al = __shfl_sync(0xffffffffu, al_l, j);
      const unsigned lo = __shfl_sync(0xffffffffu, lo_l, j), hi = __shfl_sync(0xffffffffu, hi_l, j);
      const unsigned ml = __vcmpeq4(lo, key), mh = __vcmpeq4(hi, key);
      const int b = ml ? ((__ffs(ml) - 1) >> 3) : (mh ? 4 + ((__ffs(mh) - 1) >> 3) : -1);
      if (b >= 0) {
        const KT* src = Kbuf + (long long)e * 576 + al * 72 + b * 3;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int k = 0; k < 3; ++k) acc[i * 3 + k] += __ldcs(src + i * 24 + k);
      }
      if (lane < 3) fr += Fbuf[(long long)e * 24 + al * 3 + lane];
    }
  }
  if (lane < len) {
    KT* dst = Kval + (long long)(r0 + lane) * 9;
#pragma unroll
    for (int v = 0; v < 9; ++v) dst[v] = acc[v];
  }
  if (lane < 3) R[(long long)a * 3 + lane] = fr;
}

template <typename KT>
void launch_gather_rows(int nn, const int* nptr, const int* nel, const uint8_t* nloc, const int* browptr,
                        const uint8_t* rank, const KT* Kbuf, const double* Fbuf, KT* Kval, double* R, int maxlen,
                        cudaStream_t st) {
  constexpr int WARPS = 8;
  const size_t sm = (size_t)WARPS * maxlen * 9 * sizeof(KT);
  const int blocks = (nn + WARPS - 1) / WARPS;
  if (blocks <= 0) return;
  if (maxlen <= 32) {
    pfem::count_launch();
    gather_rows_lane_kernel<KT><<<blocks, 32 * WARPS, 0, st>>>(nn, nptr, nel, nloc, browptr, rank, Kbuf, Fbuf, Kval, R);
    return;
  }
  if (sm > 48 * 1024)  // rows longer than a hex mesh's 27 blocks (the 8-bit rank table caps them at 256)
    cudaFuncSetAttribute(gather_rows_kernel<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  pfem::count_launch();
  gather_rows_kernel<KT><<<blocks, 32 * WARPS, sm, st>>>(nn, nptr, nel, nloc, browptr, rank, Kbuf, Fbuf, Kval, R,
                                                        maxlen);
}
template void launch_gather_rows<double>(int, const int*, const int*, const uint8_t*, const int*, const uint8_t*,
                                         const double*, const double*, double*, double*, int, cudaStream_t);
template void launch_gather_rows<float>(int, const int*, const int*, const uint8_t*, const int*, const uint8_t*,
                                        const float*, const double*, float*, double*, int, cudaStream_t);

template void launch_element_color<double>(const ElemArgs<double>&, const int*, int, bool, bool, int, cudaStream_t);
template void launch_element_color<float>(const ElemArgs<float>&, const int*, int, bool, bool, int, cudaStream_t);

}  // namespace pfem
