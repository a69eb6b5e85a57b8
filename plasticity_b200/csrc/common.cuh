// common.cuh -- shared types and device helpers for the B200 F-bar J2 path.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#define PFEM_CUDA_OK(expr)                                                        \
  do {                                                                            \
    cudaError_t e__ = (expr);                                                     \
    if (e__ != cudaSuccess) {                                                     \
      pfem_set_cuda_error(e__, #expr, __FILE__, __LINE__);                        \
      return PFEM_ERR_CUDA;                                                       \
    }                                                                             \
  } while (0)

void pfem_set_cuda_error(cudaError_t e, const char* what, const char* file, int line);

namespace pfem {

// Process-wide count of kernel launches made by this library (every launch
// site calls count_launch() once), read through pfem_kernel_launches().
long long& launch_counter();
// Set the calling thread's error message returned by pfem_last_error(NULL).
void set_last_error(const std::string& msg);
inline void count_launch() { ++launch_counter(); }

// Material constants with the derived moduli of J2Material
// (lagrangian/src/Materials.jl:104-107).
struct MatParams {
  double E, nu, sigy0, Hiso, Hkin;
  double sigsat, delta;  // saturation hardening (Materials.jl:117-127); sat = sigsat - sigy0
  double G, K, lam, sat;
};

// Hardening law of the element kernels (a template argument, fixed per model):
// linear isotropic; saturation (Voce) isotropic, sigma_y(a) = sigy0 +
// (sigsat - sigy0)(1 - exp(-delta a)) + Hiso a; linear kinematic (+ linear
// isotropic), with the back stress as extra state.
enum : int { HARD_LINEAR = 0, HARD_VOCE = 1, HARD_KIN = 2 };

// Device status word.  code != 0 marks the first inverted Gauss point seen
// (ElementInversionError, lagrangian/src/FiniteStrain.jl:42-52).
struct DevStatus {
  int code;
  int g;         // 1-based Gauss point
  long long e;   // 1-based element
  double J;
};

// ---------------- 3x3 helpers (row-major a[3*i+j]) ----------------
__device__ __forceinline__ double det3(const double* a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}
__device__ __forceinline__ void inv3(const double* a, double* r) {
  const double d = det3(a);
  const double id = 1.0 / d;
  r[0] = (a[4] * a[8] - a[5] * a[7]) * id;
  r[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  r[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  r[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  r[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  r[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  r[6] = (a[3] * a[7] - a[4] * a[6]) * id;
  r[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  r[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

// Symmetric 3x3 eigendecomposition by cyclic Jacobi rotations (a is the
// symmetric input, row-major, destroyed).  On exit w holds the eigenvalues
// and V (row-major) the eigenvectors as columns.  At most `maxsweep` sweeps;
// each sweep skips rotations whose off-diagonal entry is already zero.
__device__ __forceinline__ void eig3_jacobi(double* a, double* w, double* V) {
#pragma unroll
  for (int i = 0; i < 9; ++i) V[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = fabs(a[1]) + fabs(a[2]) + fabs(a[5]);
    const double dia = fabs(a[0]) + fabs(a[4]) + fabs(a[8]);
    if (!(off > 1e-18 * dia) || off <= 1e-300) break;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int p = (r == 2) ? 1 : 0;
      const int q = (r == 0) ? 1 : 2;
      const int o = 3 - p - q;
      const double apq = a[3 * p + q];
      if (apq != 0.0) {
        const double theta = (a[3 * q + q] - a[3 * p + p]) / (2.0 * apq);
        double t;
        if (fabs(theta) > 1e150) t = 0.5 / theta;
        else t = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        a[3 * p + p] -= t * apq;
        a[3 * q + q] += t * apq;
        a[3 * p + q] = 0.0;
        a[3 * q + p] = 0.0;
        const double arp = a[3 * o + p], arq = a[3 * o + q];
        const double np_ = c * arp - s * arq, nq_ = s * arp + c * arq;
        a[3 * o + p] = np_; a[3 * p + o] = np_;
        a[3 * o + q] = nq_; a[3 * q + o] = nq_;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double vp = V[3 * k + p], vq = V[3 * k + q];
          V[3 * k + p] = c * vp - s * vq;
          V[3 * k + q] = s * vp + c * vq;
        }
      }
    }
  }
  w[0] = a[0]; w[1] = a[4]; w[2] = a[8];
}

}  // namespace pfem
