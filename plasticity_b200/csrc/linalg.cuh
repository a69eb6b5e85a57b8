// linalg.cuh -- declarations of the solver-side kernels (linalg.cu).
#pragma once
#include <algorithm>
#include "pfem_internal.h"

namespace pfem {

// Device copy of the frozen boundary conditions plus the precomputed list of
// tangent entries that Dirichlet imposition reads and overwrites.
struct BcDev {
  int nbc = 0;                 // constrained dofs (deduplicated)
  int* dofs = nullptr;         // 0-based dof
  double* vals = nullptr;
  uint8_t* ramp = nullptr;
  double* fn = nullptr;        // ndof nodal forces at lambda = 1
  int nrows = 0;               // free rows with entries in constrained columns
  int* rows = nullptr;
  int* rptr = nullptr;         // nrows+1
  long long* rpos = nullptr;   // scalar value index into the block-CSR value array
  int* rcol = nullptr;         // constrained column (dof)
  long long nzero = 0;         // entries in constrained rows or columns
  long long* zpos = nullptr;
  uint8_t* zone = nullptr;     // 1 on the diagonal of a constrained row
};

template <typename T> void bsr_spmv(const BsrMat<T>& A, const T* x, T* y, cudaStream_t st);
template <typename T> void bsr_residual(const BsrMat<T>& A, const T* x, const T* b, T* r, cudaStream_t st);
template <typename T> void bsr_cheb_step(const BsrMat<T>& A, const T* dinv, const T* d, T* r, T* x, cudaStream_t st);
// Degree-2 Chebyshev in one pass: x (=, or += unless zero) c2 d0 + c1 (r0 - Dinv A d0).
template <typename T> void bsr_cheb2(const BsrMat<T>& A, const T* dinv, const T* d0, const T* r0, T* x, bool zero,
                                     T c1, T c2, cudaStream_t st);
// r = Dinv (b - A x), d = scale r.
template <typename T> void bsr_residual_precond(const BsrMat<T>& A, const T* dinv, const T* x, const T* b, T* r,
                                                T* d, T scale, cudaStream_t st);
template <typename T> void blockdiag_apply(int nbrow, int bs, const T* dinv, const T* v, T* r, T scale, T* d, cudaStream_t st);
template <typename T> void blockdiag_invert(const BsrMat<T>& A, T* dinv, cudaStream_t st);
template <typename T> void dot(long long n, const T* a, const T* b, T* out, T* part, cudaStream_t st, bool take_sqrt);
template <typename T> void fill(long long n, T* x, T v, cudaStream_t st);
template <typename T> void axpby(long long n, T a, const T* x, T b, T* y, cudaStream_t st);
template <typename T> void cg_xr(long long n, const T* num, const T* den, const T* p, const T* q, T* x, T* r, cudaStream_t st);
template <typename T> void cg_p(long long n, const T* num, const T* den, const T* z, T* p, cudaStream_t st);
template <typename T> void bicg_p(long long n, const T* sc, const T* r, const T* v, T* p, cudaStream_t st);
template <typename T> void bicg_s(long long n, const T* sc, const T* r, const T* v, T* s, cudaStream_t st);
template <typename T> void bicg_xr(long long n, const T* sc, const T* ph, const T* sh, const T* s, const T* t, T* x, T* r, cudaStream_t st);
template <typename T> void scalar_copy(T* dst, const T* src, cudaStream_t st);
// PCG with the dot products' final sums fused into their consumers (deterministic):
// dot_partials writes the per-CTA partials of a.b and returns their count;
// cg_p_fused: rz = sum(part), p = z + (rz / sc[0]) p, sc[2] = rz;
// cg_xr_fused: alpha = sc[2] / sum(part_pq), x += alpha p, r -= alpha q, per-CTA
// partials of r.r into part_rr (count returned), sc[0] = sc[2].
template <typename T> int dot_partials(long long n, const T* a, const T* b, T* part, cudaStream_t st);
template <typename T> void cg_p_fused(long long n, const T* part, int np, T* sc, const T* z, T* p, cudaStream_t st);
template <typename T> int cg_xr_fused(long long n, const T* part_pq, int np, T* sc, const T* p, const T* q, T* x,
                                      T* r, T* part_rr, cudaStream_t st);
template <typename A, typename B> void convert(long long n, const A* a, B* b, double s, cudaStream_t st);
template <typename T> void add_to_double(long long n, const T* x, double* U, cudaStream_t st);
template <typename KT> void impose_dirichlet(const BcDev& bc, long long ndof, double lam, const double* U, KT* K, double* R, double* dg, cudaStream_t st);
void bc_apply(const BcDev& bc, double lam, double* U, cudaStream_t st);
template <typename T> void dense_mv(int n, const T* M, const T* b, T* y, cudaStream_t st);
template <typename T> void sa_setup_level(const AmgLevel<T>& v, T w, T* cval, int nnzC, cudaStream_t st);
template <typename T> void sa_restrict(const AmgLevel<T>& v, const T* r, T* bc, cudaStream_t st);
template <typename T> void sa_prolong(const AmgLevel<T>& v, const T* xc, T* x, cudaStream_t st);
template <typename T> void sa_prolong2(const AmgLevel<T>& v, const T* xc, const T* xc2, T* x, cudaStream_t st);
// Dense inverse of the coarsest operator (dense.cu): its 6 x 6 block pattern
// (device rp, cl) and values in, the n x n row-major inverse in precision T out;
// work holds dense_inverse_work_doubles(n) doubles.
long long dense_inverse_work_doubles(int n);
template <typename T> void dense_coarse_inverse(int nbrow, const int* rp, const int* cl, const T* val, int n,
                                                double* work, T* inv, cudaStream_t st);

}  // namespace pfem
