// dense.cu -- dense inverse of the coarsest AMG operator, on the device.
//
// The smoothed-aggregation hierarchy ends in a dense solve (the reference's
// AlgebraicMultigrid.jl ends its hierarchy in a direct coarse solve as well,
// Solver.jl:136-154).  The coarsest operator (6 x 6 blocks, a few thousand
// unknowns) is expanded to a dense FP64 matrix and inverted in place by blocked
// Gauss-Jordan elimination; the cycle then applies the inverse as one dense
// matrix-vector product.  Per panel of NB columns K:
//   1. diagonal kernel (one CTA): Dg = A[K,K]^{-1} by Gauss-Jordan in shared memory;
//   2. panel kernel: the panel rows outside the diagonal block, A[K,j] <- Dg A[K,j],
//      and a copy C = A[i,K] of the panel columns of the other rows;
//   3. update kernel: A[i, j] -= C[i, :] P[:, j] for every row i outside the panel
//      (P the scaled panel rows, Dg in the panel's own columns), with the panel's
//      own columns starting from 0, which turns them into -C Dg; the tile that
//      holds the diagonal block writes Dg there.
// Every kernel reads only what the previous one finished writing, and A[K,K] is
// read only by the diagonal kernel, so no CTA sees a block half replaced.
// No row exchanges: the Galerkin operator of the (Dirichlet-imposed) tangent of a
// large mesh is close to symmetric positive definite (small coarsest levels are
// inverted on the host with partial pivoting instead); a pivot below 1e-14 of the
// largest diagonal entry is replaced by that floor.
#include <cstdint>

#include "linalg.cuh"

namespace pfem {
namespace {

constexpr int NB = 64;      // panel width
constexpr int TR_ = 128;    // update tile rows
constexpr int TC_ = 64;     // update tile columns

// Dense row-major n x n FP64 matrix from the coarsest level's 6 x 6 blocks.
template <typename T>
__global__ void bsr6_to_dense_kernel(int nbrow, const int* __restrict__ rp, const int* __restrict__ cl,
                                     const T* __restrict__ val, int n, double* __restrict__ A) {
  const long long nnzb = rp[nbrow];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nnzb * 36;
       t += (long long)gridDim.x * blockDim.x) {
    const long long k = t / 36;
    const int e = (int)(t % 36), r = e / 6, c = e % 6;
    // block row of k: binary search in rp
    int lo = 0, hi = nbrow;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (rp[mid] <= k) lo = mid; else hi = mid;
    }
    A[(long long)(lo * 6 + r) * n + cl[k] * 6 + c] = (double)val[t];
  }
}

// Rows with no entry (rigid modes absent from an aggregate) get a unit
// diagonal; one warp per row.
__global__ void dense_fix_rows_kernel(int n, double* __restrict__ A) {
  const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // whole warps
  bool nz = false;
  for (int j = lane; j < n; j += 32) nz |= A[(long long)i * n + j] != 0.0;
  nz = __any_sync(0xffffffffu, nz);
  if (!nz && lane == 0) A[(long long)i * n + i] = 1.0;
}

// scl[0] = the largest |diagonal entry| (the pivot floor's scale), one CTA.
__global__ void dense_diag_max_kernel(int n, const double* __restrict__ A, double* __restrict__ scl) {
  __shared__ double sh[32];
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(A[(long long)i * n + i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmax(m, sh[k]);
    scl[0] = m;
  }
}

// Dg = A[K,K]^{-1}: in-place Gauss-Jordan on the NB x NB diagonal block in
// shared memory, one CTA of 1024 threads (four entries each).
__global__ void __launch_bounds__(1024) gj_diag_kernel(int n, int kb, const double* __restrict__ A,
                                                       double* __restrict__ Dg, const double* __restrict__ scl) {
  __shared__ double M[NB][NB + 1];
  const int t = threadIdx.x;
  for (int e = t; e < NB * NB; e += 1024) M[e / NB][e % NB] = A[(long long)(kb + e / NB) * n + kb + e % NB];
  const double floor_abs = 1e-14 * fmax(scl[0], 1e-300);
  for (int k = 0; k < NB; ++k) {
    __syncthreads();
    double piv = M[k][k];
    if (fabs(piv) < floor_abs) piv = piv >= 0.0 ? floor_abs : -floor_abs;
    const double ip = 1.0 / piv;
    __syncthreads();
    if (t < NB) M[k][t] = (t == k ? 1.0 : M[k][t]) * ip;
    __syncthreads();
    double f[4];
    int ii[4], jj[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = t + q * 1024;
      ii[q] = e / NB;
      jj[q] = e % NB;
      f[q] = M[ii[q]][k];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (ii[q] == k) continue;
      const double old = jj[q] == k ? 0.0 : M[ii[q]][jj[q]];
      M[ii[q]][jj[q]] = old - f[q] * M[k][jj[q]];
    }
  }
  __syncthreads();
  for (int e = t; e < NB * NB; e += 1024) Dg[e] = M[e / NB][e % NB];
}

// Panel step kb.  CTAs [0, ncb): 64 panel-row columns each, A[K, j] <- Dg A[K, j]
// for j outside K (the 64 x 64 slab staged in shared memory; thread (column,
// quarter) computes 16 rows).  CTAs [ncb, ...): C[i, :] = A[i, K] for rows i
// outside K, a warp per row.
__global__ void __launch_bounds__(256) gj_panel_kernel(int n, int kb, int ncb, double* __restrict__ A,
                                                       double* __restrict__ C, const double* __restrict__ Dg) {
  extern __shared__ __align__(16) double psm[];
  const int t = threadIdx.x;
  if ((int)blockIdx.x >= ncb) {
    const int w = t >> 5, lane = t & 31;
    const int i = ((int)blockIdx.x - ncb) * 8 + w;
    if (i < n && (i < kb || i >= kb + NB)) {
      C[(long long)i * NB + lane] = A[(long long)i * n + kb + lane];
      C[(long long)i * NB + 32 + lane] = A[(long long)i * n + kb + 32 + lane];
    }
    return;
  }
  const int j0 = (int)blockIdx.x * 64;
  if (j0 == kb) return;  // the diagonal block's columns: Dg, written by the update kernel
  double(*D)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(psm);
  double(*V)[65] = reinterpret_cast<double(*)[65]>(psm + NB * (NB + 1));
  for (int e = t; e < NB * NB; e += 256) D[e / NB][e % NB] = Dg[e];
  for (int e = t; e < NB * 64; e += 256) {
    const int r = e / 64, c = e % 64, j = j0 + c;
    V[r][c] = j < n ? A[(long long)(kb + r) * n + j] : 0.0;
  }
  __syncthreads();
  const int c = t & 63, q = t >> 6, j = j0 + c;
  if (j >= n) return;
  double out[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) out[r] = 0.0;
#pragma unroll 8
  for (int s = 0; s < NB; ++s) {
    const double v = V[s][c];
#pragma unroll
    for (int r = 0; r < 16; ++r) out[r] += D[q * 16 + r][s] * v;
  }
#pragma unroll
  for (int r = 0; r < 16; ++r) A[(long long)(kb + q * 16 + r) * n + j] = out[r];
}

// Trailing update of step kb over TR_ x TC_ tiles; rows of the panel are final.
// Thread (rg, cg) holds rows rg*8 .. +7 and columns cg + 16 b, b < 4.
__global__ void __launch_bounds__(256, 2) gj_update_kernel(int n, int kb, double* __restrict__ A,
                                                           const double* __restrict__ C,
                                                           const double* __restrict__ Dg) {
  extern __shared__ __align__(16) double usm[];
  double(*Cs)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(usm);              // TR_ x NB
  double(*Ps)[TC_ + 1] = reinterpret_cast<double(*)[TC_ + 1]>(usm + TR_ * (NB + 1));  // NB x TC_
  const int i0 = (int)blockIdx.y * TR_, j0 = (int)blockIdx.x * TC_;
  const int t = threadIdx.x;
  for (int e = t; e < TR_ * NB; e += 256) {
    const int r = e / NB, s = e % NB, i = i0 + r;
    Cs[r][s] = (i < n && (i < kb || i >= kb + NB)) ? C[(long long)i * NB + s] : 0.0;
  }
  const bool diag_cols = j0 == kb;  // TC_ == NB and both are multiples of NB: the panel is one column tile
  for (int e = t; e < NB * TC_; e += 256) {
    const int s = e / TC_, c = e % TC_, j = j0 + c;
    Ps[s][c] = j >= n ? 0.0 : diag_cols ? Dg[s * NB + c] : A[(long long)(kb + s) * n + j];
  }
  // the tile holding the diagonal block writes it (no other CTA reads it from A)
  if (diag_cols && kb >= i0 && kb < i0 + TR_)
    for (int e = t; e < NB * NB; e += 256) A[(long long)(kb + e / NB) * n + kb + e % NB] = Dg[e];
  __syncthreads();
  const int rg = t / 16, cg = t % 16;
  double acc[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 4
  for (int s = 0; s < NB; ++s) {
    double cv[8], pv[4];
#pragma unroll
    for (int a = 0; a < 8; ++a) cv[a] = Cs[rg * 8 + a][s];
#pragma unroll
    for (int b = 0; b < 4; ++b) pv[b] = Ps[s][cg + 16 * b];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += cv[a] * pv[b];
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int i = i0 + rg * 8 + a;
    if (i >= n || (i >= kb && i < kb + NB)) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = j0 + cg + 16 * b;
      if (j >= n) continue;
      double* p = A + (long long)i * n + j;
      const double old = diag_cols ? 0.0 : *p;
      *p = old - acc[a][b];
    }
  }
}

// out (n x n, stride n) = the leading n x n block of A (stride np), in precision T.
template <typename T>
__global__ void dense_out_kernel(int n, int np, const double* __restrict__ A, T* __restrict__ out) {
  const long long nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x)
    out[e] = (T)A[(e / n) * np + e % n];
}

}  // namespace

long long dense_inverse_work_doubles(int n) {
  const int np = (n + NB - 1) / NB * NB;
  return (long long)np * np + (long long)np * NB + NB * NB + 8;
}

// inv (n x n, row-major, precision T) = inverse of the coarsest operator given by
// its 6 x 6 block pattern (rp, cl: device) and values.  work holds
// dense_inverse_work_doubles(n) doubles.  The matrix is padded to a multiple of
// NB with identity rows, which leaves the inverse of the leading block unchanged.
template <typename T>
void dense_coarse_inverse(int nbrow, const int* rp, const int* cl, const T* val, int n, double* work, T* inv,
                          cudaStream_t st) {
  const int np = (n + NB - 1) / NB * NB;
  double* A = work;
  double* C = work + (long long)np * np;
  double* Dg = C + (long long)np * NB;
  double* scl = Dg + NB * NB;
  const size_t panel_sm = (size_t)(NB * (NB + 1) + NB * 65) * sizeof(double);
  const size_t update_sm = (size_t)(TR_ * (NB + 1) + NB * (TC_ + 1)) * sizeof(double);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(gj_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel_sm);
    cudaFuncSetAttribute(gj_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)update_sm);
    attr = true;
  }
  cudaMemsetAsync(A, 0, (size_t)np * np * sizeof(double), st);
  count_launch();
  bsr6_to_dense_kernel<T><<<1024, 256, 0, st>>>(nbrow, rp, cl, val, np, A);
  count_launch();
  dense_fix_rows_kernel<<<(np + 7) / 8, 256, 0, st>>>(np, A);
  count_launch();
  dense_diag_max_kernel<<<1, 1024, 0, st>>>(np, A, scl);
  const int ncb = np / 64, nrb = (np + 7) / 8;
  const dim3 ug((np + TC_ - 1) / TC_, (np + TR_ - 1) / TR_);
  for (int kb = 0; kb < np; kb += NB) {
    count_launch();
    gj_diag_kernel<<<1, 1024, 0, st>>>(np, kb, A, Dg, scl);
    count_launch();
    gj_panel_kernel<<<ncb + nrb, 256, panel_sm, st>>>(np, kb, ncb, A, C, Dg);
    count_launch();
    gj_update_kernel<<<ug, 256, update_sm, st>>>(np, kb, A, C, Dg);
  }
  count_launch();
  dense_out_kernel<T><<<2048, 256, 0, st>>>(n, np, A, inv);
}

template void dense_coarse_inverse<float>(int, const int*, const int*, const float*, int, double*, float*,
                                          cudaStream_t);
template void dense_coarse_inverse<double>(int, const int*, const int*, const double*, int, double*, double*,
                                           cudaStream_t);

}  // namespace pfem
