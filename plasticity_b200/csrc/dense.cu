// dense.cu -- dense inverse of the coarsest AMG operator, on the device.
//
// The smoothed-aggregation hierarchy ends in a dense solve (the reference's
// AlgebraicMultigrid.jl ends its hierarchy in a direct coarse solve as well,
// Solver.jl:136-154).  The coarsest operator (6 x 6 blocks, a few thousand
// unknowns) is expanded to a dense FP64 matrix and inverted in place by blocked
// Gauss-Jordan elimination; the cycle then applies the inverse as one dense
// matrix-vector product.  Per panel of NB columns:
//   1. panel kernel: every CTA inverts the NB x NB diagonal block in shared
//      memory (the same arithmetic in every CTA, so all copies agree; the first
//      one stores it in Dg), scales the panel rows outside the diagonal block by
//      it, and saves the old panel columns of the other rows in C;
//   2. update kernel: A[i, j] -= C[i, :] P[:, j] for every row i outside the
//      panel (P the scaled panel rows, Dg in the panel's own columns), with the
//      panel's own columns starting from 0, which turns them into -C D^{-1};
//      the diagonal block becomes Dg.
// The diagonal block of A is read by every panel CTA and written only by the
// update kernel, so no CTA can see it half replaced.
// No row exchanges: the Galerkin operator of the (Dirichlet-imposed) tangent is
// close to symmetric positive definite; a pivot below 1e-14 of the largest
// diagonal entry is replaced by that floor, as the host inverse did before.
#include <cstdint>

#include "linalg.cuh"

namespace pfem {
namespace {

constexpr int NB = 32;      // panel width
constexpr int TILE = 64;    // update tile (rows and columns)

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

// In-place Gauss-Jordan inverse of the NB x NB block M (shared memory), 256 threads.
__device__ void invert_block(double (*M)[NB + 1], double floor_abs) {
  const int t = threadIdx.x;
  for (int k = 0; k < NB; ++k) {
    __syncthreads();
    double piv = M[k][k];
    if (fabs(piv) < floor_abs) piv = piv >= 0.0 ? floor_abs : -floor_abs;
    const double ip = 1.0 / piv;
    __syncthreads();
    if (t < NB) M[k][t] = (t == k ? 1.0 : M[k][t]) * ip;
    __syncthreads();
    // each thread owns 4 entries of rows i != k
    double f[4];
    int ii[4], jj[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = t + q * 256;
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
}

// Panel step kb: CTAs [0, ncb) scale the panel rows (256 columns each),
// CTAs [ncb, ncb + nrb) save the panel columns of 256 rows each into C (n x NB).
__global__ void __launch_bounds__(256) gj_panel_kernel(int n, int kb, int ncb, double* __restrict__ A,
                                                       double* __restrict__ C, double* __restrict__ Dg,
                                                       const double* __restrict__ scl) {
  __shared__ double D[NB][NB + 1];
  const int t = threadIdx.x;
  if ((int)blockIdx.x >= ncb) {
    const int i = ((int)blockIdx.x - ncb) * 256 + t;
    if (i < n && (i < kb || i >= kb + NB)) {
#pragma unroll 8
      for (int s = 0; s < NB; ++s) C[(long long)i * NB + s] = A[(long long)i * n + kb + s];
    }
    return;
  }
  for (int e = t; e < NB * NB; e += 256) D[e / NB][e % NB] = A[(long long)(kb + e / NB) * n + kb + e % NB];
  invert_block(D, 1e-14 * fmax(scl[0], 1e-300));
  if (blockIdx.x == 0)
    for (int e = t; e < NB * NB; e += 256) Dg[e] = D[e / NB][e % NB];
  const int j = (int)blockIdx.x * 256 + t;
  if (j >= n || (j >= kb && j < kb + NB)) return;
  double v[NB];
#pragma unroll
  for (int s = 0; s < NB; ++s) v[s] = A[(long long)(kb + s) * n + j];
#pragma unroll 4
  for (int r = 0; r < NB; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int s = 0; s < NB; ++s) acc += D[r][s] * v[s];
    A[(long long)(kb + r) * n + j] = acc;
  }
}

// Trailing update of step kb over TILE x TILE tiles; rows of the panel are final.
__global__ void __launch_bounds__(256) gj_update_kernel(int n, int kb, double* __restrict__ A,
                                                        const double* __restrict__ C, const double* __restrict__ Dg) {
  __shared__ double Cs[TILE][NB + 1];
  __shared__ double Ps[NB][TILE + 1];
  const int i0 = (int)blockIdx.y * TILE, j0 = (int)blockIdx.x * TILE;
  const int t = threadIdx.x;
  for (int e = t; e < TILE * NB; e += 256) {
    const int r = e / NB, s = e % NB, i = i0 + r;
    Cs[r][s] = (i < n && (i < kb || i >= kb + NB)) ? C[(long long)i * NB + s] : 0.0;
  }
  for (int e = t; e < NB * TILE; e += 256) {
    const int s = e / TILE, c = e % TILE, j = j0 + c;
    Ps[s][c] = j >= n ? 0.0 : (j >= kb && j < kb + NB) ? Dg[s * NB + (j - kb)] : A[(long long)(kb + s) * n + j];
  }
  // the tile holding the diagonal block writes it (no other CTA reads it from A)
  if (kb >= i0 && kb < i0 + TILE && kb >= j0 && kb < j0 + TILE)
    for (int e = t; e < NB * NB; e += 256) A[(long long)(kb + e / NB) * n + kb + e % NB] = Dg[e];
  __syncthreads();
  const int rg = t / 16, cg = t % 16;  // rows rg*4 .. +3, columns cg + 16 b
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
#pragma unroll 8
  for (int s = 0; s < NB; ++s) {
    double cv[4], pv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) cv[a] = Cs[rg * 4 + a][s];
#pragma unroll
    for (int b = 0; b < 4; ++b) pv[b] = Ps[s][cg + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += cv[a] * pv[b];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + rg * 4 + a;
    if (i >= n || (i >= kb && i < kb + NB)) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int j = j0 + cg + 16 * b;
      if (j >= n) continue;
      double* p = A + (long long)i * n + j;
      const double old = (j >= kb && j < kb + NB) ? 0.0 : *p;
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
  cudaMemsetAsync(A, 0, (size_t)np * np * sizeof(double), st);
  count_launch();
  bsr6_to_dense_kernel<T><<<1024, 256, 0, st>>>(nbrow, rp, cl, val, np, A);
  count_launch();
  dense_fix_rows_kernel<<<(np + 7) / 8, 256, 0, st>>>(np, A);
  count_launch();
  dense_diag_max_kernel<<<1, 1024, 0, st>>>(np, A, scl);
  const int ncb = (np + 255) / 256, nrb = (np + 255) / 256;
  const dim3 ug((np + TILE - 1) / TILE, (np + TILE - 1) / TILE);
  for (int kb = 0; kb < np; kb += NB) {
    count_launch();
    gj_panel_kernel<<<ncb + nrb, 256, 0, st>>>(np, kb, ncb, A, C, Dg, scl);
    count_launch();
    gj_update_kernel<<<ug, 256, 0, st>>>(np, kb, A, C, Dg);
  }
  count_launch();
  dense_out_kernel<T><<<2048, 256, 0, st>>>(n, np, A, inv);
}

template void dense_coarse_inverse<float>(int, const int*, const int*, const float*, int, double*, float*,
                                          cudaStream_t);
template void dense_coarse_inverse<double>(int, const int*, const int*, const double*, int, double*, double*,
                                           cudaStream_t);

}  // namespace pfem
