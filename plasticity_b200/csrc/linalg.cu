// linalg.cu -- block-CSR SpMV, smoother / Krylov vector kernels, reductions,
// Dirichlet imposition and AMG transfer kernels.  All are HBM-bound; each is
// written so that one pass over the matrix does all the work the caller needs
// from that pass (SpMV + residual, SpMV + block-Jacobi Chebyshev update).
#include <cstdint>
#include <type_traits>

#include "linalg.cuh"

namespace pfem {

// ------------------------------------------------------------------ SpMV
// Half a warp per block row; lane k holds block rowptr[i]+k (+16, ...), loads
// the whole bs x bs block and the matching bs entries of x, and the half-warp
// reduces the bs partial sums by a fixed xor tree.  Mode selects the epilogue:
//   0: y = A x
//   1: y = b - A x                          (residual)
//   2: r -= Dinv (A x); xo += x             (Chebyshev step on x = d)
//   3: xo = c2 x + c1 (y - Dinv A x)        (fused degree-2 Chebyshev, x = d0, y = r0)
//   4: as 3, added to xo
//   5: y = Dinv (b - A x), xo = c1 y        (preconditioned residual + first direction)
template <typename T, int BS, int MODE, bool VEC = false, int LANES = 16, bool C16 = false>
__global__ void __launch_bounds__(256) bsr_spmv_kernel(int nbrow, const int* __restrict__ rowptr,
                                                       const int* __restrict__ col,
                                                       const int16_t* __restrict__ col16,
                                                       const T* __restrict__ val,
                                                       const T* __restrict__ x, T* __restrict__ y,
                                                       const T* __restrict__ b,
                                                       const T* __restrict__ dinv, T* __restrict__ xo,
                                                       T c1, T c2) {
  // LANES lanes per block row: half a warp for 3 x 3 blocks (a level-0 row has at
  // most 27 blocks: two per lane), a warp for 6 x 6 blocks (one 144-byte block
  // per lane); values and column ids are read once, through the streaming
  // (evict-first) path so they do not push the gathered x out of the caches.
  static_assert(LANES == 16 || LANES == 32, "half or whole warps per row");
  const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) / LANES);
  const int lane = threadIdx.x & (LANES - 1);
  const bool ok = row < nbrow;
  const int s = ok ? rowptr[row] : 0, e = ok ? rowptr[row + 1] : 0;
  T acc[BS];
#pragma unroll
  for (int i = 0; i < BS; ++i) acc[i] = T(0);
  for (int k = s + lane; k < e; k += LANES) {
    const int c = C16 ? row + (int)__ldcs(col16 + k) : __ldcs(col + k);
    const T* B = val + (long long)k * (BS * BS);
    T bv[BS * BS];
    if constexpr (VEC) {
      // 16-byte streaming loads (a 6 x 6 block is 144 / 288 bytes; the launcher
      // checks that val is 16-byte aligned, so every block is)
      using V = typename std::conditional<std::is_same<T, float>::value, float4, double2>::type;
      constexpr int PER = 16 / (int)sizeof(T), NV = BS * BS / PER;
      static_assert(BS * BS % PER == 0, "vector loads need whole 16-byte groups");
      const V* B4 = reinterpret_cast<const V*>(B);
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const V v = __ldcs(B4 + q);
        const T* vt = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int j = 0; j < PER; ++j) bv[q * PER + j] = vt[j];
      }
    } else {
#pragma unroll
      for (int q = 0; q < BS * BS; ++q) bv[q] = __ldcs(B + q);
    }
    T xv[BS];
#pragma unroll
    for (int j = 0; j < BS; ++j) xv[j] = x[(long long)c * BS + j];
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) acc[i] += bv[i * BS + j] * xv[j];
  }
#pragma unroll
  for (int i = 0; i < BS; ++i) {
    T v = acc[i];
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[i] = v;
  }
  if (ok && lane < BS) {
    const long long base = (long long)row * BS;
    if (MODE == 5) {
      // r = Dinv (b - A x) (into y), d = c1 r (into xo)
      const T* D = dinv + (long long)row * (BS * BS);
      T t = T(0);
#pragma unroll
      for (int j = 0; j < BS; ++j) t += D[lane * BS + j] * (b[base + j] - acc[j]);
      y[base + lane] = t;
      xo[base + lane] = c1 * t;
      return;
    }
    T v = acc[0];
#pragma unroll
    for (int i = 1; i < BS; ++i)
      if (lane == i) v = acc[i];
    if (MODE == 0) {
      y[base + lane] = v;
    } else if (MODE == 1) {
      y[base + lane] = b[base + lane] - v;
    } else {
      // t = (Dinv A d)_lane with d = x (the gathered vector)
      const T* D = dinv + (long long)row * (BS * BS);
      T t = T(0);
#pragma unroll
      for (int j = 0; j < BS; ++j) t += D[lane * BS + j] * acc[j];
      if (MODE == 2) {
        y[base + lane] -= t;
        xo[base + lane] += x[base + lane];
      } else {
        // degree-2 Chebyshev in one pass: r1 = r0 - Dinv A d0,
        // x2 = x0 + c2 d0 + c1 r1 (c2 = 1 + rn rho, c1 = 2 rn / delta)
        const T upd = c2 * x[base + lane] + c1 * (y[base + lane] - t);
        if (MODE == 3) xo[base + lane] = upd;
        else xo[base + lane] += upd;
      }
    }
  }
}

template <typename T, int MODE>
static void spmv_launch(const BsrMat<T>& A, const T* x, T* y, const T* b, const T* dinv, T* xo, T c1, T c2,
                        cudaStream_t st) {
  // 6 x 6 levels of fewer than kWarpRowsBelow rows fill too few warp slots with half
  // a warp per row: give each row a whole warp there (measured at 64^3: level 2,
  // 512 rows, 7.4 -> 6.5 us per pass; level 1, 10,648 rows, 14.3 -> 18.2 us)
  constexpr int kWarpRowsBelow = 4096;
  const bool wide = A.bs == 6 && A.nbrow < kWarpRowsBelow;
  // 128-thread blocks: the whole cycle inside a CUDA graph measured 422.1 us against
  // 425.0 us with 256 at 64^3 (1.3667 vs 1.3679 ms at 100^3)
  constexpr int kThreads = 128;
  const long long threads = (long long)A.nbrow * (wide ? 32 : 16);
  const int blocks = (int)((threads + kThreads - 1) / kThreads);
  const bool aligned = (reinterpret_cast<uintptr_t>(A.val) & 15) == 0;
  pfem::count_launch();
  if (A.bs == 3 && A.col16)
    bsr_spmv_kernel<T, 3, MODE, false, 16, true><<<blocks, kThreads, 0, st>>>(A.nbrow, A.rowptr, A.col, A.col16,
                                                                              A.val, x, y, b, dinv, xo, c1, c2);
  else if (A.bs == 3)
    bsr_spmv_kernel<T, 3, MODE><<<blocks, kThreads, 0, st>>>(A.nbrow, A.rowptr, A.col, A.col16, A.val, x, y, b, dinv, xo, c1, c2);
  else if (aligned && wide)
    bsr_spmv_kernel<T, 6, MODE, true, 32><<<blocks, kThreads, 0, st>>>(A.nbrow, A.rowptr, A.col, A.col16, A.val, x, y, b, dinv, xo,
                                                                  c1, c2);
  else if (aligned)
    bsr_spmv_kernel<T, 6, MODE, true><<<blocks, kThreads, 0, st>>>(A.nbrow, A.rowptr, A.col, A.col16, A.val, x, y, b, dinv, xo, c1,
                                                              c2);
  else
    bsr_spmv_kernel<T, 6, MODE><<<blocks, kThreads, 0, st>>>(A.nbrow, A.rowptr, A.col, A.col16, A.val, x, y, b, dinv, xo, c1, c2);
}

template <typename T>
void bsr_spmv(const BsrMat<T>& A, const T* x, T* y, cudaStream_t st) {
  spmv_launch<T, 0>(A, x, y, nullptr, nullptr, nullptr, T(0), T(0), st);
}
template <typename T>
void bsr_residual(const BsrMat<T>& A, const T* x, const T* b, T* r, cudaStream_t st) {
  spmv_launch<T, 1>(A, x, r, b, nullptr, nullptr, T(0), T(0), st);
}
template <typename T>
void bsr_cheb_step(const BsrMat<T>& A, const T* dinv, const T* d, T* r, T* x, cudaStream_t st) {
  spmv_launch<T, 2>(A, d, r, nullptr, dinv, x, T(0), T(0), st);
}
template <typename T>
void bsr_cheb2(const BsrMat<T>& A, const T* dinv, const T* d0, const T* r0, T* x, bool zero, T c1, T c2,
               cudaStream_t st) {
  if (zero) spmv_launch<T, 3>(A, d0, const_cast<T*>(r0), nullptr, dinv, x, c1, c2, st);
  else spmv_launch<T, 4>(A, d0, const_cast<T*>(r0), nullptr, dinv, x, c1, c2, st);
}
template <typename T>
void bsr_residual_precond(const BsrMat<T>& A, const T* dinv, const T* x, const T* b, T* r, T* d, T scale,
                          cudaStream_t st) {
  spmv_launch<T, 5>(A, x, r, b, dinv, d, scale, T(0), st);
}

// ------------------------------------------------------------------ block diagonal
// r = Dinv * v per block row (one thread per scalar row); optional scale.
template <typename T, int BS>
__global__ void blockdiag_apply_kernel(int nbrow, const T* __restrict__ dinv, const T* __restrict__ v,
                                       T* __restrict__ r, T scale, T* __restrict__ d) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nbrow * BS) return;
  const long long row = i / BS;
  const int li = (int)(i - row * BS);
  const T* D = dinv + row * (BS * BS) + li * BS;
  const T* vv = v + row * BS;
  T t = T(0);
#pragma unroll
  for (int j = 0; j < BS; ++j) t += D[j] * vv[j];
  r[i] = t;
  if (d) d[i] = scale * t;
}
template <typename T>
void blockdiag_apply(int nbrow, int bs, const T* dinv, const T* v, T* r, T scale, T* d, cudaStream_t st) {
  const long long n = (long long)nbrow * bs;
  const int blocks = (int)((n + 255) / 256);
  if (bs == 3) { pfem::count_launch(); blockdiag_apply_kernel<T, 3><<<blocks, 256, 0, st>>>(nbrow, dinv, v, r, scale, d); }
  else { pfem::count_launch(); blockdiag_apply_kernel<T, 6><<<blocks, 256, 0, st>>>(nbrow, dinv, v, r, scale, d); }
}

// Invert the diagonal blocks (Gauss-Jordan with partial pivoting in double).
// A singular block (a Dirichlet-free rigid aggregate, say) gets the inverse of
// its diagonal instead, with zero diagonal entries mapped to 1.
template <typename T, int BS>
__global__ void blockdiag_invert_kernel(int nbrow, const int* __restrict__ rowptr, const int* __restrict__ col,
                                        const T* __restrict__ val, T* __restrict__ dinv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nbrow) return;
  double a[BS][2 * BS];
  int kd = -1;
  for (int k = rowptr[row]; k < rowptr[row + 1]; ++k)
    if (col[k] == row) { kd = k; break; }
  for (int i = 0; i < BS; ++i)
    for (int j = 0; j < BS; ++j) {
      a[i][j] = kd >= 0 ? (double)val[(long long)kd * BS * BS + i * BS + j] : 0.0;
      a[i][BS + j] = (i == j) ? 1.0 : 0.0;
    }
  bool ok = true;
  double scl = 0.0;
  for (int i = 0; i < BS; ++i) scl = fmax(scl, fabs(a[i][i]));
  for (int c = 0; c < BS && ok; ++c) {
    int piv = c;
    double best = fabs(a[c][c]);
    for (int r = c + 1; r < BS; ++r)
      if (fabs(a[r][c]) > best) { best = fabs(a[r][c]); piv = r; }
    if (!(best > 1e-13 * scl) || !(best > 0.0)) { ok = false; break; }
    if (piv != c)
      for (int j = 0; j < 2 * BS; ++j) { double t = a[c][j]; a[c][j] = a[piv][j]; a[piv][j] = t; }
    const double ip = 1.0 / a[c][c];
    for (int j = 0; j < 2 * BS; ++j) a[c][j] *= ip;
    for (int r = 0; r < BS; ++r)
      if (r != c) {
        const double f = a[r][c];
        if (f != 0.0)
          for (int j = 0; j < 2 * BS; ++j) a[r][j] -= f * a[c][j];
      }
  }
  T* D = dinv + (long long)row * BS * BS;
  if (ok) {
    for (int i = 0; i < BS; ++i)
      for (int j = 0; j < BS; ++j) D[i * BS + j] = (T)a[i][BS + j];
  } else {
    for (int i = 0; i < BS; ++i)
      for (int j = 0; j < BS; ++j) {
        double dv = kd >= 0 ? (double)val[(long long)kd * BS * BS + i * BS + i] : 0.0;
        D[i * BS + j] = (i == j) ? (T)(dv != 0.0 ? 1.0 / dv : 1.0) : T(0);
      }
  }
}
template <typename T>
void blockdiag_invert(const BsrMat<T>& A, T* dinv, cudaStream_t st) {
  const int blocks = (A.nbrow + 127) / 128;
  if (A.bs == 3) { pfem::count_launch(); blockdiag_invert_kernel<T, 3><<<blocks, 128, 0, st>>>(A.nbrow, A.rowptr, A.col, A.val, dinv); }
  else { pfem::count_launch(); blockdiag_invert_kernel<T, 6><<<blocks, 128, 0, st>>>(A.nbrow, A.rowptr, A.col, A.val, dinv); }
}

// ------------------------------------------------------------------ reductions
// Deterministic two-pass dot product: per-block partials, then one block.
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 1184;  // 148 SMs x 8

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : T(0);
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

template <typename T>
__global__ void dot_partial_kernel(long long n, const T* __restrict__ a, const T* __restrict__ b,
                                   T* __restrict__ part) {
  __shared__ T sh[32];
  T v = T(0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
template <typename T>
__global__ void sum_final_kernel(int np, const T* __restrict__ part, T* __restrict__ out, int sqrt_out) {
  __shared__ T sh[32];
  T v = T(0);
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) *out = sqrt_out ? sqrt(v) : v;
}
template <typename T>
void dot(long long n, const T* a, const T* b, T* out, T* part, cudaStream_t st, bool take_sqrt) {
  long long nb = (n + RED_THREADS - 1) / RED_THREADS;
  const int blocks = (int)(nb < RED_BLOCKS ? (nb > 0 ? nb : 1) : RED_BLOCKS);
  pfem::count_launch(); dot_partial_kernel<T><<<blocks, RED_THREADS, 0, st>>>(n, a, b, part);
  pfem::count_launch(); sum_final_kernel<T><<<1, 1024, 0, st>>>(blocks, part, out, take_sqrt ? 1 : 0);
}

// ------------------------------------------------------------------ vector ops
template <typename T>
__global__ void fill_kernel(long long n, T* x, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}
template <typename T>
void fill(long long n, T* x, T v, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  if (n > 0) { pfem::count_launch(); fill_kernel<T><<<blocks > 0 ? blocks : 1, 256, 0, st>>>(n, x, v); }
}
// y = a*x + b*y with host scalars
template <typename T>
__global__ void axpby_kernel(long long n, T a, const T* __restrict__ x, T b, T* __restrict__ y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}
template <typename T>
void axpby(long long n, T a, const T* x, T b, T* y, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  if (n > 0) { pfem::count_launch(); axpby_kernel<T><<<blocks, 256, 0, st>>>(n, a, x, b, y); }
}
// CG update with device scalars: alpha = num/den;  x += alpha p;  r -= alpha q
template <typename T>
__global__ void cg_xr_kernel(long long n, const T* __restrict__ num, const T* __restrict__ den,
                             const T* __restrict__ p, const T* __restrict__ q, T* __restrict__ x,
                             T* __restrict__ r) {
  const T al = *num / *den;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += al * p[i];
    r[i] -= al * q[i];
  }
}
template <typename T>
void cg_xr(long long n, const T* num, const T* den, const T* p, const T* q, T* x, T* r, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); cg_xr_kernel<T><<<blocks, 256, 0, st>>>(n, num, den, p, q, x, r);
}
// p = z + (num/den) p
template <typename T>
__global__ void cg_p_kernel(long long n, const T* __restrict__ num, const T* __restrict__ den,
                            const T* __restrict__ z, T* __restrict__ p) {
  const T be = *num / *den;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + be * p[i];
}
template <typename T>
void cg_p(long long n, const T* num, const T* den, const T* z, T* p, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); cg_p_kernel<T><<<blocks, 256, 0, st>>>(n, num, den, z, p);
}
// ---- PCG updates with the final reduction fused in ----
// Every CTA sums the same np partials in the same order (a strided pass and a
// fixed tree), so all CTAs see the same scalar and the result is deterministic.
template <typename T>
__device__ __forceinline__ T all_sum_partials(const T* __restrict__ part, int np, T* sh) {
  T v = T(0);
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
  v = block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[32] = v;
  __syncthreads();
  return sh[32];
}
// rz = sum(part_rz);  p = z + (rz / sc[0]) p;  sc[2] = rz
template <typename T>
__global__ void cg_p_fused_kernel(long long n, const T* __restrict__ part, int np, T* __restrict__ sc,
                                  const T* __restrict__ z, T* __restrict__ p) {
  __shared__ T sh[33];
  const T rz = all_sum_partials(part, np, sh);
  const T be = rz / sc[0];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + be * p[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) sc[2] = rz;
}
// pq = sum(part_pq);  alpha = sc[2] / pq;  x += alpha p;  r -= alpha q;
// part_rr[cta] = this CTA's share of r.r;  sc[0] = sc[2] (r.z of the next beta)
template <typename T>
__global__ void cg_xr_fused_kernel(long long n, const T* __restrict__ part_pq, int np, T* __restrict__ sc,
                                   const T* __restrict__ p, const T* __restrict__ q, T* __restrict__ x,
                                   T* __restrict__ r, T* __restrict__ part_rr) {
  __shared__ T sh[33];
  const T pq = all_sum_partials(part_pq, np, sh);
  const T al = sc[2] / pq;
  T acc = T(0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += al * p[i];
    const T ri = r[i] - al * q[i];
    r[i] = ri;
    acc += ri * ri;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part_rr[blockIdx.x] = acc;
  if (blockIdx.x == 0 && threadIdx.x == 0) sc[0] = sc[2];
}
template <typename T>
int dot_partials(long long n, const T* a, const T* b, T* part, cudaStream_t st) {
  long long nb = (n + RED_THREADS - 1) / RED_THREADS;
  const int blocks = (int)(nb < RED_BLOCKS ? (nb > 0 ? nb : 1) : RED_BLOCKS);
  pfem::count_launch(); dot_partial_kernel<T><<<blocks, RED_THREADS, 0, st>>>(n, a, b, part);
  return blocks;
}
int fused_update_blocks(long long n) {
  const long long nb = (n + RED_THREADS - 1) / RED_THREADS;
  return (int)(nb < RED_BLOCKS ? (nb > 0 ? nb : 1) : RED_BLOCKS);
}
template <typename T>
void cg_p_fused(long long n, const T* part, int np, T* sc, const T* z, T* p, cudaStream_t st) {
  pfem::count_launch();
  cg_p_fused_kernel<T><<<fused_update_blocks(n), RED_THREADS, 0, st>>>(n, part, np, sc, z, p);
}
template <typename T>
int cg_xr_fused(long long n, const T* part_pq, int np, T* sc, const T* p, const T* q, T* x, T* r, T* part_rr,
                cudaStream_t st) {
  const int blocks = fused_update_blocks(n);
  pfem::count_launch();
  cg_xr_fused_kernel<T><<<blocks, RED_THREADS, 0, st>>>(n, part_pq, np, sc, p, q, x, r, part_rr);
  return blocks;
}

// BiCGStab helpers with device scalars s[0..]: see krylov code for layout.
template <typename T>
__global__ void bicg_p_kernel(long long n, const T* __restrict__ sc, const T* __restrict__ r,
                              const T* __restrict__ v, T* __restrict__ p) {
  // beta = (rho_new/rho_old)*(alpha/omega); p = r + beta (p - omega v)
  const T beta = (sc[0] / sc[1]) * (sc[2] / sc[3]);
  const T om = sc[3];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = r[i] + beta * (p[i] - om * v[i]);
}
template <typename T>
void bicg_p(long long n, const T* sc, const T* r, const T* v, T* p, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); bicg_p_kernel<T><<<blocks, 256, 0, st>>>(n, sc, r, v, p);
}
// s = r - alpha v  (alpha = sc[0]/sc[4])
template <typename T>
__global__ void bicg_s_kernel(long long n, const T* __restrict__ sc, const T* __restrict__ r,
                              const T* __restrict__ v, T* __restrict__ s) {
  const T al = sc[0] / sc[4];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s[i] = r[i] - al * v[i];
}
template <typename T>
void bicg_s(long long n, const T* sc, const T* r, const T* v, T* s, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); bicg_s_kernel<T><<<blocks, 256, 0, st>>>(n, sc, r, v, s);
}
// x += alpha ph + omega sh;  r = s - omega t  (alpha = sc[0]/sc[4], omega = sc[5]/sc[6])
template <typename T>
__global__ void bicg_xr_kernel(long long n, const T* __restrict__ sc, const T* __restrict__ ph,
                               const T* __restrict__ sh, const T* __restrict__ s, const T* __restrict__ t,
                               T* __restrict__ x, T* __restrict__ r) {
  const T al = sc[0] / sc[4];
  const T om = sc[5] / sc[6];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += al * ph[i] + om * sh[i];
    r[i] = s[i] - om * t[i];
  }
}
template <typename T>
void bicg_xr(long long n, const T* sc, const T* ph, const T* sh, const T* s, const T* t, T* x, T* r,
             cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); bicg_xr_kernel<T><<<blocks, 256, 0, st>>>(n, sc, ph, sh, s, t, x, r);
}
// scalar bookkeeping: dst[i] = src[j]
template <typename T>
__global__ void scalar_copy_kernel(T* dst, const T* src) { *dst = *src; }
template <typename T>
void scalar_copy(T* dst, const T* src, cudaStream_t st) {
  pfem::count_launch();
  scalar_copy_kernel<T><<<1, 1, 0, st>>>(dst, src);
}

// precision conversion
template <typename A, typename B>
__global__ void convert_kernel(long long n, const A* __restrict__ a, B* __restrict__ b, double s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (B)(s * (double)a[i]);
}
template <typename A, typename B>
void convert(long long n, const A* a, B* b, double s, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); convert_kernel<A, B><<<blocks, 256, 0, st>>>(n, a, b, s);
}
// U += (double) x
template <typename T>
__global__ void add_to_double_kernel(long long n, const T* __restrict__ x, double* __restrict__ U) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    U[i] += (double)x[i];
}
template <typename T>
void add_to_double(long long n, const T* x, double* U, cudaStream_t st) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
  pfem::count_launch(); add_to_double_kernel<T><<<blocks, 256, 0, st>>>(n, x, U);
}

// ------------------------------------------------------------------ Dirichlet (K3)
// R -= lambda * Fn  over all dofs, then dg = g(lambda) - U on constrained dofs.
__global__ void residual_fext_kernel(long long n, double lam, const double* __restrict__ fn,
                                     double* __restrict__ R) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    R[i] -= lam * fn[i];
}
__global__ void bc_dg_kernel(int nbc, const int* __restrict__ dofs, const double* __restrict__ vals,
                             const uint8_t* __restrict__ ramp, double lam, const double* __restrict__ U,
                             double* __restrict__ dg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbc) return;
  const int d = dofs[i];
  const double g = ramp[i] ? lam * vals[i] : vals[i];
  dg[d] = g - U[d];
}
// Free rows touching constrained columns: R[row] += sum_k K[pos_k] * dg[col_k]
// (impose_dirichlet!, BoundaryConditions.jl:248-256).  One thread per row.
template <typename KT>
__global__ void bc_rhs_kernel(int nrows, const int* __restrict__ rows, const int* __restrict__ ptr,
                              const long long* __restrict__ pos, const int* __restrict__ cols,
                              const KT* __restrict__ K, const double* __restrict__ dg,
                              double* __restrict__ R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  double s = 0.0;
  for (int k = ptr[i]; k < ptr[i + 1]; ++k) s += (double)K[pos[k]] * dg[cols[k]];
  R[rows[i]] += s;
}
// Zero constrained rows / columns, unit diagonal (BoundaryConditions.jl:259-266).
template <typename KT>
__global__ void bc_zero_kernel(long long n, const long long* __restrict__ pos, const uint8_t* __restrict__ one,
                               KT* __restrict__ K) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    K[pos[i]] = one[i] ? KT(1) : KT(0);
}
// R[d] = -dg[d] (BoundaryConditions.jl:269-272)
__global__ void bc_set_kernel(int nbc, const int* __restrict__ dofs, const double* __restrict__ dg,
                              double* __restrict__ R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbc) return;
  R[dofs[i]] = -dg[dofs[i]];
}
template <typename KT>
void impose_dirichlet(const BcDev& bc, long long ndof, double lam, const double* U, KT* K, double* R,
                      double* dg, cudaStream_t st) {
  const int b1 = (int)std::min<long long>((ndof + 255) / 256, 4096);
  pfem::count_launch(); residual_fext_kernel<<<b1, 256, 0, st>>>(ndof, lam, bc.fn, R);
  if (bc.nbc == 0) return;
  pfem::count_launch(); bc_dg_kernel<<<(bc.nbc + 255) / 256, 256, 0, st>>>(bc.nbc, bc.dofs, bc.vals, bc.ramp, lam, U, dg);
  if (bc.nrows > 0) {  // none when every dof is constrained
    pfem::count_launch();
    bc_rhs_kernel<KT><<<(bc.nrows + 127) / 128, 128, 0, st>>>(bc.nrows, bc.rows, bc.rptr, bc.rpos, bc.rcol, K, dg, R);
  }
  if (bc.nzero > 0) {
    const int b2 = (int)std::min<long long>((bc.nzero + 255) / 256, 4096);
    pfem::count_launch(); bc_zero_kernel<KT><<<b2, 256, 0, st>>>(bc.nzero, bc.zpos, bc.zone, K);
  }
  pfem::count_launch(); bc_set_kernel<<<(bc.nbc + 255) / 256, 256, 0, st>>>(bc.nbc, bc.dofs, dg, R);
}
// Set U[d] = g(lambda) on constrained dofs (predictors honour the BCs).
__global__ void bc_apply_kernel(int nbc, const int* __restrict__ dofs, const double* __restrict__ vals,
                                const uint8_t* __restrict__ ramp, double lam, double* __restrict__ U) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nbc) return;
  U[dofs[i]] = ramp[i] ? lam * vals[i] : vals[i];
}
void bc_apply(const BcDev& bc, double lam, double* U, cudaStream_t st) {
  if (bc.nbc > 0) { pfem::count_launch(); bc_apply_kernel<<<(bc.nbc + 255) / 256, 256, 0, st>>>(bc.nbc, bc.dofs, bc.vals, bc.ramp, lam, U); }
}

// ------------------------------------------------------------------ coarse solve
// Dense coarse solve y = Ainv b (one warp per row).
template <typename T>
__global__ void dense_mv_kernel(int n, const T* __restrict__ M, const T* __restrict__ b, T* __restrict__ y) {
  const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  T s = T(0);
  for (int j = lane; j < n; j += 32) s += M[(long long)row * n + j] * b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[row] = s;
}
template <typename T>
void dense_mv(int n, const T* M, const T* b, T* y, cudaStream_t st) {
  const int blocks = (int)(((long long)n * 32 + 255) / 256);
  pfem::count_launch(); dense_mv_kernel<T><<<blocks, 256, 0, st>>>(n, M, b, y);
}

// ------------------------------------------------------------------ smoothed aggregation
// P = (I - w D^-1 A) T with the tentative T (one bs x 6 block per fine row).
// One thread per P block p (row n, aggregate J):
//   P_p = [J == agg(n)] T_n - w Dinv_n sum_{k in row n, agg(col k) == J} A_k T_col(k)
// pslot[k] names the P block that A block k feeds.
template <typename T, int BS>
__global__ void sa_prolongator_kernel(int nnzP, const int* __restrict__ p_row, const int* __restrict__ p_cl,
                                      const int* __restrict__ rowptr, const int* __restrict__ col,
                                      const T* __restrict__ val, const int* __restrict__ pslot,
                                      const int* __restrict__ agg, const T* __restrict__ Tb,
                                      const T* __restrict__ dinv, T w, T* __restrict__ pval) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnzP) return;
  const int n = p_row[p];
  T acc[BS][6];
#pragma unroll
  for (int i = 0; i < BS; ++i)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[i][c] = T(0);
  for (int k = rowptr[n]; k < rowptr[n + 1]; ++k) {
    if (pslot[k] != p) continue;
    const T* A = val + (long long)k * BS * BS;
    const T* Tm = Tb + (long long)col[k] * BS * 6;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) {
        const T a = A[i * BS + j];
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[i][c] += a * Tm[j * 6 + c];
      }
  }
  const T* D = dinv + (long long)n * BS * BS;
  const bool own = p_cl[p] == agg[n];
  const T* Tn = Tb + (long long)n * BS * 6;
  T* P = pval + (long long)p * BS * 6;
#pragma unroll
  for (int i = 0; i < BS; ++i)
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      T s = T(0);
#pragma unroll
      for (int j = 0; j < BS; ++j) s += D[i * BS + j] * acc[j][c];
      P[i * 6 + c] = (own ? Tn[i * 6 + c] : T(0)) - w * s;
    }
}

__device__ __forceinline__ int find_sorted(const int* __restrict__ a, int lo, int hi, int key) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const int v = a[mid];
    if (v == key) return mid;
    if (v < key) lo = mid + 1; else hi = mid;
  }
  return -1;
}

// AP block q (row n, coarse column J) = sum_{k in row n} A_k P[col k, J].
template <typename T, int BS>
__global__ void sa_ap_kernel(int nnzAP, const int* __restrict__ ap_row, const int* __restrict__ ap_cl,
                             const int* __restrict__ rowptr, const int* __restrict__ col,
                             const T* __restrict__ val, const int* __restrict__ p_rp,
                             const int* __restrict__ p_cl, const T* __restrict__ pval, T* __restrict__ apval) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnzAP) return;
  const int n = ap_row[q], J = ap_cl[q];
  T acc[BS][6];
#pragma unroll
  for (int i = 0; i < BS; ++i)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[i][c] = T(0);
  for (int k = rowptr[n]; k < rowptr[n + 1]; ++k) {
    const int m = col[k];
    const int p = find_sorted(p_cl, p_rp[m], p_rp[m + 1], J);
    if (p < 0) continue;
    const T* A = val + (long long)k * BS * BS;
    const T* P = pval + (long long)p * BS * 6;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) {
        const T a = A[i * BS + j];
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[i][c] += a * P[j * 6 + c];
      }
  }
  T* O = apval + (long long)q * BS * 6;
#pragma unroll
  for (int i = 0; i < BS; ++i)
#pragma unroll
    for (int c = 0; c < 6; ++c) O[i * 6 + c] = acc[i][c];
}

// Coarse block c (I, J) = sum_{p in P^T row I} P_p^T AP[row(p), J]   (6 x 6)
template <typename T, int BS>
__global__ void sa_rap_kernel(int nnzC, const int* __restrict__ c_row, const int* __restrict__ c_cl,
                              const int* __restrict__ pt_rp, const int* __restrict__ pt_blk,
                              const int* __restrict__ p_row, const T* __restrict__ pval,
                              const int* __restrict__ ap_rp, const int* __restrict__ ap_cl,
                              const T* __restrict__ apval, T* __restrict__ cval) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nnzC) return;
  const int I = c_row[c], J = c_cl[c];
  T acc[6][6];
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[r][q] = T(0);
  for (int t = pt_rp[I]; t < pt_rp[I + 1]; ++t) {
    const int p = pt_blk[t];
    const int n = p_row[p];
    const int q = find_sorted(ap_cl, ap_rp[n], ap_rp[n + 1], J);
    if (q < 0) continue;
    const T* P = pval + (long long)p * BS * 6;
    const T* AP = apval + (long long)q * BS * 6;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        const T pr = P[i * 6 + r];
#pragma unroll
        for (int q2 = 0; q2 < 6; ++q2) acc[r][q2] += pr * AP[i * 6 + q2];
      }
  }
  T* O = cval + (long long)c * 36;
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int q = 0; q < 6; ++q) O[r * 6 + q] = acc[r][q];
}

// P^T copy: block t of the aggregate-ordered list is P block pt_blk[t].
template <typename T, int BS>
__global__ void sa_transpose_copy_kernel(int nnzP, const int* __restrict__ pt_blk, const T* __restrict__ pval,
                                         T* __restrict__ ptval) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)nnzP * BS * 6) return;
  const long long t = e / (BS * 6);
  const int q = (int)(e - t * (BS * 6));
  ptval[e] = pval[(long long)pt_blk[t] * (BS * 6) + q];
}

// Six consecutive values from an address that is 8-byte aligned (float) or
// 16-byte aligned (double), as three 8- or 16-byte loads: every 6-value row of a
// bs x 6 transfer block and every 6-vector of a coarse level is.
template <typename T, bool STREAM>
__device__ __forceinline__ void load6(const T* __restrict__ p, T* v) {
  using V2 = typename std::conditional<std::is_same<T, float>::value, float2, double2>::type;
  const V2* q = reinterpret_cast<const V2*>(p);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const V2 w = STREAM ? __ldcs(q + k) : __ldg(q + k);
    v[2 * k] = w.x;
    v[2 * k + 1] = w.y;
  }
}

// Restriction bc = P^T r, WPA warps per aggregate: the lanes stride over the
// aggregate's P blocks in the P^T-ordered copy (consecutive lanes read
// consecutive blocks), each warp combines its six partial sums by a fixed xor
// tree and the WPA warp sums are added in warp order, so the result is
// deterministic.  Coarse levels have few aggregates of many blocks each; there
// WPA = 4 spreads an aggregate over 128 lanes.
template <typename T, int BS, int WPA>
__global__ void __launch_bounds__(256) sa_restrict_kernel(int nagg, const int* __restrict__ pt_rp,
                                                          const int* __restrict__ pt_row,
                                                          const T* __restrict__ ptval, const T* __restrict__ r,
                                                          T* __restrict__ bc) {
  __shared__ T part[8][6];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * (8 / WPA) + wid / WPA;
  const int w = wid % WPA;
  T s[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  if (I < nagg) {
    const int t1 = pt_rp[I + 1];
    for (int t = pt_rp[I] + w * 32 + lane; t < t1; t += 32 * WPA) {
      const T* P = ptval + (long long)t * BS * 6;
      const T* rv = r + (long long)pt_row[t] * BS;
#pragma unroll
      for (int j = 0; j < BS; ++j) {
        const T rj = rv[j];
        T pv[6];
        load6<T, false>(P + j * 6, pv);
#pragma unroll
        for (int c = 0; c < 6; ++c) s[c] += pv[c] * rj;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_xor_sync(0xffffffffu, s[c], o);
  T out = s[0];
#pragma unroll
  for (int c = 1; c < 6; ++c)
    if (lane == c) out = s[c];
  if constexpr (WPA == 1) {
    if (I < nagg && lane < 6) bc[(long long)I * 6 + lane] = out;
  } else {
    if (lane < 6) part[wid][lane] = out;
    __syncthreads();
    if (w == 0 && I < nagg && lane < 6) {
      T v = part[wid][lane];
#pragma unroll
      for (int q = 1; q < WPA; ++q) v += part[wid + q][lane];
      bc[(long long)I * 6 + lane] = v;
    }
  }
}
// Prolongation x[n*BS+j] += sum_{p in P row n} (P_p xc[col(p)])_j
// (TWO: x += P (xc + xc2), the two corrections of a W-cycle visit).
template <typename T, int BS, bool TWO = false>
__global__ void sa_prolong_kernel(int nbrow, const int* __restrict__ p_rp, const int* __restrict__ p_cl,
                                  const T* __restrict__ pval, const T* __restrict__ xc, const T* __restrict__ xc2,
                                  T* __restrict__ x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)nbrow * BS) return;
  const int n = (int)(i / BS), j = (int)(i % BS);
  T s = T(0);
  for (int p = p_rp[n]; p < p_rp[n + 1]; ++p) {
    const T* P = pval + (long long)p * BS * 6 + j * 6;
    const long long a = (long long)p_cl[p] * 6;
    T pv[6], xv[6];
    load6<T, true>(P, pv);
    load6<T, false>(xc + a, xv);
    if (TWO) {
      T x2v[6];
      load6<T, false>(xc2 + a, x2v);
#pragma unroll
      for (int c = 0; c < 6; ++c) xv[c] += x2v[c];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) s += pv[c] * xv[c];
  }
  x[i] += s;
}

template <typename T>
void sa_setup_level(const AmgLevel<T>& v, T w, T* cval, int nnzC, cudaStream_t st) {
  const int BSs = v.A.bs;
  if (BSs == 3) {
    pfem::count_launch();
    sa_prolongator_kernel<T, 3><<<(v.nnzP + 127) / 128, 128, 0, st>>>(v.nnzP, v.p_row, v.p_cl, v.A.rowptr, v.A.col,
                                                                     v.A.val, v.pslot, v.agg, v.T, v.dinv, w, v.p_val);
    pfem::count_launch();
    sa_ap_kernel<T, 3><<<(v.nnzAP + 127) / 128, 128, 0, st>>>(v.nnzAP, v.ap_row, v.ap_cl, v.A.rowptr, v.A.col, v.A.val,
                                                             v.p_rp, v.p_cl, v.p_val, v.ap_val);
    pfem::count_launch();
    sa_rap_kernel<T, 3><<<(nnzC + 127) / 128, 128, 0, st>>>(nnzC, v.c_row, v.c_cl, v.pt_rp, v.pt_blk, v.p_row, v.p_val,
                                                           v.ap_rp, v.ap_cl, v.ap_val, cval);
    pfem::count_launch();
    sa_transpose_copy_kernel<T, 3><<<(int)(((long long)v.nnzP * 18 + 255) / 256), 256, 0, st>>>(v.nnzP, v.pt_blk,
                                                                                               v.p_val, v.pt_val);
  } else {
    pfem::count_launch();
    sa_prolongator_kernel<T, 6><<<(v.nnzP + 127) / 128, 128, 0, st>>>(v.nnzP, v.p_row, v.p_cl, v.A.rowptr, v.A.col,
                                                                     v.A.val, v.pslot, v.agg, v.T, v.dinv, w, v.p_val);
    pfem::count_launch();
    sa_ap_kernel<T, 6><<<(v.nnzAP + 127) / 128, 128, 0, st>>>(v.nnzAP, v.ap_row, v.ap_cl, v.A.rowptr, v.A.col, v.A.val,
                                                             v.p_rp, v.p_cl, v.p_val, v.ap_val);
    pfem::count_launch();
    sa_rap_kernel<T, 6><<<(nnzC + 127) / 128, 128, 0, st>>>(nnzC, v.c_row, v.c_cl, v.pt_rp, v.pt_blk, v.p_row, v.p_val,
                                                           v.ap_rp, v.ap_cl, v.ap_val, cval);
    pfem::count_launch();
    sa_transpose_copy_kernel<T, 6><<<(int)(((long long)v.nnzP * 36 + 255) / 256), 256, 0, st>>>(v.nnzP, v.pt_blk,
                                                                                               v.p_val, v.pt_val);
  }
}
// Aggregates below this count get four warps each in the restriction.
constexpr int kRestrictWideBelow = 4096;

template <typename T>
void sa_restrict(const AmgLevel<T>& v, const T* r, T* bc, cudaStream_t st) {
  const bool wide = v.nagg < kRestrictWideBelow;
  const long long warps = (long long)v.nagg * (wide ? 4 : 1);
  const int blocks = (int)((warps + 7) / 8);
  pfem::count_launch();
  if (v.A.bs == 3) {
    if (wide) sa_restrict_kernel<T, 3, 4><<<blocks, 256, 0, st>>>(v.nagg, v.pt_rp, v.pt_row, v.pt_val, r, bc);
    else sa_restrict_kernel<T, 3, 1><<<blocks, 256, 0, st>>>(v.nagg, v.pt_rp, v.pt_row, v.pt_val, r, bc);
  } else {
    if (wide) sa_restrict_kernel<T, 6, 4><<<blocks, 256, 0, st>>>(v.nagg, v.pt_rp, v.pt_row, v.pt_val, r, bc);
    else sa_restrict_kernel<T, 6, 1><<<blocks, 256, 0, st>>>(v.nagg, v.pt_rp, v.pt_row, v.pt_val, r, bc);
  }
}
template <typename T>
static void prolong_launch(const AmgLevel<T>& v, const T* xc, const T* xc2, T* x, cudaStream_t st) {
  const long long n = (long long)v.A.nbrow * v.A.bs;
  const int blocks = (int)((n + 255) / 256);
  pfem::count_launch();
  if (v.A.bs == 3) {
    if (xc2) sa_prolong_kernel<T, 3, true><<<blocks, 256, 0, st>>>(v.A.nbrow, v.p_rp, v.p_cl, v.p_val, xc, xc2, x);
    else sa_prolong_kernel<T, 3><<<blocks, 256, 0, st>>>(v.A.nbrow, v.p_rp, v.p_cl, v.p_val, xc, xc, x);
  } else {
    if (xc2) sa_prolong_kernel<T, 6, true><<<blocks, 256, 0, st>>>(v.A.nbrow, v.p_rp, v.p_cl, v.p_val, xc, xc2, x);
    else sa_prolong_kernel<T, 6><<<blocks, 256, 0, st>>>(v.A.nbrow, v.p_rp, v.p_cl, v.p_val, xc, xc, x);
  }
}
template <typename T>
void sa_prolong(const AmgLevel<T>& v, const T* xc, T* x, cudaStream_t st) {
  prolong_launch<T>(v, xc, nullptr, x, st);
}
template <typename T>
void sa_prolong2(const AmgLevel<T>& v, const T* xc, const T* xc2, T* x, cudaStream_t st) {
  prolong_launch<T>(v, xc, xc2, x, st);
}

// ------------------------------------------------------------------ instantiations
#define PFEM_INST(T)                                                                               \
  template void bsr_spmv<T>(const BsrMat<T>&, const T*, T*, cudaStream_t);                         \
  template void bsr_residual<T>(const BsrMat<T>&, const T*, const T*, T*, cudaStream_t);           \
  template void bsr_cheb_step<T>(const BsrMat<T>&, const T*, const T*, T*, T*, cudaStream_t);      \
  template void bsr_cheb2<T>(const BsrMat<T>&, const T*, const T*, const T*, T*, bool, T, T, cudaStream_t); \
  template void bsr_residual_precond<T>(const BsrMat<T>&, const T*, const T*, const T*, T*, T*, T,    \
                                        cudaStream_t);                                             \
  template void blockdiag_apply<T>(int, int, const T*, const T*, T*, T, T*, cudaStream_t);         \
  template void blockdiag_invert<T>(const BsrMat<T>&, T*, cudaStream_t);                           \
  template void dot<T>(long long, const T*, const T*, T*, T*, cudaStream_t, bool);                 \
  template void fill<T>(long long, T*, T, cudaStream_t);                                           \
  template void axpby<T>(long long, T, const T*, T, T*, cudaStream_t);                             \
  template void cg_xr<T>(long long, const T*, const T*, const T*, const T*, T*, T*, cudaStream_t); \
  template void cg_p<T>(long long, const T*, const T*, const T*, T*, cudaStream_t);                \
  template void bicg_p<T>(long long, const T*, const T*, const T*, T*, cudaStream_t);              \
  template void bicg_s<T>(long long, const T*, const T*, const T*, T*, cudaStream_t);              \
  template void bicg_xr<T>(long long, const T*, const T*, const T*, const T*, const T*, T*, T*,    \
                           cudaStream_t);                                                          \
  template void scalar_copy<T>(T*, const T*, cudaStream_t);                                        \
  template int dot_partials<T>(long long, const T*, const T*, T*, cudaStream_t);                   \
  template void cg_p_fused<T>(long long, const T*, int, T*, const T*, T*, cudaStream_t);           \
  template int cg_xr_fused<T>(long long, const T*, int, T*, const T*, const T*, T*, T*, T*,         \
                              cudaStream_t);                                                       \
  template void add_to_double<T>(long long, const T*, double*, cudaStream_t);                      \
  template void impose_dirichlet<T>(const BcDev&, long long, double, const double*, T*, double*,   \
                                    double*, cudaStream_t);                                        \
  template void dense_mv<T>(int, const T*, const T*, T*, cudaStream_t);                            \
  template void sa_setup_level<T>(const AmgLevel<T>&, T, T*, int, cudaStream_t);                   \
  template void sa_restrict<T>(const AmgLevel<T>&, const T*, T*, cudaStream_t);                    \
  template void sa_prolong<T>(const AmgLevel<T>&, const T*, T*, cudaStream_t);                     \
  template void sa_prolong2<T>(const AmgLevel<T>&, const T*, const T*, T*, cudaStream_t);
PFEM_INST(float)
PFEM_INST(double)
template void convert<double, float>(long long, const double*, float*, double, cudaStream_t);
template void convert<float, double>(long long, const float*, double*, double, cudaStream_t);
template void convert<double, double>(long long, const double*, double*, double, cudaStream_t);

}  // namespace pfem
