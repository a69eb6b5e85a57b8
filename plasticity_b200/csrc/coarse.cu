// coarse.cu -- the bottom of the AMG cycle in one launch.
//
// Below level 1 the hierarchy's levels are small (at 64^3: level 2 has 512 block
// rows of 6 x 6 blocks, 1.7 MB, and the dense level 162 unknowns), and a visit to
// the last non-dense level is eight latency-bound kernels of a few microseconds
// each: block-Jacobi start, fused Chebyshev step, residual, restriction, dense
// product, prolongation, preconditioned residual, fused Chebyshev step.  A
// W-cycle makes two such visits (the second from the coarse residual).  Here one
// thread-block cluster runs all of them as phases separated by cluster barriers
// (hardware barriers: no flag polling), with every vector in L2.  The arithmetic
// of each phase, and the order of every sum, is that of the standalone kernels in
// linalg.cu, so the cycle is the same operator.
#include <cooperative_groups.h>

#include <type_traits>

#include "linalg.cuh"

namespace cg = cooperative_groups;

namespace pfem {

namespace {

constexpr int kTailCtas = 8;        // portable cluster size
constexpr int kTailThreads = 1024;  // per CTA
constexpr int kTailWarps = kTailCtas * kTailThreads / 32;

template <typename T>
struct TailArgs {
  int nbrow;  // block rows of the level (6 x 6 blocks)
  const int* rowptr;
  const int* col;
  const T* val;
  const T* dinv;
  T inv_th, c1, c2;  // degree-2 Chebyshev coefficients of the level
  int nagg;          // aggregates = dense level block rows
  const int* pt_rp;
  const int* pt_row;
  const T* pt_val;
  const int* p_rp;
  const int* p_cl;
  const T* p_val;
  int nc;  // dense level unknowns
  const T* cinv;
  const T* b;
  T* x;
  T* b2;
  T* x2;
  T *r, *d, *t, *cb, *cx;
  int twice;
};

// Block-Jacobi start of a zero-guess Chebyshev smoothing: r = Dinv b, d = r / th
// (blockdiag_apply_kernel).
template <typename T>
__device__ void tail_blockdiag(const TailArgs<T>& a, const T* __restrict__ b, int gt, int gn) {
  const int n = a.nbrow * 6;
  for (int i = gt; i < n; i += gn) {
    const int row = i / 6, j = i - row * 6;
    const T* D = a.dinv + (long long)row * 36 + j * 6;
    const T* bb = b + (long long)row * 6;
    T s = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) s += D[k] * bb[k];
    a.r[i] = s;
    a.d[i] = a.inv_th * s;
  }
}

// One pass over the level's matrix, half a warp per block row, with the
// epilogues of bsr_spmv_kernel<T, 6, MODE, true>:
//   1: y = b - A x;  3: xo = c2 x + c1 (y - Dinv A x);  4: as 3, added to xo;
//   5: y = Dinv (b - A x), xo = c1 y.
template <typename T, int MODE>
__device__ void tail_spmv(const TailArgs<T>& a, const T* __restrict__ x, T* __restrict__ y,
                          const T* __restrict__ b, T* __restrict__ xo, T c1, T c2, int gw, int lane32) {
  using V = typename std::conditional<std::is_same<T, float>::value, float4, double2>::type;
  constexpr int PER = 16 / (int)sizeof(T), NV = 36 / PER;
  const int half = lane32 >> 4, lane = lane32 & 15;
  // each warp takes two rows per round; the round count is uniform over the warp
  for (int r0 = 2 * gw; r0 < a.nbrow; r0 += 2 * kTailWarps) {
    const int row = r0 + half;
    const bool ok = row < a.nbrow;
    const int s = ok ? a.rowptr[row] : 0, e = ok ? a.rowptr[row + 1] : 0;
    T acc[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) acc[i] = T(0);
    for (int k = s + lane; k < e; k += 16) {
      const int c = __ldcs(a.col + k);
      const V* B4 = reinterpret_cast<const V*>(a.val + (long long)k * 36);
      T bv[36];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const V v = __ldcs(B4 + q);
        const T* vt = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int j = 0; j < PER; ++j) bv[q * PER + j] = vt[j];
      }
      T xv[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) xv[j] = x[(long long)c * 6 + j];
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) acc[i] += bv[i * 6 + j] * xv[j];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      T v = acc[i];
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[i] = v;
    }
    if (ok && lane < 6) {
      const long long base = (long long)row * 6;
      const T* D = a.dinv + (long long)row * 36;
      if (MODE == 5) {
        T t = T(0);
#pragma unroll
        for (int j = 0; j < 6; ++j) t += D[lane * 6 + j] * (b[base + j] - acc[j]);
        y[base + lane] = t;
        xo[base + lane] = c1 * t;
      } else {
        T v = acc[0];
#pragma unroll
        for (int i = 1; i < 6; ++i)
          if (lane == i) v = acc[i];
        if (MODE == 1) {
          y[base + lane] = b[base + lane] - v;
        } else {
          T t = T(0);
#pragma unroll
          for (int j = 0; j < 6; ++j) t += D[lane * 6 + j] * acc[j];
          const T upd = c2 * x[base + lane] + c1 * (y[base + lane] - t);
          if (MODE == 3) xo[base + lane] = upd;
          else xo[base + lane] += upd;
        }
      }
    }
  }
}

// Restriction cb = P^T t: aggregates are dealt to the cluster's CTAs, and all 32
// warps of a CTA share one aggregate (lanes stride over its P^T blocks), each warp
// reduces by the xor tree and the warp sums are added in warp order.
template <typename T>
__device__ void tail_restrict(const TailArgs<T>& a, T (*part)[6], int cta) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int I = cta; I < a.nagg; I += kTailCtas) {
    T s[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    const int t1 = a.pt_rp[I + 1];
    for (int t = a.pt_rp[I] + threadIdx.x; t < t1; t += kTailThreads) {
      const T* P = a.pt_val + (long long)t * 36;
      const T* rv = a.t + (long long)a.pt_row[t] * 6;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const T rj = rv[j];
#pragma unroll
        for (int c = 0; c < 6; ++c) s[c] += __ldg(P + j * 6 + c) * rj;
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
    if (lane < 6) part[wid][lane] = out;
    __syncthreads();
    if (threadIdx.x < 6) {
      T v = part[0][threadIdx.x];
      for (int q = 1; q < kTailThreads / 32; ++q) v += part[q][threadIdx.x];
      a.cb[(long long)I * 6 + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// cx = Cinv cb, a warp per row (dense_mv_kernel).
template <typename T>
__device__ void tail_dense(const TailArgs<T>& a, int gw, int lane) {
  for (int row = gw; row < a.nc; row += kTailWarps) {
    T s = T(0);
    for (int j = lane; j < a.nc; j += 32) s += a.cinv[(long long)row * a.nc + j] * a.cb[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) a.cx[row] = s;
  }
}

// x += P cx, a thread per unknown (sa_prolong_kernel).
template <typename T>
__device__ void tail_prolong(const TailArgs<T>& a, T* __restrict__ x, int gt, int gn) {
  const int n = a.nbrow * 6;
  for (int i = gt; i < n; i += gn) {
    const int row = i / 6, j = i - row * 6;
    T s = T(0);
    for (int p = a.p_rp[row]; p < a.p_rp[row + 1]; ++p) {
      const T* P = a.p_val + (long long)p * 36 + j * 6;
      const T* xa = a.cx + (long long)a.p_cl[p] * 6;
#pragma unroll
      for (int c = 0; c < 6; ++c) s += __ldcs(P + c) * xa[c];
    }
    x[i] += s;
  }
}

// One V visit to the level with right-hand side b, result x (zero start).
template <typename T>
__device__ void tail_visit(const TailArgs<T>& a, const T* b, T* x, T (*part)[6], int cta, int gt, int gn, int gw,
                           int lane) {
  cg::cluster_group cl = cg::this_cluster();
  tail_blockdiag<T>(a, b, gt, gn);
  cl.sync();
  tail_spmv<T, 3>(a, a.d, a.r, nullptr, x, a.c1, a.c2, gw, lane);  // x = c2 d + c1 (r - Dinv A d)
  cl.sync();
  tail_spmv<T, 1>(a, x, a.t, b, nullptr, T(0), T(0), gw, lane);  // t = b - A x
  cl.sync();
  tail_restrict<T>(a, part, cta);
  cl.sync();
  tail_dense<T>(a, gw, lane);
  cl.sync();
  tail_prolong<T>(a, x, gt, gn);
  cl.sync();
  tail_spmv<T, 5>(a, x, a.r, b, a.d, a.inv_th, T(0), gw, lane);  // r = Dinv (b - A x), d = r / th
  cl.sync();
  tail_spmv<T, 4>(a, a.d, a.r, nullptr, x, a.c1, a.c2, gw, lane);  // x += c2 d + c1 (r - Dinv A d)
}

template <typename T>
__global__ void __cluster_dims__(kTailCtas, 1, 1) __launch_bounds__(kTailThreads, 1)
    coarse_tail_kernel(const TailArgs<T> a) {
  __shared__ T part[kTailThreads / 32][6];
  cg::cluster_group cl = cg::this_cluster();
  const int cta = (int)cl.block_rank();
  const int gt = cta * kTailThreads + threadIdx.x, gn = kTailCtas * kTailThreads;
  const int gw = gt >> 5, lane = threadIdx.x & 31;
  tail_visit<T>(a, a.b, a.x, part, cta, gt, gn, gw, lane);
  if (a.twice) {
    // W: the second iteration on this level starts from its residual b - A x
    cl.sync();
    tail_spmv<T, 1>(a, a.x, a.b2, a.b, nullptr, T(0), T(0), gw, lane);
    cl.sync();
    tail_visit<T>(a, a.b2, a.x2, part, cta, gt, gn, gw, lane);
  }
}

}  // namespace

template <typename T>
void coarse_tail(const AmgLevel<T>& v, int nc, const T* cinv, T* cb, T* cx, const T* b, T* x, bool twice,
                 T inv_th, T c1, T c2, cudaStream_t st) {
  TailArgs<T> a;
  a.nbrow = v.A.nbrow;
  a.rowptr = v.A.rowptr;
  a.col = v.A.col;
  a.val = v.A.val;
  a.dinv = v.dinv;
  a.inv_th = inv_th;
  a.c1 = c1;
  a.c2 = c2;
  a.nagg = v.nagg;
  a.pt_rp = v.pt_rp;
  a.pt_row = v.pt_row;
  a.pt_val = v.pt_val;
  a.p_rp = v.p_rp;
  a.p_cl = v.p_cl;
  a.p_val = v.p_val;
  a.nc = nc;
  a.cinv = cinv;
  a.b = b;
  a.x = x;
  a.b2 = v.b2;
  a.x2 = v.x2;
  a.r = v.r;
  a.d = v.d;
  a.t = v.t;
  a.cb = cb;
  a.cx = cx;
  a.twice = twice ? 1 : 0;
  pfem::count_launch();
  coarse_tail_kernel<T><<<kTailCtas, kTailThreads, 0, st>>>(a);
}

template void coarse_tail<float>(const AmgLevel<float>&, int, const float*, float*, float*, const float*, float*,
                                 bool, float, float, float, cudaStream_t);
template void coarse_tail<double>(const AmgLevel<double>&, int, const double*, double*, double*, const double*,
                                  double*, bool, double, double, double, cudaStream_t);

}  // namespace pfem
