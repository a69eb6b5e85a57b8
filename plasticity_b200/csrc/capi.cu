// capi.cu -- the extern "C" boundary (include/pfem_b200.h): context set-up,
// host-side one-time topology work, the device Newton load loop, the Krylov
// solvers and the aggregation AMG they use.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "linalg.cuh"
#include "mlp.cuh"

using namespace pfem;

static thread_local std::string g_cuda_err;
static long long g_launches = 0;
long long& pfem::launch_counter() { return g_launches; }
void pfem::set_last_error(const std::string& msg) { g_cuda_err = msg; }
void pfem_set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what,
           file, line);
  g_cuda_err = buf;
}

namespace {

template <typename T>
struct KrylovWork {
  long long n = 0;
  T *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
  T *rh = nullptr, *v = nullptr, *s = nullptr, *t = nullptr, *ph = nullptr, *sh = nullptr;
  T* sc = nullptr;    // device scalars
  T* part = nullptr;  // reduction partials
  T* b = nullptr;
  T *xa = nullptr, *b0 = nullptr;  // iterative refinement: accumulated solution, saved right-hand side
};

// The preconditioned-CG loop captured as one CUDA graph: a prefix (x = 0,
// r = b, |b|) and a conditional WHILE node whose body is one iteration
// (V-cycle, two dot products, the p / x / r updates, |r|) ending in a
// one-thread kernel that sets the loop condition from the device-resident
// residual.  One launch and one host synchronisation per linear solve.
// Re-captured when the AMG hierarchy is rebuilt (its Chebyshev coefficients
// are kernel arguments); the tolerance and iteration cap are read from ctl.
struct CgGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t body_stream = nullptr;
  long long amg_version = -1;
  double* ctl = nullptr;   // device: [0] rtol, [1] itmax, [2] absolute threshold (set on the device)
  int* state = nullptr;    // device: [0] iterations, [1] converged
  long long prefix_kernels = 0, body_kernels = 0;
};

struct HostLevel {
  int nbrow = 0, bs = 0;
  std::vector<int> rowptr, col;   // matrix pattern of this level
  std::vector<int> grp, gcl;      // graph the aggregates are grown on
  int nagg = 0;
  std::vector<int> agg;
  std::vector<double> T;          // nbrow*bs*6 tentative prolongator blocks
  std::vector<int> p_rp, p_cl, p_row, pslot, pt_rp, pt_blk;  // smoothed P pattern
  std::vector<int> ap_rp, ap_cl, ap_row;                      // A P pattern
  std::vector<int> c_row;         // row of every block of the next level's pattern
};

}  // namespace

struct pfem_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  long long nn = 0, ne = 0, ngp = 0, ndof = 0;
  int kind = PFEM_HEX8_FINITE_FBAR;
  MatParams mat{};
  std::string err;
  std::vector<void*> allocs;
  std::vector<int> bc_dofs;    // deduplicated Dirichlet dofs of the last pfem_set_bcs
  std::vector<int64_t> neu_dofs_last;  // the Neumann arrays of the last pfem_set_bcs, as given
  std::vector<double> neu_vals_last;

  // host topology
  std::vector<double> X;        // nn*3
  std::vector<int> elem;        // ne*8, 0-based
  std::vector<int> browptr, bcol;
  long long nnzb = 0;
  int ncolors_ref = 0;
  std::vector<int64_t> color_ref;
  std::vector<int> color_ptr;   // device coloring, CSR over colors
  // device topology / state
  double* dX = nullptr;
  int* dElem = nullptr;
  uint8_t* dRank = nullptr;
  int* dBrowptr = nullptr;
  int* dBcol = nullptr;
  int16_t* dBcol16 = nullptr;  // dBcol as offsets from the row, when all fit in 16 bits
  double* dSigy = nullptr;
  int* dColorList = nullptr;
  int* dAllElems = nullptr;
  double *dCpi = nullptr, *dAlpha = nullptr, *dEpsp = nullptr, *dTau = nullptr;
  double* dBeta = nullptr;  // 6 x ngp committed back stress, kinematic hardening only
  double* dOut = nullptr;   // 6 x ngp scratch for per-GP results in the caller's layout (lazy)
  int hard = HARD_LINEAR;   // hardening law of the element kernels
  uint8_t* dFlags = nullptr;
  double *dU = nullptr, *dR = nullptr, *dDg = nullptr, *dUprev = nullptr, *dUprev2 = nullptr;
  double* dUprev3 = nullptr;
  double bbox_lo[3] = {0, 0, 0}, bbox_ext[3] = {1, 1, 1};
  double *dUtmp = nullptr, *dScal = nullptr, *dPart = nullptr;
  double* dK64 = nullptr;
  float* dK32 = nullptr;
  double* dDenseWork = nullptr;  // FP64 work matrix of the coarse dense inverse (both precisions)
  // gathered assembly: node -> incident elements (increasing), the node's position
  // in each, the longest block row, element-ordered tangents and forces (lazy)
  int *dNptr = nullptr, *dNel = nullptr;
  uint8_t* dNloc = nullptr;
  int max_row = 0;
  bool colored_assembly = false;
  float* dKbuf32 = nullptr;
  double* dKbuf64 = nullptr;
  double* dFbuf = nullptr;
  DevStatus* dStatus = nullptr;
  // boundary conditions
  bool bcs_set = false;
  BcDev bc;
  double fn_norm = 0.0;
  // solver
  std::vector<HostLevel> hl;
  bool amg_struct = false;
  Amg<float> amg32;
  Amg<double> amg64;
  KrylovWork<float> kw32;
  KrylovWork<double> kw64;
  CgGraph cg32, cg64;
  int tangent_prec = -1;  // precision of the last imposed tangent
  cudaEvent_t e0 = nullptr, e1 = nullptr, t0 = nullptr, t1 = nullptr;
  // learned predictor
  pfem::MlpState mlp;
  int steps_taken = 0;
  // adaptive AMG reuse (amg_rebuild = 2): Krylov iterations per decade of the
  // first solve after the last rebuild, and whether a later solve exceeded it
  double amg_ipd_base = -1.0;
  bool amg_stale = true;
  double amg_excess = 0.0;      // Krylov iterations above the fresh rate since the last rebuild
  double amg_cost_iters = 0.0;  // what a rebuild costs, in Krylov iterations
  double lam_prev = 0.0, lam_prev2 = 0.0, lam_prev3 = 0.0;
};

namespace {

int fail(pfem_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}
int cuda_fail(pfem_ctx* c) {
  if (c) c->err = g_cuda_err;
  return PFEM_ERR_CUDA;
}
#define CK(expr)                                              \
  do {                                                        \
    cudaError_t e__ = (expr);                                 \
    if (e__ != cudaSuccess) {                                 \
      pfem_set_cuda_error(e__, #expr, __FILE__, __LINE__);    \
      return cuda_fail(ctx);                                  \
    }                                                         \
  } while (0)
#define CKL()                                                 \
  do {                                                        \
    cudaError_t e__ = cudaGetLastError();                     \
    if (e__ != cudaSuccess) {                                 \
      pfem_set_cuda_error(e__, "kernel launch", __FILE__, __LINE__); \
      return cuda_fail(ctx);                                  \
    }                                                         \
  } while (0)

template <typename T>
cudaError_t dalloc(pfem_ctx* ctx, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e == cudaSuccess) ctx->allocs.push_back((void*)*p);
  return e;
}
// Host transfers of the API run on the library's stream, which is non-blocking:
// a legacy-stream cudaMemcpy is not ordered with its kernels (a pageable
// host-to-device copy may still be in flight when it returns, and a
// device-to-host copy does not wait for kernels queued on the stream).
cudaError_t h2d(const pfem_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->st);
  return e == cudaSuccess ? cudaStreamSynchronize(ctx->st) : e;
}
cudaError_t d2h(const pfem_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->st);
  return e == cudaSuccess ? cudaStreamSynchronize(ctx->st) : e;
}
template <typename T>
cudaError_t upload(pfem_ctx* ctx, T** p, const std::vector<T>& h) {
  cudaError_t e = dalloc(ctx, p, h.size());
  if (e != cudaSuccess) return e;
  if (!h.empty()) e = h2d(ctx, *p, h.data(), h.size() * sizeof(T));
  return e;
}

// Free one allocation made by dalloc/upload (nullptr is a no-op).
// Device temporaries of one entry-point call, released on every return path
// (including the early returns of CK).
struct TmpDev {
  std::vector<void*> p;
  template <typename T>
  cudaError_t alloc(T** out, size_t bytes) {
    *out = nullptr;
    cudaError_t e = cudaMalloc((void**)out, bytes);
    if (e == cudaSuccess) p.push_back((void*)*out);
    return e;
  }
  ~TmpDev() {
    for (void* q : p) cudaFree(q);
  }
};

template <typename T>
void dfree(pfem_ctx* ctx, T*& p) {
  if (!p) return;
  auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), (void*)p);
  if (it != ctx->allocs.end()) ctx->allocs.erase(it);
  cudaFree((void*)p);
  p = nullptr;
}

template <class Fn>
void par_for(long long n, Fn fn) {
  const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 20000 || nt == 1) {
    for (long long i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  const long long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const long long b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([=, &fn]() {
      for (long long i = b; i < e; ++i) fn(i);
    });
  }
  for (auto& t : th) t.join();
}

// par_for over contiguous chunks: fn(begin, end) once per thread, so a thread
// can keep scratch (marker arrays) across its rows.
template <typename Fn>
void par_chunks(long long n, Fn fn) {
  const int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 20000 || nt == 1) {
    fn(0ll, n);
    return;
  }
  std::vector<std::thread> th;
  const long long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const long long b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([=, &fn]() { fn(b, e); });
  }
  for (auto& t : th) t.join();
}

// Symbolic sparse product (Gustavson): row r of the result is the sorted set
// of map(j) over j in B(k), k in A(r), with A = (arp, acl) and B = (brp, bcl);
// brp = null means B(k) = {k}; map = null is the identity.  Columns lie in
// [0, ncols).  Two passes with a per-thread marker array: counts, then fill
// and sort each (short) row.
void symbolic_product(int nrows, const int* arp, const int* acl, const int* brp, const int* bcl,
                      const int* map, int ncols, std::vector<int>& rp, std::vector<int>& cl) {
  rp.assign((size_t)nrows + 1, 0);
  auto visit = [&](int r, std::vector<int>& mark, auto&& emit) {
    for (int t = arp[r]; t < arp[r + 1]; ++t) {
      const int k = acl[t];
      const int q0 = brp ? brp[k] : 0, q1 = brp ? brp[k + 1] : 1;
      for (int q = q0; q < q1; ++q) {
        const int j0 = brp ? bcl[q] : k;
        const int j = map ? map[j0] : j0;
        if (mark[j] != r) { mark[j] = r; emit(j); }
      }
    }
  };
  par_chunks(nrows, [&](long long b, long long e) {
    std::vector<int> mark(ncols, -1);
    for (long long r = b; r < e; ++r) {
      int cnt = 0;
      visit((int)r, mark, [&](int) { ++cnt; });
      rp[r + 1] = cnt;
    }
  });
  for (int r = 0; r < nrows; ++r) rp[r + 1] += rp[r];
  cl.resize(rp[nrows]);
  par_chunks(nrows, [&](long long b, long long e) {
    std::vector<int> mark(ncols, -1);
    for (long long r = b; r < e; ++r) {
      int* o = cl.data() + rp[r];
      int n = 0;
      visit((int)r, mark, [&](int j) { o[n++] = j; });
      std::sort(o, o + n);
    }
  });
}

// element_colors reference rule (Assembly.jl:172-206): parity colors when
// the node coordinates form an axis-aligned structured box, else one color.
int reference_colors(const std::vector<double>& X, long long nn, long long ne,
                     std::vector<int64_t>& color) {
  color.assign(ne, 0);
  if (ne == 0) return 0;
  // _box_dims: distinct rounded coordinates per axis.  A box needs at least
  // two distinct values on each of the other axes, so more than nn/4 on one
  // axis already rules it out and the count stops there.
  long long dims[3];
  const long long cap = nn / 4;
  size_t tsize = 16;
  while (tsize < (size_t)(2 * cap + 2)) tsize <<= 1;
  std::vector<uint64_t> table(tsize);
  std::vector<uint8_t> used(tsize);
  for (int d = 0; d < 3; ++d) {
    // open-addressing set of the rounded values' bit patterns (-0.0 folded
    // into 0.0, so membership is numeric equality)
    std::fill(used.begin(), used.end(), 0);
    long long count = 0;
    for (long long n = 0; n < nn && count <= cap; ++n) {
      double v = std::round(X[n * 3 + d] * 1e12) / 1e12;
      if (v == 0.0) v = 0.0;
      uint64_t key;
      std::memcpy(&key, &v, sizeof(key));
      size_t h = (size_t)((key * 0x9E3779B97F4A7C15ull) >> 17) & (tsize - 1);
      while (used[h] && table[h] != key) h = (h + 1) & (tsize - 1);
      if (!used[h]) {
        used[h] = 1;
        table[h] = key;
        ++count;
      }
    }
    if (count > cap) return 1;
    dims[d] = count - 1;
  }
  const long long nx = dims[0], ny = dims[1], nz = dims[2];
  if (!(nx >= 1 && ny >= 1 && nz >= 1 && nx * ny * nz == ne && (nx + 1) * (ny + 1) * (nz + 1) == nn))
    return 1;
  int raw[8] = {0};
  std::vector<int> c8(ne);
  long long e = 0;
  for (long long k = 0; k < nz; ++k)
    for (long long j = 0; j < ny; ++j)
      for (long long i = 0; i < nx; ++i) {
        const int c = (int)((i & 1) + 2 * (j & 1) + 4 * (k & 1));
        c8[e++] = c;
        raw[c]++;
      }
  int remap[8], nc = 0;
  for (int c = 0; c < 8; ++c) remap[c] = raw[c] ? nc++ : -1;
  for (long long q = 0; q < ne; ++q) color[q] = remap[c8[q]];
  return nc;
}

// Greedy first-fit element coloring on the shared-node graph (used when the
// reference rule gives a single color, i.e. on perturbed meshes).
int greedy_colors(const std::vector<int>& elem, long long nn, long long ne, std::vector<int>& col) {
  std::vector<int> nptr(nn + 1, 0);
  for (long long e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) nptr[elem[e * 8 + a] + 1]++;
  for (long long n = 0; n < nn; ++n) nptr[n + 1] += nptr[n];
  std::vector<int> nel(nptr[nn]);
  std::vector<int> fill(nptr.begin(), nptr.end() - 1);
  for (long long e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) nel[fill[elem[e * 8 + a]]++] = (int)e;
  col.assign(ne, -1);
  int nc = 0;
  for (long long e = 0; e < ne; ++e) {
    uint64_t used = 0;
    for (int a = 0; a < 8; ++a) {
      const int n = elem[e * 8 + a];
      for (int k = nptr[n]; k < nptr[n + 1]; ++k) {
        const int o = nel[k];
        if (col[o] >= 0 && col[o] < 64) used |= (1ull << col[o]);
      }
    }
    int c = 0;
    while (c < 64 && (used >> c) & 1ull) ++c;
    col[e] = c;
    nc = std::max(nc, c + 1);
  }
  return nc;
}

// Greedy aggregation on a block graph: phase 1 roots whose neighbourhood is
// untouched, phase 2 attaches leftovers to an adjacent aggregate, phase 3
// groups whatever remains with its unaggregated neighbours.
int aggregate(int nb, const int* rp, const int* cl, std::vector<int>& agg) {
  agg.assign(nb, -1);
  int na = 0;
  for (int n = 0; n < nb; ++n) {
    if (agg[n] >= 0) continue;
    bool free_ = true;
    for (int k = rp[n]; k < rp[n + 1] && free_; ++k)
      if (agg[cl[k]] >= 0) free_ = false;
    if (!free_) continue;
    for (int k = rp[n]; k < rp[n + 1]; ++k) agg[cl[k]] = na;
    agg[n] = na;
    ++na;
  }
  std::vector<int> agg1 = agg;
  for (int n = 0; n < nb; ++n) {
    if (agg[n] >= 0) continue;
    for (int k = rp[n]; k < rp[n + 1]; ++k)
      if (agg1[cl[k]] >= 0) { agg[n] = agg1[cl[k]]; break; }
  }
  for (int n = 0; n < nb; ++n) {
    if (agg[n] >= 0) continue;
    agg[n] = na;
    for (int k = rp[n]; k < rp[n + 1]; ++k)
      if (agg[cl[k]] < 0) agg[cl[k]] = na;
    ++na;
  }
  return na;
}

// Thin QR (modified Gram-Schmidt, two passes) of an m x 6 block, row-major.
void mgs_qr(int m, std::vector<double>& A, double R[36]) {
  std::memset(R, 0, 36 * sizeof(double));
  double n0[6];
  for (int c = 0; c < 6; ++c) {
    double s = 0;
    for (int i = 0; i < m; ++i) s += A[i * 6 + c] * A[i * 6 + c];
    n0[c] = std::sqrt(s);
  }
  for (int c = 0; c < 6; ++c) {
    for (int pass = 0; pass < 2; ++pass)
      for (int k = 0; k < c; ++k) {
        double s = 0;
        for (int i = 0; i < m; ++i) s += A[i * 6 + k] * A[i * 6 + c];
        R[k * 6 + c] += s;
        for (int i = 0; i < m; ++i) A[i * 6 + c] -= s * A[i * 6 + k];
      }
    double s = 0;
    for (int i = 0; i < m; ++i) s += A[i * 6 + c] * A[i * 6 + c];
    s = std::sqrt(s);
    if (s > 1e-10 * std::max(n0[c], 1e-300)) {
      R[c * 6 + c] = s;
      for (int i = 0; i < m; ++i) A[i * 6 + c] /= s;
    } else {
      R[c * 6 + c] = 0.0;
      for (int i = 0; i < m; ++i) A[i * 6 + c] = 0.0;
    }
  }
}

// Host side of the smoothed-aggregation hierarchy (one-time, mesh-only):
// aggregates, tentative prolongators from the six rigid-body modes
// (Solver.jl:117-129), and the patterns of P = (I - w D^-1 A) T, of A P and
// of the Galerkin operator P^T A P of every level.  Level 0 uses the
// tangent's block pattern in place (its rowptr/col stay empty).
// The hierarchy stops at the first level with at most this many unknowns; that
// level is inverted densely (dense.cu on the device, or on the host when small)
// and applied as one dense matrix-vector product per cycle.  The inverse costs
// n^3 at every rebuild: at 64^3 a 3,072-unknown dense level 2 saves a W-cycle's
// two visits to it (about 100 us per cycle) but adds about 11 ms per rebuild,
// so by default the hierarchy goes one level further there (162 unknowns).
// PFEM_COARSE_DENSE_MAX overrides the bound.
constexpr long long kCoarseDenseMax = 1500;
// Coarsest levels up to this size are inverted on the host with partial pivoting
// (n^3 <= 2.7e7 multiply-adds: 1.3 ms at 162 unknowns, but 16 ms at 384); larger
// ones on the device without row exchanges (about 1.4 ms at 384), which the
// coarse operators of all but the smallest meshes (full aggregates, every rigid
// mode present) do not need.
// The adaptive AMG policy charges a rebuild this many Krylov iterations.
constexpr double kRebuildCostIters = 12.0;
constexpr int kCoarseHostMax = 300;

void build_amg_structure(pfem_ctx* c) {
  long long dense_max = kCoarseDenseMax;
  if (const char* e = getenv("PFEM_COARSE_DENSE_MAX")) dense_max = std::max(1LL, atoll(e));
  c->hl.clear();
  HostLevel cur;
  cur.nbrow = (int)c->nn;
  cur.bs = 3;
  std::vector<double> B;
  double ctr[3] = {0, 0, 0};
  for (long long n = 0; n < c->nn; ++n)
    for (int d = 0; d < 3; ++d) ctr[d] += c->X[n * 3 + d] / (double)c->nn;
  bool first = true;
  for (int lev = 0; lev < 10; ++lev) {
    const int nb = cur.nbrow, bs = cur.bs;
    if ((long long)nb * bs <= dense_max && !first) break;
    const int* rp = first ? c->browptr.data() : cur.rowptr.data();
    const int* cl = first ? c->bcol.data() : cur.col.data();
    const int* grp = first ? rp : cur.grp.data();
    const int* gcl = first ? cl : cur.gcl.data();
    cur.nagg = aggregate(nb, grp, gcl, cur.agg);
    if (cur.nagg >= nb || (long long)cur.nagg * 6 >= (long long)nb * bs) break;
    const int na = cur.nagg;
    std::vector<int> aptr(na + 1, 0), amem(nb);
    for (int n = 0; n < nb; ++n) aptr[cur.agg[n] + 1]++;
    for (int a = 0; a < na; ++a) aptr[a + 1] += aptr[a];
    {
      std::vector<int> f(aptr.begin(), aptr.end() - 1);
      for (int n = 0; n < nb; ++n) amem[f[cur.agg[n]]++] = n;
    }
    // tentative prolongator: per-aggregate QR of the near-null-space block
    cur.T.assign((size_t)nb * bs * 6, 0.0);
    std::vector<double> Bc((size_t)na * 36, 0.0);
    par_for(na, [&](long long a) {
      const int m = aptr[a + 1] - aptr[a];
      std::vector<double> M((size_t)m * bs * 6);
      if (first) {
        // One global centre for every aggregate: the six columns must be the
        // same six rigid-body modes everywhere, or the coarse near-null-space
        // (the R factors) stops describing rigid motion on the next level.
        const double cx = ctr[0], cy = ctr[1], cz = ctr[2];
        for (int q = 0; q < m; ++q) {
          const int n = amem[aptr[a] + q];
          const double x = c->X[n * 3] - cx, y = c->X[n * 3 + 1] - cy, z = c->X[n * 3 + 2] - cz;
          double* r0 = &M[(q * 3 + 0) * 6];
          double* r1 = &M[(q * 3 + 1) * 6];
          double* r2 = &M[(q * 3 + 2) * 6];
          for (int k = 0; k < 6; ++k) r0[k] = r1[k] = r2[k] = 0.0;
          r0[0] = 1; r1[1] = 1; r2[2] = 1;
          r1[3] = -z; r2[3] = y;
          r0[4] = z; r2[4] = -x;
          r0[5] = -y; r1[5] = x;
        }
      } else {
        for (int q = 0; q < m; ++q) {
          const int n = amem[aptr[a] + q];
          for (int i = 0; i < bs * 6; ++i) M[(size_t)q * bs * 6 + i] = B[(size_t)n * bs * 6 + i];
        }
      }
      double R[36];
      mgs_qr(m * bs, M, R);
      for (int q = 0; q < m; ++q) {
        const int n = amem[aptr[a] + q];
        for (int i = 0; i < bs * 6; ++i) cur.T[(size_t)n * bs * 6 + i] = M[(size_t)q * bs * 6 + i];
      }
      for (int i = 0; i < 36; ++i) Bc[(size_t)a * 36 + i] = R[i];
    });
    // P pattern: row n -> aggregates of its matrix neighbours
    symbolic_product(nb, rp, cl, nullptr, nullptr, cur.agg.data(), na, cur.p_rp, cur.p_cl);
    const int nnzP = cur.p_rp[nb];
    cur.p_row.resize(nnzP);
    par_for(nb, [&](long long n) {
      for (int t = cur.p_rp[n]; t < cur.p_rp[n + 1]; ++t) cur.p_row[t] = (int)n;
    });
    cur.pslot.resize(rp[nb]);
    par_for(nb, [&](long long n) {
      const int* b0 = cur.p_cl.data() + cur.p_rp[n];
      const int* b1 = cur.p_cl.data() + cur.p_rp[n + 1];
      for (int k = rp[n]; k < rp[n + 1]; ++k)
        cur.pslot[k] = cur.p_rp[n] + (int)(std::lower_bound(b0, b1, cur.agg[cl[k]]) - b0);
    });
    // P^T
    cur.pt_rp.assign(na + 1, 0);
    for (int v : cur.p_cl) cur.pt_rp[v + 1]++;
    for (int a = 0; a < na; ++a) cur.pt_rp[a + 1] += cur.pt_rp[a];
    cur.pt_blk.resize(nnzP);
    {
      std::vector<int> f(cur.pt_rp.begin(), cur.pt_rp.end() - 1);
      for (int p = 0; p < nnzP; ++p) cur.pt_blk[f[cur.p_cl[p]]++] = p;
    }
    // A P pattern: row n -> union of the P rows of its neighbours
    symbolic_product(nb, rp, cl, cur.p_rp.data(), cur.p_cl.data(), nullptr, na, cur.ap_rp, cur.ap_cl);
    cur.ap_row.resize(cur.ap_rp[nb]);
    par_for(nb, [&](long long n) {
      for (int t = cur.ap_rp[n]; t < cur.ap_rp[n + 1]; ++t) cur.ap_row[t] = (int)n;
    });
    // Galerkin pattern of the next level: row I -> union of the AP rows of P^T(I)
    HostLevel nxt;
    nxt.nbrow = na;
    nxt.bs = 6;
    {
      std::vector<int> ptn(nnzP);  // P^T entries as the row of P they come from
      par_for(nnzP, [&](long long t) { ptn[t] = cur.p_row[cur.pt_blk[t]]; });
      symbolic_product(na, cur.pt_rp.data(), ptn.data(), cur.ap_rp.data(), cur.ap_cl.data(), nullptr, na,
                       nxt.rowptr, nxt.col);
    }
    cur.c_row.resize(nxt.rowptr[na]);
    par_for(na, [&](long long a) {
      for (int t = nxt.rowptr[a]; t < nxt.rowptr[a + 1]; ++t) cur.c_row[t] = (int)a;
    });
    // aggregation graph of the next level: aggregates adjacent in this graph
    symbolic_product(na, aptr.data(), amem.data(), grp, gcl, cur.agg.data(), na, nxt.grp, nxt.gcl);
    cur.grp.clear(); cur.grp.shrink_to_fit();
    cur.gcl.clear(); cur.gcl.shrink_to_fit();
    c->hl.push_back(std::move(cur));
    cur = std::move(nxt);
    B = std::move(Bc);
    first = false;
  }
  if (first) {  // no level was coarsened: the finest level keeps its own pattern copy
    cur.rowptr = c->browptr;
    cur.col = c->bcol;
  }
  c->hl.push_back(std::move(cur));  // coarsest: pattern only
  c->amg_struct = true;
}

template <typename T>
Amg<T>& amg_of(pfem_ctx* c);
template <>
Amg<float>& amg_of<float>(pfem_ctx* c) { return c->amg32; }
template <>
Amg<double>& amg_of<double>(pfem_ctx* c) { return c->amg64; }
template <typename T>
KrylovWork<T>& kw_of(pfem_ctx* c);
template <>
KrylovWork<float>& kw_of<float>(pfem_ctx* c) { return c->kw32; }
template <>
KrylovWork<double>& kw_of<double>(pfem_ctx* c) { return c->kw64; }
template <typename T>
CgGraph& cg_of(pfem_ctx* c);
template <>
CgGraph& cg_of<float>(pfem_ctx* c) { return c->cg32; }
template <>
CgGraph& cg_of<double>(pfem_ctx* c) { return c->cg64; }
template <typename T>
T* K_of(pfem_ctx* c);
template <>
float* K_of<float>(pfem_ctx* c) { return c->dK32; }
template <>
double* K_of<double>(pfem_ctx* c) { return c->dK64; }

__global__ void hash_fill_kernel(long long n, float* xf, double* xd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
    const double v = 0.5 + (double)(h & 0xFFFFFF) / (double)0x1000000;
    if (xf) xf[i] = (float)v;
    if (xd) xd[i] = v;
  }
}
template <typename T>
__global__ void scale_by_inv_kernel(long long n, const T* __restrict__ s, const T* __restrict__ w, T* __restrict__ v) {
  const T inv = T(1) / *s;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = w[i] * inv;
}
template <typename T>
__global__ void bicg_finish_kernel(T* sc) {
  sc[2] = sc[0] / sc[4];
  sc[3] = sc[5] / sc[6];
  sc[1] = sc[0];
}
template <typename T>
__global__ void bicg_init_kernel(T* sc) {
  sc[1] = T(1); sc[2] = T(1); sc[3] = T(1);
}

// Allocate the device side of the hierarchy for precision T (once).
template <typename T>
int amg_alloc(pfem_ctx* ctx) {
  Amg<T>& A = amg_of<T>(ctx);
  if (!A.lv.empty()) return PFEM_OK;
  const int L = (int)ctx->hl.size() - 1;
  if (L < 1) return fail(ctx, PFEM_ERR_STATE, "mesh too small to build an aggregation hierarchy");
  A.lv.resize(L);
  for (int l = 0; l < L; ++l) {
    const HostLevel& h = ctx->hl[l];
    AmgLevel<T>& v = A.lv[l];
    v.A.nbrow = h.nbrow;
    v.A.bs = h.bs;
    v.A.nnzb = l == 0 ? ctx->nnzb : h.rowptr[h.nbrow];
    if (l == 0) {
      v.A.rowptr = ctx->dBrowptr;
      v.A.col = ctx->dBcol;
      v.A.col16 = ctx->dBcol16;
    } else {
      CK(upload(ctx, &v.A.rowptr, h.rowptr));
      CK(upload(ctx, &v.A.col, h.col));
      CK(dalloc(ctx, &v.A.val, (size_t)v.A.nnzb * h.bs * h.bs));
    }
    CK(dalloc(ctx, &v.dinv, (size_t)h.nbrow * h.bs * h.bs));
    v.nagg = h.nagg;
    CK(upload(ctx, &v.agg, h.agg));
    std::vector<T> Th(h.T.begin(), h.T.end());
    CK(upload(ctx, &v.T, Th));
    v.nnzP = (int)h.p_cl.size();
    CK(upload(ctx, &v.p_rp, h.p_rp)); CK(upload(ctx, &v.p_cl, h.p_cl)); CK(upload(ctx, &v.p_row, h.p_row));
    CK(upload(ctx, &v.pslot, h.pslot)); CK(upload(ctx, &v.pt_rp, h.pt_rp)); CK(upload(ctx, &v.pt_blk, h.pt_blk));
    {
      std::vector<int> ptr_row(h.pt_blk.size());
      for (size_t t = 0; t < h.pt_blk.size(); ++t) ptr_row[t] = h.p_row[h.pt_blk[t]];
      CK(upload(ctx, &v.pt_row, ptr_row));
    }
    CK(dalloc(ctx, &v.p_val, (size_t)v.nnzP * h.bs * 6));
    CK(dalloc(ctx, &v.pt_val, (size_t)v.nnzP * h.bs * 6));
    v.nnzAP = (int)h.ap_cl.size();
    CK(upload(ctx, &v.ap_rp, h.ap_rp)); CK(upload(ctx, &v.ap_cl, h.ap_cl)); CK(upload(ctx, &v.ap_row, h.ap_row));
    CK(dalloc(ctx, &v.ap_val, (size_t)v.nnzAP * h.bs * 6));
    CK(upload(ctx, &v.c_row, h.c_row));
    CK(upload(ctx, &v.c_cl, ctx->hl[l + 1].col));
    const size_t n = (size_t)h.nbrow * h.bs;
    CK(dalloc(ctx, &v.x, n)); CK(dalloc(ctx, &v.b, n)); CK(dalloc(ctx, &v.r, n));
    CK(dalloc(ctx, &v.d, n)); CK(dalloc(ctx, &v.t, n));
    if (l >= 2) { CK(dalloc(ctx, &v.b2, n)); CK(dalloc(ctx, &v.x2, n)); }
  }
  const HostLevel& hc = ctx->hl[L];
  A.coarse_n = hc.nbrow * hc.bs;
  A.coarse_nnzb = hc.rowptr[hc.nbrow];
  CK(dalloc(ctx, &A.coarse_val, (size_t)A.coarse_nnzb * 36));
  CK(upload(ctx, &A.coarse_rp, hc.rowptr));
  CK(upload(ctx, &A.coarse_cl, hc.col));
  CK(dalloc(ctx, &A.coarse_inv, (size_t)A.coarse_n * A.coarse_n));
  if (!ctx->dDenseWork) CK(dalloc(ctx, &ctx->dDenseWork, (size_t)pfem::dense_inverse_work_doubles(A.coarse_n)));
  CK(dalloc(ctx, &A.cx, (size_t)A.coarse_n));
  CK(dalloc(ctx, &A.cb, (size_t)A.coarse_n));
  return PFEM_OK;
}

template <typename T>
int krylov_alloc(pfem_ctx* ctx) {
  KrylovWork<T>& w = kw_of<T>(ctx);
  if (w.n == ctx->ndof) return PFEM_OK;
  const size_t n = ctx->ndof;
  w.n = ctx->ndof;
  CK(dalloc(ctx, &w.x, n)); CK(dalloc(ctx, &w.r, n)); CK(dalloc(ctx, &w.z, n));
  CK(dalloc(ctx, &w.p, n)); CK(dalloc(ctx, &w.q, n)); CK(dalloc(ctx, &w.rh, n));
  CK(dalloc(ctx, &w.v, n)); CK(dalloc(ctx, &w.s, n)); CK(dalloc(ctx, &w.t, n));
  CK(dalloc(ctx, &w.ph, n)); CK(dalloc(ctx, &w.sh, n)); CK(dalloc(ctx, &w.b, n));
  CK(dalloc(ctx, &w.xa, n)); CK(dalloc(ctx, &w.b0, n));
  CK(dalloc(ctx, &w.sc, 16)); CK(dalloc(ctx, &w.part, 3 * 2048));  // three partial sets of the fused PCG body
  return PFEM_OK;
}

// Gauss-Jordan inverse of a dense n x n matrix (row-major, double) with
// partial pivoting; near-singular pivots are regularised.  Used for small
// coarsest levels (at most kCoarseHostMax unknowns), where a pivot-free
// elimination can meet tiny pivots: partially constrained aggregates leave
// coarse rows that are nearly dependent.
void dense_inverse_host(int n, std::vector<double>& a, std::vector<double>& inv) {
  // In-place Gauss-Jordan with partial pivoting (n^3 multiply-adds): column c of the
  // identity is never stored, the pivot row's slot c takes 1 / pivot, and the row
  // exchanges are undone on the columns at the end.
  double scl = 0;
  for (int i = 0; i < n; ++i) scl = std::max(scl, std::fabs(a[(size_t)i * n + i]));
  std::vector<int> perm(n);
  for (int c = 0; c < n; ++c) {
    int piv = c;
    double best = std::fabs(a[(size_t)c * n + c]);
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a[(size_t)r * n + c]) > best) { best = std::fabs(a[(size_t)r * n + c]); piv = r; }
    perm[c] = piv;
    if (piv != c)
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)c * n + j], a[(size_t)piv * n + j]);
    double* rc = a.data() + (size_t)c * n;
    double pv = rc[c];
    if (std::fabs(pv) < 1e-14 * std::max(scl, 1e-300)) pv = (pv >= 0 ? 1.0 : -1.0) * 1e-14 * std::max(scl, 1e-300);
    const double ip = 1.0 / pv;
    rc[c] = 1.0;
    for (int j = 0; j < n; ++j) rc[j] *= ip;
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      double* rr = a.data() + (size_t)r * n;
      const double f = rr[c];
      if (f == 0.0) continue;
      rr[c] = 0.0;
      for (int j = 0; j < n; ++j) rr[j] -= f * rc[j];
    }
  }
  for (int c = n - 1; c >= 0; --c)
    if (perm[c] != c)
      for (int i = 0; i < n; ++i) std::swap(a[(size_t)i * n + c], a[(size_t)i * n + perm[c]]);
  inv.swap(a);
}

// Numeric AMG set-up on the current (Dirichlet-imposed) tangent of precision T:
// block-Jacobi inverses, Chebyshev bounds by power iteration, Galerkin
// coarse operators, dense coarse inverse -- all on the device.  Rebuilt per load step by default
// (the reference's reuse policy, Solver.jl:243-245).
template <typename T>
int amg_setup(pfem_ctx* ctx, int cheb_degree) {
  const bool dbg = getenv("PFEM_DEBUG_AMG") != nullptr;
  auto ts = std::chrono::steady_clock::now();
  if (!ctx->amg_struct) build_amg_structure(ctx);
  int rc = amg_alloc<T>(ctx);
  if (rc) return rc;
  rc = krylov_alloc<T>(ctx);
  if (rc) return rc;
  Amg<T>& A = amg_of<T>(ctx);
  KrylovWork<T>& w = kw_of<T>(ctx);
  A.cheb_degree = cheb_degree;
  A.lv[0].A.val = K_of<T>(ctx);
  const int L = (int)A.lv.size();
  for (int l = 0; l < L; ++l) {
    AmgLevel<T>& v = A.lv[l];
    blockdiag_invert<T>(v.A, v.dinv, ctx->st);
    CKL();
    // power iteration on D^-1 A
    const long long n = (long long)v.A.nbrow * v.A.bs;
    pfem::count_launch(); hash_fill_kernel<<<256, 256, 0, ctx->st>>>(n, std::is_same<T, float>::value ? (float*)v.d : nullptr,
                                               std::is_same<T, double>::value ? (double*)v.d : nullptr);
    for (int it = 0; it < 12; ++it) {
      bsr_spmv<T>(v.A, v.d, v.t, ctx->st);
      blockdiag_apply<T>(v.A.nbrow, v.A.bs, v.dinv, v.t, v.r, T(1), nullptr, ctx->st);
      dot<T>(n, v.r, v.r, w.sc + 8, w.part, ctx->st, true);
      pfem::count_launch(); scale_by_inv_kernel<T><<<256, 256, 0, ctx->st>>>(n, w.sc + 8, v.r, v.d);
    }
    CKL();
    T lm = 0;
    CK(cudaMemcpyAsync(&lm, w.sc + 8, sizeof(T), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    v.lmax = (T)(1.1 * (double)lm);
    if (getenv("PFEM_DEBUG_AMG"))
      fprintf(stderr, "amg level %d: block rows %d bs %d nnzb %lld aggregates %d P blocks %d lmax %.4g\n", l,
              v.A.nbrow, v.A.bs, v.A.nnzb, v.nagg, v.nnzP, (double)v.lmax);
    // smoothed prolongator and Galerkin operator of the next level
    const T omega = (T)(4.0 / (3.0 * (double)lm));
    T* cval = (l + 1 < L) ? A.lv[l + 1].A.val : A.coarse_val;
    const int nnzC = (int)ctx->hl[l + 1].rowptr[ctx->hl[l + 1].nbrow];
    sa_setup_level<T>(v, omega, cval, nnzC, ctx->st);
    CKL();
  }
  if (dbg) cudaStreamSynchronize(ctx->st);
  auto tl = std::chrono::steady_clock::now();
  // coarsest operator: dense inverse, on the device (blocked Gauss-Jordan) for
  // large coarsest levels, on the host with partial pivoting for small ones
  if (A.coarse_n > kCoarseHostMax) {
    pfem::dense_coarse_inverse<T>(ctx->hl[L].nbrow, A.coarse_rp, A.coarse_cl, A.coarse_val, A.coarse_n,
                                  ctx->dDenseWork, A.coarse_inv, ctx->st);
    CKL();
  } else {
    const HostLevel& hc = ctx->hl[L];
    std::vector<T> hv((size_t)A.coarse_nnzb * 36);
    CK(cudaMemcpyAsync(hv.data(), A.coarse_val, hv.size() * sizeof(T), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const int n = A.coarse_n;
    std::vector<double> dense((size_t)n * n, 0.0), inv;
    for (int I = 0; I < hc.nbrow; ++I)
      for (int k = hc.rowptr[I]; k < hc.rowptr[I + 1]; ++k) {
        const int J = hc.col[k];
        for (int r = 0; r < 6; ++r)
          for (int c = 0; c < 6; ++c) dense[(size_t)(I * 6 + r) * n + J * 6 + c] = (double)hv[(size_t)k * 36 + r * 6 + c];
      }
    // rigid modes absent from an aggregate leave zero rows: put 1 on their diagonal
    for (int i = 0; i < n; ++i) {
      bool zero = true;
      for (int j = 0; j < n && zero; ++j) zero = dense[(size_t)i * n + j] == 0.0;
      if (zero) dense[(size_t)i * n + i] = 1.0;
    }
    dense_inverse_host(n, dense, inv);
    std::vector<T> invT(inv.begin(), inv.end());
    CK(cudaMemcpyAsync(A.coarse_inv, invT.data(), invT.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
  }
  A.built = true;
  A.version++;
  if (dbg) {
    cudaStreamSynchronize(ctx->st);
    auto te = std::chrono::steady_clock::now();
    fprintf(stderr, "amg set-up %.3f ms: levels %.3f ms, coarse inverse (%d unknowns) %.3f ms\n",
            std::chrono::duration<double, std::milli>(te - ts).count(),
            std::chrono::duration<double, std::milli>(tl - ts).count(), A.coarse_n,
            std::chrono::duration<double, std::milli>(te - tl).count());
  }
  return PFEM_OK;
}

// Chebyshev smoothing (block-Jacobi preconditioned) on level l:
// x <- x + p(D^-1 A) D^-1 (b - A x), degree A.cheb_degree, interval
// [lmax/30, lmax].  zero: x enters as 0.
// Degree-2 coefficients on [lmax/30, lmax]: x2 = x0 + d0 + d1 with d0 = r0 / th,
// r0 = Dinv (b - A x0), r1 = r0 - Dinv A d0, d1 = c1 r1 + (c2 - 1) d0.
template <typename T>
void cheb2_coeffs(const AmgLevel<T>& v, T* inv_th, T* c1, T* c2) {
  const double lmx = (double)v.lmax, lmn = lmx / 30.0;
  const double th = 0.5 * (lmx + lmn), de = 0.5 * (lmx - lmn);
  const double sg = th / de, rho = 1.0 / sg;
  const double rn = 1.0 / (2.0 * sg - rho);
  *inv_th = T(1.0 / th);
  *c1 = T(2.0 * rn / de);
  *c2 = T(1.0 + rn * rho);
}

template <typename T>
void cheb(pfem_ctx* ctx, AmgLevel<T>& v, int degree, const T* b, T* x, bool zero) {
  const long long n = (long long)v.A.nbrow * v.A.bs;
  const double lmx = (double)v.lmax, lmn = lmx / 30.0;
  const double th = 0.5 * (lmx + lmn), de = 0.5 * (lmx - lmn);
  const double sg = th / de;
  double rho = 1.0 / sg;
  if (degree == 2) {
    // one block-Jacobi pass (or a fused residual pass) and one fused SpMV pass
    T inv_th, c1, c2;
    cheb2_coeffs<T>(v, &inv_th, &c1, &c2);
    if (zero) blockdiag_apply<T>(v.A.nbrow, v.A.bs, v.dinv, b, v.r, inv_th, v.d, ctx->st);
    else bsr_residual_precond<T>(v.A, v.dinv, x, b, v.r, v.d, inv_th, ctx->st);
    bsr_cheb2<T>(v.A, v.dinv, v.d, v.r, x, zero, c1, c2, ctx->st);
    return;
  }
  if (zero) {
    fill<T>(n, x, T(0), ctx->st);
    blockdiag_apply<T>(v.A.nbrow, v.A.bs, v.dinv, b, v.r, T(1.0 / th), v.d, ctx->st);
  } else {
    bsr_residual<T>(v.A, x, b, v.t, ctx->st);
    blockdiag_apply<T>(v.A.nbrow, v.A.bs, v.dinv, v.t, v.r, T(1.0 / th), v.d, ctx->st);
  }
  for (int k = 1; k <= degree; ++k) {
    if (k < degree) {
      bsr_cheb_step<T>(v.A, v.dinv, v.d, v.r, x, ctx->st);
      const double rn = 1.0 / (2.0 * sg - rho);
      axpby<T>(n, T(2.0 * rn / de), v.r, T(rn * rho), v.d, ctx->st);
      rho = rn;
    } else {
      axpby<T>(n, T(1), v.d, T(1), x, ctx->st);
    }
  }
}

template <typename T>
void vcycle(pfem_ctx* ctx, int l, const T* b, T* x) {
  Amg<T>& A = amg_of<T>(ctx);
  const int L = (int)A.lv.size();
  AmgLevel<T>& v = A.lv[l];
  cheb<T>(ctx, v, A.cheb_degree, b, x, true);
  bsr_residual<T>(v.A, x, b, v.t, ctx->st);
  T* bn = (l + 1 < L) ? A.lv[l + 1].b : A.cb;
  T* xn = (l + 1 < L) ? A.lv[l + 1].x : A.cx;
  sa_restrict<T>(v, v.t, bn, ctx->st);
  if (l + 1 < L) vcycle<T>(ctx, l + 1, bn, xn);
  else dense_mv<T>(A.coarse_n, A.coarse_inv, bn, xn, ctx->st);
  if (l >= 1 && l + 1 < L) {
    // Below the finest level the cycle is a W: two iterations on the coarse
    // problem.  The second starts from the coarse residual bn - A_c xn, which
    // equals the restriction of the updated fine residual because A_c is the
    // Galerkin product P^T A P, so this level's matrix is not read again; both
    // corrections are prolonged in one pass.  The coarse levels cost a small
    // fraction of level 0, and the stronger coarse solve cuts the CG iterations.
    AmgLevel<T>& c = A.lv[l + 1];
    bsr_residual<T>(c.A, xn, bn, c.b2, ctx->st);
    vcycle<T>(ctx, l + 1, c.b2, c.x2);
    sa_prolong2<T>(v, xn, c.x2, x, ctx->st);
  } else {
    sa_prolong<T>(v, xn, x, ctx->st);
  }
  cheb<T>(ctx, v, A.cheb_degree, b, x, false);
}

template <typename T>
__global__ void cg_graph_init_kernel(cudaGraphConditionalHandle h, const T* __restrict__ bn, T* __restrict__ sc0,
                                     double* __restrict__ ctl, int* __restrict__ state) {
  const double b = (double)*bn;
  ctl[2] = ctl[0] * b;
  state[0] = 0;
  state[1] = b == 0.0 ? 1 : 0;  // b = 0: x = 0 is the solution
  *sc0 = T(1);                  // with p = 0, the first update p = z + (r.z / 1) p gives p = z
  cudaGraphSetConditional(h, (b > 0.0 && isfinite(b)) ? 1u : 0u);
}
// End of a PCG iteration: |r| from the np partials of r.r (fixed order, one
// CTA of 1024 threads), into sc_rn, then the loop condition.
template <typename T>
__global__ void cg_graph_check_kernel(cudaGraphConditionalHandle h, const T* __restrict__ part, int np,
                                      T* __restrict__ sc_rn, const double* __restrict__ ctl,
                                      int* __restrict__ state) {
  __shared__ T sh[32];
  T v = T(0);
  for (int i = threadIdx.x; i < np; i += blockDim.x) v += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x >= 32) return;
  v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : T(0);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x != 0) return;
  const T rn = sqrt(v);
  *sc_rn = rn;
  const int it = state[0] + 1;
  state[0] = it;
  const double r = (double)rn;
  const bool conv = r <= ctl[2];
  state[1] = conv ? 1 : 0;
  cudaGraphSetConditional(h, (!conv && isfinite(r) && it < (int)ctl[1]) ? 1u : 0u);
}

// Capture (or reuse) the device-side CG loop for the current hierarchy.
template <typename T>
int cg_graph_build(pfem_ctx* ctx) {
  CgGraph& G = cg_of<T>(ctx);
  Amg<T>& A = amg_of<T>(ctx);
  if (G.exec && G.amg_version == A.version) return PFEM_OK;
  if (G.exec) { cudaGraphExecDestroy(G.exec); G.exec = nullptr; }
  if (G.graph) { cudaGraphDestroy(G.graph); G.graph = nullptr; }
  if (!G.ctl) {
    CK(dalloc(ctx, &G.ctl, 4));
    CK(dalloc(ctx, &G.state, 4));
    CK(cudaStreamCreateWithFlags(&G.body_stream, cudaStreamNonBlocking));
  }
  KrylovWork<T>& w = kw_of<T>(ctx);
  const BsrMat<T>& K = A.lv[0].A;
  const long long n = ctx->ndof;
  cudaStream_t st = ctx->st;
  const long long c0 = pfem::launch_counter();
  cudaGraph_t g = nullptr;
  cudaGraph_t body = nullptr;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(ctx, PFEM_ERR_CUDA, std::string("CG graph capture: ") + cudaGetErrorString(e));
  auto abort_capture = [&](cudaError_t err, const char* what) {
    cudaGraph_t junk = nullptr;
    ctx->st = st;
    cudaStreamEndCapture(G.body_stream, &junk);
    cudaStreamEndCapture(st, &junk);
    if (junk) cudaGraphDestroy(junk);
    cudaGetLastError();
    return fail(ctx, PFEM_ERR_CUDA, std::string("CG graph capture (") + what + "): " + cudaGetErrorString(err));
  };
  fill<T>(n, w.x, T(0), st);
  fill<T>(n, w.p, T(0), st);
  e = cudaMemcpyAsync(w.r, w.b, n * sizeof(T), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return abort_capture(e, "r = b");
  dot<T>(n, w.b, w.b, w.sc + 10, w.part, st, true);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd);
  if (e != cudaSuccess) return abort_capture(e, "capture info");
  cudaGraphConditionalHandle h;
  e = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
  if (e != cudaSuccess) return abort_capture(e, "conditional handle");
  cg_graph_init_kernel<T><<<1, 1, 0, st>>>(h, w.sc + 10, w.sc + 0, G.ctl, G.state);
  e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd);
  if (e != cudaSuccess) return abort_capture(e, "capture info");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  e = cudaGraphAddNode(&cnode, g, deps, nd, &cp);
  if (e != cudaSuccess) return abort_capture(e, "conditional node");
  e = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
  if (e != cudaSuccess) return abort_capture(e, "capture dependencies");
  const long long c1 = pfem::launch_counter();
  // ---- loop body: one PCG iteration ----
  body = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(G.body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return abort_capture(e, "body capture");
  cudaStream_t bs = G.body_stream;
  ctx->st = bs;  // the V-cycle launches on ctx->st
  vcycle<T>(ctx, 0, w.r, w.z);
  ctx->st = st;
  // sc[0] = r.z of the previous iteration, sc[2] = r.z; the final sums of the
  // three dot products happen inside the kernels that use them
  T* const part_rz = w.part;
  T* const part_pq = w.part + 2048;
  T* const part_rr = w.part + 4096;
  const int np_rz = dot_partials<T>(n, w.r, w.z, part_rz, bs);
  cg_p_fused<T>(n, part_rz, np_rz, w.sc, w.z, w.p, bs);
  bsr_spmv<T>(K, w.p, w.q, bs);
  const int np_pq = dot_partials<T>(n, w.p, w.q, part_pq, bs);
  const int np_rr = cg_xr_fused<T>(n, part_pq, np_pq, w.sc, w.p, w.q, w.x, w.r, part_rr, bs);
  cg_graph_check_kernel<T><<<1, 1024, 0, bs>>>(h, part_rr, np_rr, w.sc + 3, G.ctl, G.state);
  e = cudaStreamEndCapture(bs, &body);
  if (e != cudaSuccess) return abort_capture(e, "body end");
  const long long c2 = pfem::launch_counter();
  e = cudaStreamEndCapture(st, &g);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, PFEM_ERR_CUDA, std::string("CG graph capture (end): ") + cudaGetErrorString(e));
  }
  G.graph = g;
  e = cudaGraphInstantiate(&G.exec, g, 0);
  if (e != cudaSuccess) {
    G.exec = nullptr;
    return fail(ctx, PFEM_ERR_CUDA, std::string("CG graph instantiate: ") + cudaGetErrorString(e));
  }
  // launches are counted when the graph runs, not when it is captured
  G.prefix_kernels = c1 - c0 + 1;
  G.body_kernels = c2 - c1 + 1;
  pfem::launch_counter() = c0;
  G.amg_version = A.version;
  return PFEM_OK;
}

// Preconditioned CG / BiCGStab on level-0 operator with the AMG V-cycle.
// b and the result x live in kw.b / kw.x.  Returns iterations (>=0) or <0.
template <typename T>
int krylov_inner(pfem_ctx* ctx, int method, double rtol, int itmax, int* iters, bool* conv) {
  Amg<T>& A = amg_of<T>(ctx);
  KrylovWork<T>& w = kw_of<T>(ctx);
  const BsrMat<T>& K = A.lv[0].A;
  const long long n = ctx->ndof;
  cudaStream_t st = ctx->st;
  *iters = 0;
  *conv = false;
  if (method == PFEM_KRYLOV_CG) {
    const bool dbg = getenv("PFEM_DEBUG_AMG") != nullptr;
    auto tg = std::chrono::steady_clock::now();
    int rc = cg_graph_build<T>(ctx);
    if (rc) return rc;
    if (dbg) {
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tg).count();
      if (ms > 0.05) fprintf(stderr, "cg graph capture + instantiate %.3f ms\n", ms);
    }
    CgGraph& G = cg_of<T>(ctx);
    const double ctl[2] = {rtol, (double)std::max(itmax, 1)};
    CK(cudaMemcpyAsync(G.ctl, ctl, sizeof(ctl), cudaMemcpyHostToDevice, st));
    CK(cudaGraphLaunch(G.exec, st));
    int sh[2] = {0, 0};
    CK(cudaMemcpyAsync(sh, G.state, sizeof(sh), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *iters = sh[0];
    *conv = sh[1] != 0;
    pfem::launch_counter() += G.prefix_kernels + (long long)sh[0] * G.body_kernels;
    return PFEM_OK;
  }
  fill<T>(n, w.x, T(0), st);
  CK(cudaMemcpyAsync(w.r, w.b, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  dot<T>(n, w.b, w.b, w.sc + 10, w.part, st, true);
  T bn = 0;
  CK(cudaMemcpyAsync(&bn, w.sc + 10, sizeof(T), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (!(bn > 0)) { *conv = true; return PFEM_OK; }
  const double thr = rtol * (double)bn;
  {  // BiCGStab: host-driven loop
    CK(cudaMemcpyAsync(w.rh, w.b, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    fill<T>(n, w.v, T(0), st);
    fill<T>(n, w.p, T(0), st);
    pfem::count_launch(); bicg_init_kernel<T><<<1, 1, 0, st>>>(w.sc);
    for (int it = 1; it <= itmax; ++it) {
      dot<T>(n, w.rh, w.r, w.sc + 0, w.part, st, false);
      bicg_p<T>(n, w.sc, w.r, w.v, w.p, st);
      vcycle<T>(ctx, 0, w.p, w.ph);
      bsr_spmv<T>(K, w.ph, w.v, st);
      dot<T>(n, w.rh, w.v, w.sc + 4, w.part, st, false);
      bicg_s<T>(n, w.sc, w.r, w.v, w.s, st);
      vcycle<T>(ctx, 0, w.s, w.sh);
      bsr_spmv<T>(K, w.sh, w.t, st);
      dot<T>(n, w.t, w.s, w.sc + 5, w.part, st, false);
      dot<T>(n, w.t, w.t, w.sc + 6, w.part, st, false);
      bicg_xr<T>(n, w.sc, w.ph, w.sh, w.s, w.t, w.x, w.r, st);
      pfem::count_launch(); bicg_finish_kernel<T><<<1, 1, 0, st>>>(w.sc);
      // |r| goes to slot 7: slot 3 holds omega for the next iteration's beta
      dot<T>(n, w.r, w.r, w.sc + 7, w.part, st, true);
      T rn = 0;
      CK(cudaMemcpyAsync(&rn, w.sc + 7, sizeof(T), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      *iters = it;
      if ((double)rn <= thr) { *conv = true; break; }
      if (!std::isfinite((double)rn)) break;
    }
  }
  CKL();
  return PFEM_OK;
}

// Solve K x = b (kw.b -> kw.x) to relative tolerance rtol.  Below the level a
// recursively updated Krylov residual reliably reaches in precision T (1e-8 in
// FP64, 1e-5 in FP32 -- the F-bar tangent is nonsymmetric, so CG and
// BiCGStab drift from the true residual there), the inner method runs inside
// an iterative-refinement loop: x += inner solve of K d = b - K x, with the
// residual recomputed from K each pass.
template <typename T>
int krylov(pfem_ctx* ctx, int method, double rtol, int itmax, int* iters, bool* conv) {
  const double floor_rtol = std::is_same<T, double>::value ? 1e-8 : 1e-5;
  if (rtol >= floor_rtol) return krylov_inner<T>(ctx, method, rtol, itmax, iters, conv);
  Amg<T>& A = amg_of<T>(ctx);
  KrylovWork<T>& w = kw_of<T>(ctx);
  const BsrMat<T>& K = A.lv[0].A;
  const long long n = ctx->ndof;
  cudaStream_t st = ctx->st;
  CK(cudaMemcpyAsync(w.b0, w.b, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  fill<T>(n, w.xa, T(0), st);
  dot<T>(n, w.b0, w.b0, w.sc + 12, w.part, st, true);
  T bn = 0;
  CK(cudaMemcpyAsync(&bn, w.sc + 12, sizeof(T), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *iters = 0;
  *conv = false;
  if (!(bn > 0)) {
    fill<T>(n, w.x, T(0), st);
    *conv = true;
    return PFEM_OK;
  }
  const double target = rtol * (double)bn;
  double rn = (double)bn;
  for (int pass = 0; pass < 8 && *iters < itmax; ++pass) {
    int it = 0;
    bool c = false;
    const double rel = std::max(floor_rtol, target / rn);
    int rc = krylov_inner<T>(ctx, method, rel, itmax - *iters, &it, &c);
    if (rc) return rc;
    *iters += it;
    axpby<T>(n, T(1), w.x, T(1), w.xa, st);
    bsr_residual<T>(K, w.xa, w.b0, w.b, st);  // next right-hand side: the true residual
    dot<T>(n, w.b, w.b, w.sc + 12, w.part, st, true);
    T r = 0;
    CK(cudaMemcpyAsync(&r, w.sc + 12, sizeof(T), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    rn = (double)r;
    if (!std::isfinite(rn)) break;
    if (rn <= target) {
      *conv = true;
      break;
    }
  }
  CK(cudaMemcpyAsync(w.x, w.xa, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(w.b, w.b0, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  CKL();
  return PFEM_OK;
}

// One full assembly of K (precision prec) and R: the element kernel over every
// element into element-ordered buffers, then the row-owned gather (or, with
// colored_assembly, zeroed K and R and one element-kernel launch per color adding
// in place); commit runs the state update over all elements in one launch.
int assemble_dev(pfem_ctx* ctx, int prec, bool commit) {
  cudaStream_t st = ctx->st;
  const bool fbar = ctx->kind == PFEM_HEX8_FINITE_FBAR;
  const bool small = ctx->kind == PFEM_HEX8_SMALL;
  CK(cudaMemsetAsync(ctx->dStatus, 0, sizeof(DevStatus), st));
  if (commit) {
    ElemArgs<double> a{};
    a.X = ctx->dX; a.elem = ctx->dElem; a.U = ctx->dU; a.cpi = ctx->dCpi; a.alpha = ctx->dAlpha;
    a.epsp = ctx->dEpsp; a.beta = ctx->dBeta; a.sigy0_e = ctx->dSigy; a.tau = ctx->dTau; a.flags = ctx->dFlags;
    a.R = ctx->dR; a.Kval = ctx->dK64; a.browptr = ctx->dBrowptr; a.rank = ctx->dRank;
    a.ngp = ctx->ngp; a.mat = ctx->mat; a.status = ctx->dStatus;
    if (small) launch_element_small<double>(a, ctx->dAllElems, (int)ctx->ne, true, ctx->hard, st);
    else launch_element_color<double>(a, ctx->dAllElems, (int)ctx->ne, true, fbar, ctx->hard, st);
    CKL();
    return PFEM_OK;
  }
  if (!ctx->colored_assembly) {
    // one launch over every element into the element-ordered buffers, then the
    // row-owned gather writes each block of K and each entry of R once
    if (!ctx->dFbuf) CK(dalloc(ctx, &ctx->dFbuf, (size_t)ctx->ne * 24));
    if (prec == PFEM_FP64) {
      if (!ctx->dKbuf64) CK(dalloc(ctx, &ctx->dKbuf64, (size_t)ctx->ne * 576));
      ElemArgs<double> a{};
      a.X = ctx->dX; a.elem = ctx->dElem; a.U = ctx->dU; a.cpi = ctx->dCpi; a.alpha = ctx->dAlpha;
      a.epsp = ctx->dEpsp; a.beta = ctx->dBeta; a.sigy0_e = ctx->dSigy; a.tau = ctx->dTau; a.flags = ctx->dFlags;
      a.R = ctx->dR; a.Kval = ctx->dK64; a.browptr = ctx->dBrowptr; a.rank = ctx->dRank;
      a.ngp = ctx->ngp; a.mat = ctx->mat; a.status = ctx->dStatus;
      a.Kbuf = ctx->dKbuf64; a.Fbuf = ctx->dFbuf;
      if (small) launch_element_small<double>(a, ctx->dAllElems, (int)ctx->ne, false, ctx->hard, st);
      else launch_element_color<double>(a, ctx->dAllElems, (int)ctx->ne, false, fbar, ctx->hard, st);
      launch_gather_rows<double>((int)ctx->nn, ctx->dNptr, ctx->dNel, ctx->dNloc, ctx->dBrowptr, ctx->dRank,
                                 ctx->dKbuf64, ctx->dFbuf, ctx->dK64, ctx->dR, ctx->max_row, st);
    } else {
      if (!ctx->dKbuf32) CK(dalloc(ctx, &ctx->dKbuf32, (size_t)ctx->ne * 576));
      ElemArgs<float> a{};
      a.X = ctx->dX; a.elem = ctx->dElem; a.U = ctx->dU; a.cpi = ctx->dCpi; a.alpha = ctx->dAlpha;
      a.epsp = ctx->dEpsp; a.beta = ctx->dBeta; a.sigy0_e = ctx->dSigy; a.tau = ctx->dTau; a.flags = ctx->dFlags;
      a.R = ctx->dR; a.Kval = ctx->dK32; a.browptr = ctx->dBrowptr; a.rank = ctx->dRank;
      a.ngp = ctx->ngp; a.mat = ctx->mat; a.status = ctx->dStatus;
      a.Kbuf = ctx->dKbuf32; a.Fbuf = ctx->dFbuf;
      if (small) launch_element_small<float>(a, ctx->dAllElems, (int)ctx->ne, false, ctx->hard, st);
      else launch_element_color<float>(a, ctx->dAllElems, (int)ctx->ne, false, fbar, ctx->hard, st);
      launch_gather_rows<float>((int)ctx->nn, ctx->dNptr, ctx->dNel, ctx->dNloc, ctx->dBrowptr, ctx->dRank,
                                ctx->dKbuf32, ctx->dFbuf, ctx->dK32, ctx->dR, ctx->max_row, st);
    }
    CKL();
    return PFEM_OK;
  }
  CK(cudaMemsetAsync(ctx->dR, 0, ctx->ndof * sizeof(double), st));
  const int nc = (int)ctx->color_ptr.size() - 1;
  if (prec == PFEM_FP64) {
    CK(cudaMemsetAsync(ctx->dK64, 0, (size_t)ctx->nnzb * 9 * sizeof(double), st));
    ElemArgs<double> a{};
    a.X = ctx->dX; a.elem = ctx->dElem; a.U = ctx->dU; a.cpi = ctx->dCpi; a.alpha = ctx->dAlpha;
    a.epsp = ctx->dEpsp; a.beta = ctx->dBeta; a.sigy0_e = ctx->dSigy; a.tau = ctx->dTau; a.flags = ctx->dFlags;
    a.R = ctx->dR; a.Kval = ctx->dK64; a.browptr = ctx->dBrowptr; a.rank = ctx->dRank;
    a.ngp = ctx->ngp; a.mat = ctx->mat; a.status = ctx->dStatus;
    for (int c = 0; c < nc; ++c) {
      const int* cl = ctx->dColorList + ctx->color_ptr[c];
      const int cn = ctx->color_ptr[c + 1] - ctx->color_ptr[c];
      if (small) launch_element_small<double>(a, cl, cn, false, ctx->hard, st);
      else launch_element_color<double>(a, cl, cn, false, fbar, ctx->hard, st);
    }
  } else {
    CK(cudaMemsetAsync(ctx->dK32, 0, (size_t)ctx->nnzb * 9 * sizeof(float), st));
    ElemArgs<float> a{};
    a.X = ctx->dX; a.elem = ctx->dElem; a.U = ctx->dU; a.cpi = ctx->dCpi; a.alpha = ctx->dAlpha;
    a.epsp = ctx->dEpsp; a.beta = ctx->dBeta; a.sigy0_e = ctx->dSigy; a.tau = ctx->dTau; a.flags = ctx->dFlags;
    a.R = ctx->dR; a.Kval = ctx->dK32; a.browptr = ctx->dBrowptr; a.rank = ctx->dRank;
    a.ngp = ctx->ngp; a.mat = ctx->mat; a.status = ctx->dStatus;
    for (int c = 0; c < nc; ++c) {
      const int* cl = ctx->dColorList + ctx->color_ptr[c];
      const int cn = ctx->color_ptr[c + 1] - ctx->color_ptr[c];
      if (small) launch_element_small<float>(a, cl, cn, false, ctx->hard, st);
      else launch_element_color<float>(a, cl, cn, false, fbar, ctx->hard, st);
    }
  }
  CKL();
  return PFEM_OK;
}

int ensure_tangent(pfem_ctx* ctx, int prec) {
  if (prec == PFEM_FP64 && !ctx->dK64) CK(dalloc(ctx, &ctx->dK64, (size_t)ctx->nnzb * 9));
  if (prec == PFEM_MIXED && !ctx->dK32) CK(dalloc(ctx, &ctx->dK32, (size_t)ctx->nnzb * 9));
  return PFEM_OK;
}

int check_status(pfem_ctx* ctx) {
  DevStatus s;
  CK(cudaMemcpyAsync(&s, ctx->dStatus, sizeof(s), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  if (s.code) {
    char buf[256];
    snprintf(buf, sizeof(buf),
             "ElementInversionError: element %lld, Gauss point %d is inverted (det F = J = %.6g <= 0)",
             s.e, s.g, s.J);
    return fail(ctx, PFEM_ERR_INVERTED_ELEMENT, buf);
  }
  return PFEM_OK;
}

// Assemble + impose Dirichlet at lambda; returns ||R|| of the imposed system.
int residual_system(pfem_ctx* ctx, int prec, double lam, double* rnorm, double* t_asm) {
  int rc = ensure_tangent(ctx, prec);
  if (rc) return rc;
  CK(cudaEventRecord(ctx->e0, ctx->st));
  rc = assemble_dev(ctx, prec, false);
  if (rc) return rc;
  CK(cudaEventRecord(ctx->e1, ctx->st));
  if (prec == PFEM_FP64) impose_dirichlet<double>(ctx->bc, ctx->ndof, lam, ctx->dU, ctx->dK64, ctx->dR, ctx->dDg, ctx->st);
  else impose_dirichlet<float>(ctx->bc, ctx->ndof, lam, ctx->dU, ctx->dK32, ctx->dR, ctx->dDg, ctx->st);
  CKL();
  dot<double>(ctx->ndof, ctx->dR, ctx->dR, ctx->dScal, ctx->dPart, ctx->st, true);
  CKL();
  CK(cudaMemcpyAsync(rnorm, ctx->dScal, sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  rc = check_status(ctx);  // synchronizes
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->e0, ctx->e1);
  if (t_asm) *t_asm += ms;
  ctx->tangent_prec = prec;
  return rc;
}

// Solve K dU = -R (device R) with precision prec; the correction stays in
// the precision-T Krylov vector kw.x.
int newton_correction(pfem_ctx* ctx, const pfem_solve_opts* o, double rtol, bool rebuild, int* kits,
                      double* t_amg, double* t_kry, bool* converged = nullptr, int itmax = -1) {
  if (itmax <= 0) itmax = o->krylov_itmax;
  const int prec = o->precision;
  int rc;
  auto t0 = std::chrono::steady_clock::now();
  if (prec == PFEM_FP64) {
    if (rebuild || !ctx->amg64.built) {
      rc = amg_setup<double>(ctx, o->cheb_degree);
      if (rc) return rc;
    } else {
      // reused hierarchy: the level-0 operator is the current tangent; the
      // smoother keeps the block-Jacobi inverse its Chebyshev interval was
      // estimated with (a fresh inverse under the old interval can diverge)
      ctx->amg64.lv[0].A.val = ctx->dK64;
    }
  } else {
    if (rebuild || !ctx->amg32.built) {
      rc = amg_setup<float>(ctx, o->cheb_degree);
      if (rc) return rc;
    } else {
      ctx->amg32.lv[0].A.val = ctx->dK32;
    }
  }
  CK(cudaStreamSynchronize(ctx->st));
  auto t1 = std::chrono::steady_clock::now();
  *t_amg += std::chrono::duration<double, std::milli>(t1 - t0).count();
  bool conv = false;
  if (prec == PFEM_FP64) {
    convert<double, double>(ctx->ndof, ctx->dR, ctx->kw64.b, -1.0, ctx->st);
    rc = krylov<double>(ctx, o->krylov, rtol, itmax, kits, &conv);
  } else {
    convert<double, float>(ctx->ndof, ctx->dR, ctx->kw32.b, -1.0, ctx->st);
    rc = krylov<float>(ctx, o->krylov, rtol, itmax, kits, &conv);
  }
  if (rc) return rc;
  CKL();
  CK(cudaStreamSynchronize(ctx->st));
  auto t2 = std::chrono::steady_clock::now();
  *t_kry += std::chrono::duration<double, std::milli>(t2 - t1).count();
  // an inexact inner solve is still a descent step; Newton judges it
  if (converged) *converged = conv;
  return PFEM_OK;
}

template <typename T>
__global__ void step_kernel(long long n, double a, const T* __restrict__ x, const double* __restrict__ u0,
                            double* __restrict__ u) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    u[i] = u0[i] + a * (double)x[i];
}

double forcing_term(const pfem_solve_opts* o, int it, double rk, double rkm1, double eta_prev) {
  // _forcing_term, Solver.jl:159-171
  if (it == 1 || rkm1 <= 0) return o->eta_max;
  double eta = o->ew_gamma * std::pow(rk / rkm1, o->ew_alpha);
  const double safe = o->ew_gamma * std::pow(eta_prev, o->ew_alpha);
  if (safe > 0.1) eta = std::max(eta, safe);
  return std::min(std::max(eta, o->eta_min), o->eta_max);
}

struct StepTimes {
  double asm_ms = 0, amg_ms = 0, kry_ms = 0, pred_ms = 0;
  int kits = 0;
};

// newton! (Solver.jl:317-389) at lambda from the current device U.  With
// o->line_search the step length is halved (at most 8 times) until the
// imposed FP64 residual norm drops; the full step is tried first and its
// assembly becomes the next iterate, so line search costs extra assemblies
// only when it backtracks.
int newton_dev(pfem_ctx* ctx, double lam, const pfem_solve_opts* o, int* iters, double* hist,
               int* khist, bool* converged, StepTimes* tm, bool have_first = false, double rn_first = 0.0) {
  *converged = false;
  const double fext_norm = std::fabs(lam) * ctx->fn_norm;
  double ref = 1.0, rkm1 = 0.0, eta_prev = o->eta_max;
  bool first = true, damped = false;
  double rn = rn_first;
  int rc = have_first ? PFEM_OK : residual_system(ctx, o->precision, lam, &rn, &tm->asm_ms);
  if (rc) return rc;
  int it;
  for (it = 1; it <= o->maxiter; ++it) {
    if (hist) hist[it - 1] = rn;
    if (it == 1) ref = std::max(std::max(rn, fext_norm), 1.0);
    if (o->verbose) fprintf(stderr, "    iter %d  |R| = %.6e\n", it, rn);
    if (!std::isfinite(rn)) return fail(ctx, PFEM_ERR_NOT_CONVERGED, "non-finite residual");
    if (rn <= o->tol * ref) {
      *converged = true;
      break;
    }
    if (it == o->maxiter) break;
    double eta = o->lin_rtol > 0 ? o->lin_rtol : forcing_term(o, it, rn, rkm1, eta_prev);
    // The step only has to bring |R| under the Newton test: a tighter inner solve in
    // the last iteration is wasted (Eisenstat-Walker's own safeguard; the reference
    // has none).  Half the needed reduction leaves room for the linearisation error.
    if (o->lin_rtol <= 0 && o->ew_need) eta = std::max(eta, std::min(o->eta_max, 0.5 * o->tol * ref / rn));
    // After a backtracked step the iterate is outside Newton's fast region; a
    // loose inner solve there gives poor directions, so tighten it.
    if (damped) eta = std::min(eta, 1e-3);
    // The first increment starts from U = 0 with the whole boundary-value jump; a loose
    // first direction there sends the line search into a long damped sequence
    // (measured at 64^3-100^3: 33-50 Newton iterations at eta_max = 0.1, 5-18 at 1e-2).
    if (o->lin_rtol <= 0 && o->eta_first > 0 && ctx->steps_taken == 0) eta = std::min(eta, o->eta_first);
    bool rebuild = o->amg_rebuild == 2 ? ctx->amg_stale : (first || o->amg_rebuild);
    first = false;
    int kits = 0;
    bool kconv = true;
    // A solve on a reused hierarchy that needs far more than its fresh rate is cut
    // short and redone on a rebuilt one (below), instead of running to convergence
    // on the stale hierarchy first.
    int cap = -1;
    if (o->amg_rebuild == 2 && !rebuild && ctx->amg_ipd_base > 0) {
      const double expect = ctx->amg_ipd_base * std::max(std::log10(1.0 / eta), 0.5);
      cap = std::min(o->krylov_itmax, std::max(12, (int)std::ceil(2.0 * (o->amg_stale_ratio * expect + 2))));
    }
    rc = newton_correction(ctx, o, eta, rebuild, &kits, &tm->amg_ms, &tm->kry_ms, &kconv, cap);
    if (rc) return rc;
    if (o->amg_rebuild == 2 && !rebuild && !kconv) {
      // a reused hierarchy that no longer reaches the tolerance: rebuild and solve again,
      // so the adaptive policy never takes a worse direction than the per-step rebuild
      tm->kits += kits;
      rebuild = true;
      rc = newton_correction(ctx, o, eta, true, &kits, &tm->amg_ms, &tm->kry_ms, &kconv);
      if (rc) return rc;
    }
    if (o->amg_rebuild == 2) {
      // iterations per decade of residual reduction asked of this solve
      const double dec = std::max(std::log10(1.0 / eta), 0.5);
      const double ipd = kits / dec;
      if (rebuild) {
        ctx->amg_ipd_base = ipd;
        ctx->amg_stale = false;
        ctx->amg_excess = 0.0;
        // what a rebuild costs, in Krylov iterations on the fresh hierarchy: a fixed
        // count, so that the policy's decisions (and the solution) do not depend on
        // timings (measured: set-up plus the CG graph's capture over one PCG iteration
        // is about 13 at 64^3 and 10 at 100^3)
        ctx->amg_cost_iters = kRebuildCostIters;
      } else {
        // stale when one solve needs amg_stale_ratio times the fresh rate, or when the
        // iterations spent above the fresh rate since the rebuild have cost more than
        // a rebuild would have
        const double expect = ctx->amg_ipd_base * dec;
        ctx->amg_excess += std::max(0.0, kits - expect);
        if (kits > o->amg_stale_ratio * expect + 2 || ctx->amg_excess > ctx->amg_cost_iters)
          ctx->amg_stale = true;
      }
    }
    if (khist) khist[it - 1] = kits;
    tm->kits += kits;
    rkm1 = rn;
    eta_prev = eta;
    CK(cudaMemcpyAsync(ctx->dUtmp, ctx->dU, ctx->ndof * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
    double a = 1.0, rt = 0.0;
    for (int bt = 0;; ++bt) {
      pfem::count_launch();
      if (o->precision == PFEM_FP64)
        step_kernel<double><<<1024, 256, 0, ctx->st>>>(ctx->ndof, a, ctx->kw64.x, ctx->dUtmp, ctx->dU);
      else
        step_kernel<float><<<1024, 256, 0, ctx->st>>>(ctx->ndof, a, ctx->kw32.x, ctx->dUtmp, ctx->dU);
      CKL();
      rc = residual_system(ctx, o->precision, lam, &rt, &tm->asm_ms);
      if (!o->line_search) {
        if (rc) return rc;
        break;
      }
      const bool inverted = rc == PFEM_ERR_INVERTED_ELEMENT;
      if (rc && !inverted) return rc;
      if (!inverted && std::isfinite(rt) && (rt < (1.0 - 1e-4 * a) * rn || bt >= 8)) break;
      if (bt >= 8) return rc ? rc : fail(ctx, PFEM_ERR_NOT_CONVERGED, "line search failed");
      a *= 0.5;
    }
    if (o->verbose) fprintf(stderr, "      eta %.2e  krylov %d  step %.4g\n", eta, kits, a);
    damped = a < 1.0;
    rn = rt;
  }
  *iters = std::min(it, o->maxiter);
  return PFEM_OK;
}

int commit_dev(pfem_ctx* ctx) {
  int rc = assemble_dev(ctx, PFEM_FP64, true);
  if (rc) return rc;
  return check_status(ctx);
}

__global__ void extrap_kernel(long long n, double f, const double* __restrict__ u1,
                              const double* __restrict__ u2, double* __restrict__ u) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    u[i] = u1[i] + f * (u1[i] - u2[i]);
}

__global__ void init_state_kernel(long long ngp, double* cpi, double* alpha, double* epsp, double* tau,
                                  double* beta) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ngp; i += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < 6; ++c) {
      cpi[c * ngp + i] = c < 3 ? 1.0 : 0.0;
      epsp[c * ngp + i] = 0.0;
      tau[c * ngp + i] = 0.0;
      if (beta) beta[c * ngp + i] = 0.0;
    }
    alpha[i] = 0.0;
  }
}

}  // namespace

template <typename T>
__global__ void diff_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                            T* __restrict__ x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = (T)(a[i] - b[i]);
}

// Smooth the learned correction Delta = U - Utmp (U the network's guess, Utmp
// the extrapolated one, whose imposed tangent K and residual R are resident)
// with `degree` block-Jacobi Chebyshev steps on K Delta = -R over
// [lmax/30, lmax]: the network's node-to-node scatter is high-frequency,
// exactly what the smoother removes, while the smooth part of its correction
// is kept.  lmax is the previous load step's estimate on the finest level.
template <typename T>
static int smooth_prediction(pfem_ctx* ctx, double lam, int degree) {
  Amg<T>& A = amg_of<T>(ctx);
  if (!A.built || degree <= 0) return PFEM_OK;
  KrylovWork<T>& w = kw_of<T>(ctx);
  AmgLevel<T>& v = A.lv[0];
  v.A.val = K_of<T>(ctx);
  blockdiag_invert<T>(v.A, v.dinv, ctx->st);
  convert<double, T>(ctx->ndof, ctx->dR, w.b, -1.0, ctx->st);
  pfem::count_launch();
  diff_kernel<T><<<1024, 256, 0, ctx->st>>>(ctx->ndof, ctx->dU, ctx->dUtmp, w.x);
  cheb<T>(ctx, v, degree, w.b, w.x, false);
  pfem::count_launch();
  step_kernel<T><<<1024, 256, 0, ctx->st>>>(ctx->ndof, 1.0, w.x, ctx->dUtmp, ctx->dU);
  bc_apply(ctx->bc, lam, ctx->dU, ctx->st);
  CKL();
  return PFEM_OK;
}

template <typename T>
static int amg_dense_t(pfem_ctx* ctx, int level, int what, double* out, int64_t* dims) {
  Amg<T>& A = amg_of<T>(ctx);
  const int L = (int)A.lv.size();
  if (!A.built || level < 0 || level > L || (what == 1 && level >= L) || (what == 2 && level != L) || what < 0 ||
      what > 2)
    return fail(ctx, PFEM_ERR_BAD_ARG, "no such AMG level");
  const HostLevel& h = ctx->hl[level];
  const int bs = h.bs, nr = h.nbrow * bs;
  if (what == 2) {  // the dense inverse of the coarsest level, as the cycle applies it
    const int n = A.coarse_n;
    if (dims) { dims[0] = n; dims[1] = n; }
    if (!out) return PFEM_OK;
    std::vector<T> v((size_t)n * n);
    CK(d2h(ctx, v.data(), A.coarse_inv, v.size() * sizeof(T)));
    for (size_t i = 0; i < v.size(); ++i) out[i] = (double)v[i];
    return PFEM_OK;
  }
  if (what == 0) {
    if (dims) { dims[0] = nr; dims[1] = nr; }
    if (!out) return PFEM_OK;
    // level 0 shares the tangent's block pattern
    const std::vector<int>& hrp = level == 0 ? ctx->browptr : h.rowptr;
    const std::vector<int>& hcl = level == 0 ? ctx->bcol : h.col;
    const long long nb = hrp[h.nbrow];
    std::vector<T> v((size_t)nb * bs * bs);
    const T* src = level < L ? A.lv[level].A.val : A.coarse_val;
    CK(d2h(ctx, v.data(), src, v.size() * sizeof(T)));
    std::fill(out, out + (size_t)nr * nr, 0.0);
    for (int I = 0; I < h.nbrow; ++I)
      for (int k = hrp[I]; k < hrp[I + 1]; ++k)
        for (int r = 0; r < bs; ++r)
          for (int c = 0; c < bs; ++c)
            out[(size_t)(I * bs + r) * nr + hcl[k] * bs + c] = (double)v[(size_t)k * bs * bs + r * bs + c];
  } else {
    const int nc = h.nagg * 6;
    if (dims) { dims[0] = nr; dims[1] = nc; }
    if (!out) return PFEM_OK;
    std::vector<T> v((size_t)h.p_cl.size() * bs * 6);
    CK(d2h(ctx, v.data(), A.lv[level].p_val, v.size() * sizeof(T)));
    std::fill(out, out + (size_t)nr * nc, 0.0);
    for (int n = 0; n < h.nbrow; ++n)
      for (int p = h.p_rp[n]; p < h.p_rp[n + 1]; ++p)
        for (int i = 0; i < bs; ++i)
          for (int c = 0; c < 6; ++c)
            out[(size_t)(n * bs + i) * nc + h.p_cl[p] * 6 + c] = (double)v[(size_t)p * bs * 6 + i * 6 + c];
  }
  return PFEM_OK;
}

// =====================================================================  C ABI
extern "C" {

void pfem_default_opts(pfem_solve_opts* o) {
  o->nsteps = 10;
  o->maxiter = 25;
  o->tol = 1e-8;
  o->precision = PFEM_FP64;
  o->krylov = PFEM_KRYLOV_CG;
  o->lin_rtol = -1.0;
  o->eta_min = 1e-8;
  o->eta_max = 0.1;
  o->ew_gamma = 0.9;
  o->ew_alpha = 1.5;
  o->krylov_itmax = 200;
  o->predictor = PFEM_PRED_PREVIOUS;
  o->amg_rebuild = 2;
  o->cheb_degree = 2;
  o->verbose = 0;
  o->line_search = 0;
  o->predictor_smooth = 8;  // whole 40-increment path at 64^3: 1.37 s (8), 1.40 s (16), 1.50 s (0)
  o->max_cuts = 0;
  o->eta_first = 1e-2;
  o->amg_stale_ratio = 1.5;
  o->ew_need = 1;
}

namespace {
// Block pattern and rank table on the device (topology.cu) for a context with
// a GPU: fills ctx->browptr / bcol (host copies for the AMG set-up and
// pfem_pattern) and leaves dElem, dBrowptr, dBcol and dRank on the device.
// Returns 1, with nothing kept, when a node has more incident elements than
// the kernel stages; the host path then builds the same pattern.
int device_pattern(pfem_ctx* ctx, const std::vector<int>& nptr, const std::vector<int>& nel) {
  const long long nn = ctx->nn, ne = ctx->ne;
  cudaStream_t st = ctx->st;
  int *dnptr = nullptr, *dnel = nullptr, *ddeg = nullptr, *derr = nullptr;
  CK(upload(ctx, &ctx->dElem, ctx->elem));
  CK(upload(ctx, &dnptr, nptr));
  CK(upload(ctx, &dnel, nel));
  CK(dalloc(ctx, &ddeg, (size_t)nn));
  CK(dalloc(ctx, &derr, 1));
  CK(cudaMemsetAsync(derr, 0, sizeof(int), st));
  launch_node_rows((int)nn, dnptr, dnel, ctx->dElem, nullptr, ddeg, nullptr, derr, st);
  CKL();
  int herr = 0;
  std::vector<int> deg(nn);
  CK(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(deg.data(), ddeg, nn * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  auto release = [&]() {
    dfree(ctx, dnptr); dfree(ctx, dnel); dfree(ctx, ddeg); dfree(ctx, derr);
  };
  if (herr) {
    release();
    dfree(ctx, ctx->dElem);
    return 1;
  }
  ctx->browptr.assign(nn + 1, 0);
  long long acc = 0;
  for (long long n = 0; n < nn; ++n) {
    acc += deg[n];
    if (acc * 9 >= (1ll << 31)) return fail(ctx, PFEM_ERR_BAD_ARG, "pattern too large for 32-bit indices");
    ctx->browptr[n + 1] = (int)acc;
  }
  CK(upload(ctx, &ctx->dBrowptr, ctx->browptr));
  CK(dalloc(ctx, &ctx->dBcol, (size_t)acc));
  launch_node_rows((int)nn, dnptr, dnel, ctx->dElem, ctx->dBrowptr, nullptr, ctx->dBcol, derr, st);
  CKL();
  CK(dalloc(ctx, &ctx->dRank, (size_t)ne * 64));
  launch_rank_table(ne, ctx->dElem, ctx->dBrowptr, ctx->dBcol, ctx->dRank, st);
  CKL();
  ctx->bcol.resize(acc);
  CK(cudaMemcpyAsync(ctx->bcol.data(), ctx->dBcol, acc * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  release();
  return PFEM_OK;
}
}  // namespace

const char* pfem_last_error(const pfem_ctx* ctx) {
  if (!ctx) return g_cuda_err.c_str();
  return ctx->err.c_str();
}

int pfem_create(pfem_ctx** out, const double* nodes, int64_t nn, const int64_t* elements, int64_t ne,
                int32_t kind, const pfem_material* m, const double* sigy0_e, int32_t device) {
  if (!out || !nodes || !elements || !m || nn <= 0 || ne <= 0) return PFEM_ERR_BAD_ARG;
  *out = nullptr;
  // J2Material guards, Materials.jl:90-103 (sigsat == 0 stands for the keyword
  // default sigsat = sigy0)
  if (!(m->E > 0) || !(m->nu > -1 && m->nu < 0.5) || !(m->sigy0 > 0) || !(m->Hiso >= 0) || !(m->Hkin >= 0)) {
    g_cuda_err = "invalid material parameters (E>0, -1<nu<0.5, sigy0>0, Hiso>=0, Hkin>=0)";
    return PFEM_ERR_BAD_ARG;
  }
  const double sigsat = m->sigsat == 0.0 ? m->sigy0 : m->sigsat;
  if (!(sigsat >= m->sigy0) || !(m->delta >= 0)) {
    g_cuda_err = "invalid saturation parameters (sigsat >= sigy0, delta >= 0)";
    return PFEM_ERR_BAD_ARG;
  }
  const bool voce = m->delta > 0 && sigsat > m->sigy0;
  if (voce && m->Hkin > 0) {
    g_cuda_err = "saturation hardening (sigsat > sigy0, delta > 0) with kinematic hardening (Hkin > 0) is not supported";
    return PFEM_ERR_BAD_ARG;
  }
  if (kind != PFEM_HEX8_SMALL && kind != PFEM_HEX8_FINITE && kind != PFEM_HEX8_FINITE_FBAR) {
    g_cuda_err = "kind must be PFEM_HEX8_SMALL, PFEM_HEX8_FINITE or PFEM_HEX8_FINITE_FBAR";
    return PFEM_ERR_BAD_ARG;
  }
  for (int64_t i = 0; i < 8 * ne; ++i)
    if (elements[i] < 1 || elements[i] > nn) {
      g_cuda_err = "element connectivity out of range (1-based node ids expected)";
      return PFEM_ERR_BAD_ARG;
    }
  if (sigy0_e)
    for (int64_t e = 0; e < ne; ++e)
      if (!(sigy0_e[e] > 0)) {
        g_cuda_err = "per-element sigy0 must be positive";
        return PFEM_ERR_BAD_ARG;
      }
  pfem_ctx* ctx = new pfem_ctx();
  ctx->device = device;
  ctx->nn = nn; ctx->ne = ne; ctx->ngp = 8 * ne; ctx->ndof = 3 * nn;
  ctx->kind = kind;
  ctx->mat.E = m->E; ctx->mat.nu = m->nu; ctx->mat.sigy0 = m->sigy0; ctx->mat.Hiso = m->Hiso; ctx->mat.Hkin = m->Hkin;
  ctx->mat.sigsat = sigsat; ctx->mat.delta = m->delta; ctx->mat.sat = sigsat - m->sigy0;
  ctx->hard = m->Hkin > 0 ? HARD_KIN : (voce ? HARD_VOCE : HARD_LINEAR);
  ctx->mat.G = m->E / (2.0 * (1.0 + m->nu));
  ctx->mat.K = m->E / (3.0 * (1.0 - 2.0 * m->nu));
  ctx->mat.lam = m->E * m->nu / ((1.0 + m->nu) * (1.0 - 2.0 * m->nu));
  auto bail = [&](int rc) {
    if (ctx->err.empty()) ctx->err = g_cuda_err;
    g_cuda_err = ctx->err;
    pfem_destroy(ctx);
    return rc;
  };
  if (device >= 0) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { pfem_set_cuda_error(e, "cudaSetDevice", __FILE__, __LINE__); return bail(PFEM_ERR_CUDA); }
    e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { pfem_set_cuda_error(e, "cudaStreamCreate", __FILE__, __LINE__); return bail(PFEM_ERR_CUDA); }
    cudaEventCreate(&ctx->e0);
    cudaEventCreate(&ctx->e1);
    cudaEventCreate(&ctx->t0);
    cudaEventCreate(&ctx->t1);
  }
  if ((long long)ctx->ndof >= (1ll << 31)) return bail(fail(ctx, PFEM_ERR_BAD_ARG, "mesh too large for 32-bit dof indices"));
  // ---- host topology ----
  ctx->X.assign(nodes, nodes + 3 * nn);
  ctx->elem.resize(8 * ne);
  for (int64_t i = 0; i < 8 * ne; ++i) ctx->elem[i] = (int)(elements[i] - 1);
  // node adjacency via node->element incidence
  std::vector<int> nptr(nn + 1, 0);
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) nptr[ctx->elem[e * 8 + a] + 1]++;
  for (int64_t n = 0; n < nn; ++n) nptr[n + 1] += nptr[n];
  std::vector<int> nel(nptr[nn]);
  {
    std::vector<int> f(nptr.begin(), nptr.end() - 1);
    for (int64_t e = 0; e < ne; ++e)
      for (int a = 0; a < 8; ++a) nel[f[ctx->elem[e * 8 + a]]++] = (int)e;
  }
  // block pattern: row n = sorted, distinct nodes of the elements incident to
  // n (Assembly.jl:62-82, :99-111).  With a GPU it is built on the device
  // (topology.cu); topology-only contexts, and meshes with a node in more than
  // 64 elements, build it here: two passes (count, fill) over rows of a few
  // dozen entries with one reused buffer per thread.
  bool dev_pattern = false;
  if (device >= 0) {
    const int rc = device_pattern(ctx, nptr, nel);
    if (rc < 0) return bail(rc);
    dev_pattern = rc == PFEM_OK;
  }
  if (!dev_pattern) {
    ctx->browptr.assign(nn + 1, 0);
    auto node_row = [&](long long n, std::vector<int>& buf) {
      buf.clear();
      for (int k = nptr[n]; k < nptr[n + 1]; ++k)
        for (int b = 0; b < 8; ++b) buf.push_back(ctx->elem[(long long)nel[k] * 8 + b]);
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
    };
    par_chunks(nn, [&](long long b, long long e) {
      std::vector<int> buf;
      for (long long n = b; n < e; ++n) {
        node_row(n, buf);
        ctx->browptr[n + 1] = (int)buf.size();
      }
    });
    long long acc = 0;
    for (int64_t n = 0; n < nn; ++n) {
      acc += ctx->browptr[n + 1];
      if (acc * 9 >= (1ll << 31)) return bail(fail(ctx, PFEM_ERR_BAD_ARG, "pattern too large for 32-bit indices"));
      ctx->browptr[n + 1] = (int)acc;
    }
    ctx->bcol.resize(ctx->browptr[nn]);
    par_chunks(nn, [&](long long b, long long e) {
      std::vector<int> buf;
      for (long long n = b; n < e; ++n) {
        node_row(n, buf);
        std::copy(buf.begin(), buf.end(), ctx->bcol.begin() + ctx->browptr[n]);
      }
    });
  }
  ctx->nnzb = ctx->browptr[nn];
  for (int64_t n = 0; n < nn; ++n)
    if (ctx->browptr[n + 1] - ctx->browptr[n] > 256)
      return bail(fail(ctx, PFEM_ERR_BAD_ARG, "a node has more than 256 neighbours (8-bit rank table)"));
  // rank[e][a][b] = position of node b in node a's block row (host path only;
  // the device path built it in place)
  std::vector<uint8_t> rank;
  if (!dev_pattern && device >= 0) {
    rank.resize((size_t)ne * 64);
    par_for(ne, [&](long long e) {
      for (int a = 0; a < 8; ++a) {
        const int na_ = ctx->elem[e * 8 + a];
        const int* b0 = ctx->bcol.data() + ctx->browptr[na_];
        const int* b1 = ctx->bcol.data() + ctx->browptr[na_ + 1];
        for (int b = 0; b < 8; ++b)
          rank[(size_t)e * 64 + a * 8 + b] = (uint8_t)(std::lower_bound(b0, b1, ctx->elem[e * 8 + b]) - b0);
      }
    });
  }
  // colors: the reference's rule is reported; the device uses it when it
  // yields independent sets (> 1 color), else a greedy coloring.
  ctx->ncolors_ref = reference_colors(ctx->X, nn, ne, ctx->color_ref);
  std::vector<int> col;
  int nc;
  if (ctx->ncolors_ref > 1) {
    col.assign(ctx->color_ref.begin(), ctx->color_ref.end());
    nc = ctx->ncolors_ref;
  } else {
    nc = greedy_colors(ctx->elem, nn, ne, col);
  }
  ctx->color_ptr.assign(nc + 1, 0);
  for (int64_t e = 0; e < ne; ++e) ctx->color_ptr[col[e] + 1]++;
  for (int c = 0; c < nc; ++c) ctx->color_ptr[c + 1] += ctx->color_ptr[c];
  std::vector<int> clist(ne), all(ne);
  {
    std::vector<int> f(ctx->color_ptr.begin(), ctx->color_ptr.end() - 1);
    for (int64_t e = 0; e < ne; ++e) clist[f[col[e]]++] = (int)e;
  }
  std::iota(all.begin(), all.end(), 0);
  for (int d = 0; d < 3; ++d) {
    double lo = 1e300, hi = -1e300;
    for (int64_t n = 0; n < nn; ++n) { lo = std::min(lo, ctx->X[n * 3 + d]); hi = std::max(hi, ctx->X[n * 3 + d]); }
    ctx->bbox_lo[d] = lo;
    ctx->bbox_ext[d] = hi > lo ? hi - lo : 1.0;
  }
  if (device < 0) {  // topology-only context: pattern / colors, no device work
    *out = ctx;
    return PFEM_OK;
  }
  // ---- device upload ----
  cudaError_t ce;
#define UP(ptr, vec) if ((ce = upload(ctx, &ptr, vec)) != cudaSuccess) { pfem_set_cuda_error(ce, #ptr, __FILE__, __LINE__); return bail(PFEM_ERR_CUDA); }
#define AL(ptr, n) if ((ce = dalloc(ctx, &ptr, n)) != cudaSuccess) { pfem_set_cuda_error(ce, #ptr, __FILE__, __LINE__); return bail(PFEM_ERR_CUDA); }
  UP(ctx->dX, ctx->X);
  if (!dev_pattern) {
    UP(ctx->dElem, ctx->elem);
    UP(ctx->dRank, rank);
    UP(ctx->dBrowptr, ctx->browptr);
    UP(ctx->dBcol, ctx->bcol);
  }
  UP(ctx->dColorList, clist);
  UP(ctx->dAllElems, all);
  {
    std::vector<uint8_t> nloc(nel.size());
    par_for(nn, [&](long long n) {
      for (int k = nptr[n]; k < nptr[n + 1]; ++k) {
        const int* en = ctx->elem.data() + (long long)nel[k] * 8;
        int a = 0;
        while (a < 7 && en[a] != (int)n) ++a;
        nloc[k] = (uint8_t)a;
      }
    });
    UP(ctx->dNptr, nptr);
    UP(ctx->dNel, nel);
    UP(ctx->dNloc, nloc);
    for (int64_t n = 0; n < nn; ++n) ctx->max_row = std::max(ctx->max_row, ctx->browptr[n + 1] - ctx->browptr[n]);
    // the block column ids as 16-bit offsets from the row (a node-ordered mesh's
    // neighbours lie within a few planes of nodes): the level-0 SpMV then reads 2
    // bytes per block instead of 4
    {
      std::vector<int16_t> c16(ctx->bcol.size());
      std::atomic<bool> fits{true};
      par_for(nn, [&](long long n) {
        for (int k = ctx->browptr[n]; k < ctx->browptr[n + 1]; ++k) {
          const long long d = (long long)ctx->bcol[k] - n;
          if (d < INT16_MIN || d > INT16_MAX) fits = false;
          else c16[k] = (int16_t)d;
        }
      });
      if (fits) UP(ctx->dBcol16, c16);
    }
    const char* am = getenv("PFEM_ASSEMBLY");
    ctx->colored_assembly = am && std::string(am) == "colored";
  }
  if (sigy0_e) {
    std::vector<double> s(sigy0_e, sigy0_e + ne);
    UP(ctx->dSigy, s);
  }
  AL(ctx->dCpi, 6 * ctx->ngp);
  AL(ctx->dAlpha, ctx->ngp);
  AL(ctx->dEpsp, 6 * ctx->ngp);
  if (ctx->hard == HARD_KIN) AL(ctx->dBeta, 6 * ctx->ngp);
  AL(ctx->dTau, 6 * ctx->ngp);
  AL(ctx->dFlags, ctx->ngp);
  AL(ctx->dU, ctx->ndof);
  AL(ctx->dR, ctx->ndof);
  AL(ctx->dDg, ctx->ndof);
  AL(ctx->dUprev, ctx->ndof);
  AL(ctx->dUprev2, ctx->ndof);
  AL(ctx->dUprev3, ctx->ndof);
  AL(ctx->dUtmp, ctx->ndof);
  AL(ctx->dScal, 16);
  AL(ctx->dPart, 2048);
  AL(ctx->dStatus, 1);
#undef UP
#undef AL
  int rc = pfem_reset(ctx);
  if (rc) return bail(rc);
  *out = ctx;
  return PFEM_OK;
}

void pfem_destroy(pfem_ctx* ctx) {
  if (!ctx) return;
  if (ctx->device < 0) {
    delete ctx;
    return;
  }
  cudaSetDevice(ctx->device);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  for (CgGraph* g : {&ctx->cg32, &ctx->cg64}) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->body_stream) cudaStreamDestroy(g->body_stream);
  }
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->e0) cudaEventDestroy(ctx->e0);
  if (ctx->e1) cudaEventDestroy(ctx->e1);
  if (ctx->t0) cudaEventDestroy(ctx->t0);
  if (ctx->t1) cudaEventDestroy(ctx->t1);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
}

int pfem_inversion_info(const pfem_ctx* ctx, int64_t* e, int32_t* g, double* J) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return PFEM_ERR_STATE;
  DevStatus s;
  if (d2h(ctx, &s, ctx->dStatus, sizeof(s)) != cudaSuccess) return PFEM_ERR_CUDA;
  if (e) *e = s.code ? s.e : 0;
  if (g) *g = s.code ? s.g : 0;
  if (J) *J = s.code ? s.J : 0.0;
  return PFEM_OK;
}

int pfem_pattern(const pfem_ctx* ctx, int64_t* nnz, int64_t* colptr, int64_t* rowval) {
  if (!ctx || !nnz) return PFEM_ERR_BAD_ARG;
  *nnz = ctx->nnzb * 9;
  if (!colptr && !rowval) return PFEM_OK;
  // Column j = 3n+c holds rows 3m+1..3m+3 for every neighbour m of n
  // (ascending): the count-then-fill layout of Assembly.jl:119-146.
  if (colptr) {
    colptr[0] = 1;
    for (long long n = 0; n < ctx->nn; ++n) {
      const int64_t d = 3 * (int64_t)(ctx->browptr[n + 1] - ctx->browptr[n]);
      for (int c = 0; c < 3; ++c) colptr[3 * n + c + 1] = colptr[3 * n + c] + d;
    }
  }
  if (rowval) {
    int64_t p = 0;
    for (long long n = 0; n < ctx->nn; ++n)
      for (int c = 0; c < 3; ++c)
        for (int k = ctx->browptr[n]; k < ctx->browptr[n + 1]; ++k) {
          const int64_t r0 = 3 * (int64_t)ctx->bcol[k];
          rowval[p++] = r0 + 1;
          rowval[p++] = r0 + 2;
          rowval[p++] = r0 + 3;
        }
  }
  return PFEM_OK;
}

int pfem_colors(const pfem_ctx* ctx, int32_t* ncolors, int64_t* color_of_element) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ncolors) *ncolors = ctx->ncolors_ref;
  if (color_of_element) std::copy(ctx->color_ref.begin(), ctx->color_ref.end(), color_of_element);
  return PFEM_OK;
}

int pfem_set_bcs(pfem_ctx* ctx, const int64_t* dir_dofs, const double* dir_vals, const uint8_t* dir_ramp,
                 int64_t ndir, const int64_t* neu_dofs, const double* neu_vals, int64_t nneu) {
  if (!ctx || ndir < 0 || nneu < 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  const long long ndof = ctx->ndof;
  // _freeze_bcs: last assignment wins (Solver.jl:192-218).  The entries are ordered
  // by dof (a stable sort keeps a dof's assignments in call order) and the last of
  // each run is kept: host work in the number of constraints, not of dofs, so that
  // per-increment updates stay cheap.
  for (int64_t i = 0; i < ndir; ++i)
    if (dir_dofs[i] < 1 || dir_dofs[i] > ndof) return fail(ctx, PFEM_ERR_BAD_ARG, "Dirichlet dof out of range");
  for (int64_t i = 0; i < nneu; ++i)
    if (neu_dofs[i] < 1 || neu_dofs[i] > ndof) return fail(ctx, PFEM_ERR_BAD_ARG, "Neumann dof out of range");
  std::vector<int64_t> order((size_t)ndir);
  for (int64_t i = 0; i < ndir; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t c) { return dir_dofs[a] < dir_dofs[c]; });
  std::vector<int> dofs;
  std::vector<double> vals;
  std::vector<uint8_t> ramp;
  for (int64_t k = 0; k < ndir; ++k) {
    const int64_t i = order[k];
    if (k + 1 < ndir && dir_dofs[order[k + 1]] == dir_dofs[i]) continue;  // a later assignment follows
    dofs.push_back((int)(dir_dofs[i] - 1));
    vals.push_back(dir_vals[i]);
    ramp.push_back(dir_ramp ? dir_ramp[i] : 1);
  }
  // the Neumann load vector is rebuilt (an O(ndof) pass and upload) only when it changed
  const bool same_neu = ctx->bcs_set && (size_t)nneu == ctx->neu_dofs_last.size() &&
                        std::equal(neu_dofs, neu_dofs + nneu, ctx->neu_dofs_last.begin()) &&
                        std::equal(neu_vals, neu_vals + nneu, ctx->neu_vals_last.begin());
  std::vector<double> fn;
  if (!same_neu) {
    fn.assign(ndof, 0.0);
    for (int64_t i = 0; i < nneu; ++i) fn[neu_dofs[i] - 1] += neu_vals[i];
    double s = 0;
    for (double v : fn) s += v * v;
    ctx->fn_norm = std::sqrt(s);
  }
  BcDev& b = ctx->bc;
  if (ctx->bcs_set && dofs == ctx->bc_dofs) {
    // same constrained dofs: the imposition lists stand, only values change
    // not usable until every copy has landed: a failed copy leaves the context
    // without boundary conditions rather than with a half-updated set
    ctx->bcs_set = false;
    CK(cudaStreamSynchronize(ctx->st));
    CK(h2d(ctx, b.vals, vals.data(), vals.size() * sizeof(double)));
    CK(h2d(ctx, b.ramp, ramp.data(), ramp.size() * sizeof(uint8_t)));
    if (!same_neu) {
      CK(h2d(ctx, b.fn, fn.data(), fn.size() * sizeof(double)));
      ctx->neu_dofs_last.assign(neu_dofs, neu_dofs + nneu);
      ctx->neu_vals_last.assign(neu_vals, neu_vals + nneu);
    }
    ctx->bcs_set = true;
    return PFEM_OK;
  }
  if (same_neu) {  // the constrained set changed but the loads did not: rebuild fn for the upload below
    fn.assign(ndof, 0.0);
    for (int64_t i = 0; i < nneu; ++i) fn[neu_dofs[i] - 1] += neu_vals[i];
  }
  std::vector<uint8_t> isbc(ndof, 0);
  for (int d : dofs) isbc[d] = 1;
  // entries touched by the imposition
  auto blk = [&](int n, int m) -> long long {
    const int* b0 = ctx->bcol.data() + ctx->browptr[n];
    const int* b1 = ctx->bcol.data() + ctx->browptr[n + 1];
    return ctx->browptr[n] + (long long)(std::lower_bound(b0, b1, m) - b0);
  };
  std::vector<std::pair<long long, uint8_t>> zl;
  std::vector<std::tuple<int, int, long long>> rl;  // (row, col, pos)
  for (int d : dofs) {
    const int n = d / 3, c = d % 3;
    for (int k = ctx->browptr[n]; k < ctx->browptr[n + 1]; ++k) {
      const int m = ctx->bcol[k];
      for (int j = 0; j < 3; ++j) zl.push_back({(long long)k * 9 + c * 3 + j, (uint8_t)(3 * m + j == d)});
      // column d: block (m, n), entry (i, c)
      const long long bk = blk(m, n);
      for (int i = 0; i < 3; ++i) {
        const int r = 3 * m + i;
        const long long pos = bk * 9 + i * 3 + c;
        zl.push_back({pos, (uint8_t)(r == d)});
        if (!isbc[r]) rl.emplace_back(r, d, pos);
      }
    }
  }
  std::sort(zl.begin(), zl.end());
  zl.erase(std::unique(zl.begin(), zl.end(), [](auto& a, auto& b) { return a.first == b.first; }), zl.end());
  std::sort(rl.begin(), rl.end());
  std::vector<int> rows, rptr(1, 0), rcol;
  std::vector<long long> rpos, zpos;
  std::vector<uint8_t> zone;
  for (size_t i = 0; i < rl.size(); ++i) {
    const int r = std::get<0>(rl[i]);
    if (rows.empty() || rows.back() != r) {
      if (!rows.empty()) rptr.push_back((int)rpos.size());
      rows.push_back(r);
    }
    rpos.push_back(std::get<2>(rl[i]));
    rcol.push_back(std::get<1>(rl[i]));
  }
  rptr.push_back((int)rpos.size());
  if (rows.empty()) rptr.assign(1, 0);
  for (auto& z : zl) { zpos.push_back(z.first); zone.push_back(z.second); }
  // the old lists go away before the new ones exist: until every upload below has
  // succeeded the context has no boundary conditions (a later call with the same
  // dofs must take this path again, not the value-only fast path above)
  ctx->bcs_set = false;
  ctx->bc_dofs.clear();
  dfree(ctx, b.dofs); dfree(ctx, b.vals); dfree(ctx, b.ramp); dfree(ctx, b.fn); dfree(ctx, b.rows);
  dfree(ctx, b.rptr); dfree(ctx, b.rpos); dfree(ctx, b.rcol); dfree(ctx, b.zpos); dfree(ctx, b.zone);
  b = BcDev();
  b.nbc = (int)dofs.size();
  b.nrows = (int)rows.size();
  b.nzero = (long long)zpos.size();
  CK(upload(ctx, &b.dofs, dofs));
  CK(upload(ctx, &b.vals, vals));
  CK(upload(ctx, &b.ramp, ramp));
  CK(upload(ctx, &b.fn, fn));
  CK(upload(ctx, &b.rows, rows));
  CK(upload(ctx, &b.rptr, rptr));
  CK(upload(ctx, &b.rpos, rpos));
  CK(upload(ctx, &b.rcol, rcol));
  CK(upload(ctx, &b.zpos, zpos));
  CK(upload(ctx, &b.zone, zone));
  ctx->bc_dofs = dofs;
  ctx->neu_dofs_last.assign(neu_dofs, neu_dofs + nneu);
  ctx->neu_vals_last.assign(neu_vals, neu_vals + nneu);
  ctx->bcs_set = true;
  ctx->amg_stale = true;  // a new constrained set changes the imposed tangent's structure
  return PFEM_OK;
}

int pfem_reset(pfem_ctx* ctx) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  pfem::count_launch(); init_state_kernel<<<1024, 256, 0, ctx->st>>>(ctx->ngp, ctx->dCpi, ctx->dAlpha, ctx->dEpsp, ctx->dTau,
                                                                     ctx->dBeta);
  CKL();
  CK(cudaMemsetAsync(ctx->dFlags, 0, ctx->ngp, ctx->st));
  CK(cudaMemsetAsync(ctx->dU, 0, ctx->ndof * sizeof(double), ctx->st));
  CK(cudaMemsetAsync(ctx->dUprev, 0, ctx->ndof * sizeof(double), ctx->st));
  CK(cudaMemsetAsync(ctx->dUprev2, 0, ctx->ndof * sizeof(double), ctx->st));
  CK(cudaMemsetAsync(ctx->dUprev3, 0, ctx->ndof * sizeof(double), ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  ctx->steps_taken = 0;
  ctx->amg_stale = true;
  ctx->mlp.used_count = 0;
  ctx->mlp.have_feat = false;
  ctx->lam_prev = ctx->lam_prev2 = ctx->lam_prev3 = 0.0;
  return PFEM_OK;
}

int pfem_set_state(pfem_ctx* ctx, const double* cpi, const double* alpha, const double* epsp) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  const long long ngp = ctx->ngp;
  auto put = [&](const double* h, double* d) -> int {
    std::vector<double> t(6 * ngp);
    for (long long g = 0; g < ngp; ++g)
      for (int k = 0; k < 6; ++k) t[k * ngp + g] = h[g * 6 + k];
    CK(h2d(ctx, d, t.data(), t.size() * sizeof(double)));
    return PFEM_OK;
  };
  int rc;
  if (cpi && (rc = put(cpi, ctx->dCpi))) return rc;
  if (epsp && (rc = put(epsp, ctx->dEpsp))) return rc;
  if (alpha) CK(h2d(ctx, ctx->dAlpha, alpha, ngp * sizeof(double)));
  return PFEM_OK;
}

int pfem_get_back_stress(const pfem_ctx* ctx, double* beta) {
  if (!ctx || !beta) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return PFEM_ERR_STATE;
  const long long ngp = ctx->ngp;
  if (!ctx->dBeta) {
    std::fill(beta, beta + 6 * ngp, 0.0);
    return PFEM_OK;
  }
  cudaSetDevice(ctx->device);
  if (cudaStreamSynchronize(ctx->st) != cudaSuccess) return PFEM_ERR_CUDA;
  std::vector<double> t(6 * ngp);
  if (d2h(ctx, t.data(), ctx->dBeta, t.size() * sizeof(double)) != cudaSuccess)
    return PFEM_ERR_CUDA;
  for (long long g = 0; g < ngp; ++g)
    for (int k = 0; k < 6; ++k) beta[g * 6 + k] = t[k * ngp + g];
  return PFEM_OK;
}

int pfem_set_back_stress(pfem_ctx* ctx, const double* beta) {
  if (!ctx || !beta) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (!ctx->dBeta) return fail(ctx, PFEM_ERR_BAD_ARG, "the model has no kinematic hardening (Hkin = 0)");
  cudaSetDevice(ctx->device);
  const long long ngp = ctx->ngp;
  std::vector<double> t(6 * ngp);
  for (long long g = 0; g < ngp; ++g)
    for (int k = 0; k < 6; ++k) t[k * ngp + g] = beta[g * 6 + k];
  CK(cudaStreamSynchronize(ctx->st));
  CK(h2d(ctx, ctx->dBeta, t.data(), t.size() * sizeof(double)));
  return PFEM_OK;
}

int pfem_set_displacement(pfem_ctx* ctx, const double* U) {
  if (!ctx || !U) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  CK(cudaMemcpyAsync(ctx->dU, U, ctx->ndof * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return PFEM_OK;
}

int pfem_assemble(pfem_ctx* ctx, const double* U, int32_t commit, int32_t precision, double* R, double* Kvals,
                  double* tau, uint8_t* flags) {
  if (!ctx || !U) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = pfem_set_displacement(ctx, U);
  if (rc) return rc;
  const int prec = precision == PFEM_MIXED ? PFEM_MIXED : PFEM_FP64;
  if (commit) {
    rc = commit_dev(ctx);
    if (rc) return rc;
  } else {
    rc = ensure_tangent(ctx, prec);
    if (rc) return rc;
    rc = assemble_dev(ctx, prec, false);
    if (rc) return rc;
    rc = check_status(ctx);
    if (rc) return rc;
    ctx->tangent_prec = -1;  // not imposed
  }
  if (R && !commit) CK(d2h(ctx, R, ctx->dR, ctx->ndof * sizeof(double)));
  if (Kvals && !commit) {
    const size_t nv = (size_t)ctx->nnzb * 9;
    std::vector<double> kv(nv);
    if (prec == PFEM_FP64) {
      CK(d2h(ctx, kv.data(), ctx->dK64, nv * sizeof(double)));
    } else {
      std::vector<float> kf(nv);
      CK(d2h(ctx, kf.data(), ctx->dK32, nv * sizeof(float)));
      for (size_t i = 0; i < nv; ++i) kv[i] = kf[i];
    }
    // block (n, m) entry (i, k) -> CSR row 3n+i, position 3*t + k in that row
    int64_t p = 0;
    for (long long n = 0; n < ctx->nn; ++n)
      for (int i = 0; i < 3; ++i)
        for (int k = ctx->browptr[n]; k < ctx->browptr[n + 1]; ++k)
          for (int c = 0; c < 3; ++c) Kvals[p++] = kv[(size_t)k * 9 + i * 3 + c];
  }
  return pfem_get_state(ctx, nullptr, tau, nullptr, nullptr, nullptr, flags);
}

static int mlp_alloc(pfem_ctx* ctx) {
  MlpState& m = ctx->mlp;
  if (m.alloc) return PFEM_OK;
  CK(dalloc(ctx, &m.w, MLP_NPARAMS)); CK(dalloc(ctx, &m.m, MLP_NPARAMS)); CK(dalloc(ctx, &m.v, MLP_NPARAMS));
  CK(dalloc(ctx, &m.g, MLP_NPARAMS)); CK(dalloc(ctx, &m.loss, 4)); CK(dalloc(ctx, &m.err, 4));
  char* f = nullptr;
  CK(dalloc(ctx, &f, (size_t)ctx->nn * 32));
  m.feat = f;
  CK(dalloc(ctx, &m.out, (size_t)ctx->nn * 3));
  CK(dalloc(ctx, &m.anode, (size_t)ctx->nn));
  CK(dalloc(ctx, &m.scale, 4));
  std::vector<float> val(ctx->nn, 0.0f);
  for (long long e = 0; e < ctx->ne; ++e)
    for (int a = 0; a < 8; ++a) val[ctx->elem[e * 8 + a]] += 1.0f;
  CK(upload(ctx, &m.valence, val));
  CK(cudaMemset(m.m, 0, MLP_NPARAMS * sizeof(float)));
  CK(cudaMemset(m.v, 0, MLP_NPARAMS * sizeof(float)));
  CK(cudaMemset(m.w, 0, MLP_NPARAMS * sizeof(float)));
  CK(cudaMemset(m.err, 0, 4 * sizeof(int)));
  m.alloc = true;
  return PFEM_OK;
}

static int mlp_check_err(pfem_ctx* ctx) {
  int e = 0;
  CK(d2h(ctx, &e, ctx->mlp.err, sizeof(int)));
  if (e) {
    cudaMemset(ctx->mlp.err, 0, sizeof(int));
    return fail(ctx, PFEM_ERR_CUDA, "tensor-core MMA wait timed out in the predictor kernel");
  }
  return PFEM_OK;
}

// Predictor for the load step to lambda.  Returns, when the learned guess was
// evaluated, the FP64 residual of the guess that was kept (its tangent is
// resident), so Newton can start from it without re-assembling.
static int step_begin(pfem_ctx* ctx, double lam, const pfem_solve_opts* o, StepTimes* tm, bool* have_first,
                      double* rn_first) {
  const long long n = ctx->ndof;
  *have_first = false;
  auto t0 = std::chrono::steady_clock::now();
  MlpState& ml = ctx->mlp;
  ml.have_feat = false;
  ml.last_r_ex = ml.last_r_ml = -1.0;
  ml.last_used = false;
  const double dl_prev = ctx->lam_prev - ctx->lam_prev2;
  const double r = dl_prev > 0 ? (lam - ctx->lam_prev) / dl_prev : 0.0;
  const double dl_prev2 = ctx->lam_prev2 - ctx->lam_prev3;
  const double rho = dl_prev2 > 0 ? dl_prev / dl_prev2 : 0.0;  // dU_n ~ rho dU_{n-1} when linear
  if (o->predictor != PFEM_PRED_PREVIOUS && ctx->steps_taken >= 1) {
    pfem::count_launch(); extrap_kernel<<<1024, 256, 0, ctx->st>>>(n, r, ctx->dUprev, ctx->dUprev2, ctx->dU);
    bc_apply(ctx->bc, lam, ctx->dU, ctx->st);
    CKL();
  }
  const bool want_learned = o->predictor == PFEM_PRED_LEARNED && ml.ready;
  if ((ml.recording || want_learned) && ctx->steps_taken >= 2 && o->predictor != PFEM_PRED_PREVIOUS) {
    int rc = mlp_alloc(ctx);
    if (rc) return rc;
    mlp_nodal_alpha(ctx->ne, ctx->nn, ctx->dElem, ctx->dAlpha, ml.valence, ml.anode, ctx->st);
    mlp_features(ctx->nn, ctx->dX, ctx->bbox_lo, ctx->bbox_ext, ctx->dUprev, ctx->dUprev2, ctx->dUprev3, ml.anode,
                 lam - ctx->lam_prev, lam, rho, ml.scale, ctx->dPart, ml.feat, ctx->st);
    CKL();
    ml.have_feat = true;
    ml.r_ratio = r;
  }
  if (want_learned && ml.have_feat) {
    // FP64 residual of the extrapolated guess, then of the learned one; keep the smaller.
    double r_ex = 0, r_ml = 0;
    int rc = residual_system(ctx, o->precision, lam, &r_ex, &tm->asm_ms);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->dUtmp, ctx->dU, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
    rc = mlp_launch(false, ml.w, ml.feat, nullptr, nullptr, ctx->nn, ml.out, nullptr, nullptr, ml.err, 148, ctx->st);
    if (rc) return fail(ctx, PFEM_ERR_CUDA, "predictor kernel launch failed");
    mlp_apply(ctx->nn, ctx->dUprev, ctx->dUprev2, r, ml.scale, ml.out, ctx->dU, ctx->st);
    bc_apply(ctx->bc, lam, ctx->dU, ctx->st);
    CKL();
    rc = mlp_check_err(ctx);
    if (rc) return rc;
    rc = o->precision == PFEM_FP64 ? smooth_prediction<double>(ctx, lam, o->predictor_smooth)
                                   : smooth_prediction<float>(ctx, lam, o->predictor_smooth);
    if (rc) return rc;
    rc = residual_system(ctx, o->precision, lam, &r_ml, &tm->asm_ms);
    if (o->verbose) fprintf(stderr, "  predictor: |R| extrapolated %.6e  learned %.6e\n", r_ex, r_ml);
    const bool learned_ok = rc == PFEM_OK && std::isfinite(r_ml) && r_ml < r_ex;
    if (rc && rc != PFEM_ERR_INVERTED_ELEMENT) return rc;
    ml.last_r_ex = r_ex;
    ml.last_r_ml = r_ml;
    ml.last_used = learned_ok;
    if (learned_ok) {
      ml.used_count++;
      *rn_first = r_ml;
    } else {
      CK(cudaMemcpyAsync(ctx->dU, ctx->dUtmp, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
      rc = residual_system(ctx, o->precision, lam, rn_first, &tm->asm_ms);
      if (rc) return rc;
    }
    *have_first = true;
  }
  CK(cudaStreamSynchronize(ctx->st));
  tm->pred_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return PFEM_OK;
}

static int step_end(pfem_ctx* ctx, double lam) {
  MlpState& ml = ctx->mlp;
  if (ml.recording && ml.have_feat && ml.ds_n + ctx->nn <= ml.ds_cap) {
    // training pair: features of this step, target = (dU_{n+1} - r dU_n) / s
    CK(cudaMemcpyAsync(static_cast<char*>(ml.ds_x) + (size_t)ml.ds_n * 32, ml.feat, (size_t)ctx->nn * 32,
                       cudaMemcpyDeviceToDevice, ctx->st));
    mlp_targets(ctx->nn, ctx->dU, ctx->dUprev, ctx->dUprev2, ml.r_ratio, ml.scale, ml.ds_t + (size_t)ml.ds_n * 3,
                ctx->st);
    CKL();
    ml.ds_n += ctx->nn;
  }
  CK(cudaMemcpyAsync(ctx->dUprev3, ctx->dUprev2, ctx->ndof * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->dUprev2, ctx->dUprev, ctx->ndof * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
  CK(cudaMemcpyAsync(ctx->dUprev, ctx->dU, ctx->ndof * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
  ctx->lam_prev3 = ctx->lam_prev2;
  ctx->lam_prev2 = ctx->lam_prev;
  ctx->lam_prev = lam;
  ctx->steps_taken++;
  return PFEM_OK;
}

int pfem_newton(pfem_ctx* ctx, double lambda, const pfem_solve_opts* o, int32_t* iters, double* res_hist,
                int32_t* krylov_hist) {
  if (!ctx || !o) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (!ctx->bcs_set) return fail(ctx, PFEM_ERR_STATE, "pfem_set_bcs must be called first");
  cudaSetDevice(ctx->device);
  StepTimes tm;
  bool hf = false;
  double r0 = 0;
  int rc = step_begin(ctx, lambda, o, &tm, &hf, &r0);
  if (rc) return rc;
  std::vector<int> kh(o->maxiter, 0);
  bool conv = false;
  int it = 0;
  rc = newton_dev(ctx, lambda, o, &it, res_hist, kh.data(), &conv, &tm, hf, r0);
  if (iters) *iters = it;
  if (krylov_hist) std::copy(kh.begin(), kh.end(), krylov_hist);
  if (rc) return rc;
  if (!conv) return fail(ctx, PFEM_ERR_NOT_CONVERGED, "load step did not converge");
  rc = commit_dev(ctx);
  if (rc) return rc;
  return step_end(ctx, lambda);
}

int pfem_predict(pfem_ctx* ctx, double lambda, const pfem_solve_opts* o, double* U, double* r_extrap,
                 double* r_learned, int32_t* learned_used) {
  if (!ctx || !o) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (!ctx->bcs_set) return fail(ctx, PFEM_ERR_STATE, "pfem_set_bcs must be called first");
  cudaSetDevice(ctx->device);
  StepTimes tm;
  bool hf = false;
  double r0 = 0;
  int rc = step_begin(ctx, lambda, o, &tm, &hf, &r0);
  if (rc) return rc;
  const MlpState& ml = ctx->mlp;
  if (r_extrap) *r_extrap = ml.last_r_ex;
  if (r_learned) *r_learned = ml.last_r_ml;
  if (learned_used) *learned_used = ml.last_used ? 1 : 0;
  if (r_extrap && ml.last_r_ex < 0) {
    rc = residual_system(ctx, o->precision, lambda, r_extrap, &tm.asm_ms);
    if (rc) return rc;
  }
  if (U) CK(d2h(ctx, U, ctx->dU, ctx->ndof * sizeof(double)));
  return PFEM_OK;
}

int pfem_solve(pfem_ctx* ctx, const pfem_solve_opts* o, pfem_solve_result* res, int32_t* iters_per_step,
               double* residuals, int32_t* krylov_per_iter) {
  if (!ctx || !o || o->nsteps <= 0 || o->maxiter <= 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (!ctx->bcs_set) return fail(ctx, PFEM_ERR_STATE, "pfem_set_bcs must be called first");
  cudaSetDevice(ctx->device);
  auto t0 = std::chrono::steady_clock::now();
  pfem_solve_result r;
  std::memset(&r, 0, sizeof(r));
  r.converged = 1;
  int rc = pfem_reset(ctx);
  if (rc) return rc;
  StepTimes tm;
  for (int n = 1; n <= o->nsteps && r.converged; ++n) {
    const double lam_n = (double)n / o->nsteps;
    double lam = lam_n;
    int cuts = 0;
    for (;;) {
      if (o->verbose) fprintf(stderr, "Load step %d/%d  (lambda=%g)\n", n, o->nsteps, lam);
      bool hf = false, conv = false;
      double r0 = 0;
      int it = 0;
      rc = step_begin(ctx, lam, o, &tm, &hf, &r0);
      if (rc == PFEM_OK)
        rc = newton_dev(ctx, lam, o, &it, residuals ? residuals + (size_t)(n - 1) * o->maxiter : nullptr,
                        krylov_per_iter ? krylov_per_iter + (size_t)(n - 1) * o->maxiter : nullptr, &conv, &tm, hf,
                        r0);
      r.newton_iters_total += it;
      if (iters_per_step) iters_per_step[n - 1] = it;  // the last attempt, matching its residual history
      const bool soft = rc == PFEM_ERR_NOT_CONVERGED || rc == PFEM_ERR_INVERTED_ELEMENT;
      if (rc && !soft) return rc;
      if (rc == PFEM_OK && conv) {
        rc = commit_dev(ctx);
        if (rc) return rc;
        rc = step_end(ctx, lam);
        if (rc) return rc;
        if (lam >= lam_n) break;
        lam = lam_n;  // a cut sub-step converged: go on to the load step's own load factor
        continue;
      }
      if (cuts >= o->max_cuts) {
        r.converged = 0;
        break;
      }
      // retry from the last converged state with half the increment
      ++cuts;
      ++r.load_step_cuts;
      CK(cudaMemcpyAsync(ctx->dU, ctx->dUprev, ctx->ndof * sizeof(double), cudaMemcpyDeviceToDevice, ctx->st));
      lam = ctx->lam_prev + 0.5 * (lam - ctx->lam_prev);
      ctx->err.clear();
      // the hierarchy was built on the abandoned attempt's iterates (possibly next to an
      // inverted element): the retry starts from a hierarchy of the converged state
      ctx->amg_stale = true;
    }
    if (r.converged) r.steps_done = n;
  }
  CK(cudaStreamSynchronize(ctx->st));
  r.krylov_iters_total = tm.kits;
  r.time_assembly_ms = tm.asm_ms;
  r.time_amg_setup_ms = tm.amg_ms;
  r.time_krylov_ms = tm.kry_ms;
  r.time_predictor_ms = tm.pred_ms;
  r.predictor_learned_used = ctx->mlp.used_count;
  r.time_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (res) *res = r;
  return r.converged ? PFEM_OK : fail(ctx, PFEM_ERR_NOT_CONVERGED, "a load step did not converge");
}

int pfem_residual(pfem_ctx* ctx, double lambda, int32_t precision, double* rnorm, double* R) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (!ctx->bcs_set) return fail(ctx, PFEM_ERR_STATE, "pfem_set_bcs must be called first");
  cudaSetDevice(ctx->device);
  double rn = 0, t = 0;
  int rc = residual_system(ctx, precision == PFEM_MIXED ? PFEM_MIXED : PFEM_FP64, lambda, &rn, &t);
  if (rc) return rc;
  if (rnorm) *rnorm = rn;
  if (R) CK(d2h(ctx, R, ctx->dR, ctx->ndof * sizeof(double)));
  return PFEM_OK;
}

int pfem_linear_solve(pfem_ctx* ctx, const double* b, double* x, double rtol, int32_t rebuild_pc,
                      const pfem_solve_opts* o, int32_t* niter) {
  if (!ctx || !b || !x || !o) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  if (ctx->tangent_prec < 0) return fail(ctx, PFEM_ERR_STATE, "no imposed tangent resident (run pfem_newton first)");
  cudaSetDevice(ctx->device);
  const int prec = ctx->tangent_prec;
  int rc;
  bool conv = false;
  int it = 0;
  std::vector<double> hb(b, b + ctx->ndof);
  if (prec == PFEM_FP64) {
    if (rebuild_pc || !ctx->amg64.built) { rc = amg_setup<double>(ctx, o->cheb_degree); if (rc) return rc; }
    ctx->amg64.lv[0].A.val = ctx->dK64;
    CK(h2d(ctx, ctx->kw64.b, hb.data(), ctx->ndof * sizeof(double)));
    rc = krylov<double>(ctx, o->krylov, rtol, o->krylov_itmax, &it, &conv);
    if (rc) return rc;
    CK(d2h(ctx, x, ctx->kw64.x, ctx->ndof * sizeof(double)));
  } else {
    if (rebuild_pc || !ctx->amg32.built) { rc = amg_setup<float>(ctx, o->cheb_degree); if (rc) return rc; }
    ctx->amg32.lv[0].A.val = ctx->dK32;
    std::vector<float> hf(hb.begin(), hb.end());
    CK(h2d(ctx, ctx->kw32.b, hf.data(), ctx->ndof * sizeof(float)));
    rc = krylov<float>(ctx, o->krylov, rtol, o->krylov_itmax, &it, &conv);
    if (rc) return rc;
    std::vector<float> xf(ctx->ndof);
    CK(d2h(ctx, xf.data(), ctx->kw32.x, ctx->ndof * sizeof(float)));
    for (long long i = 0; i < ctx->ndof; ++i) x[i] = xf[i];
  }
  if (niter) *niter = it;
  return conv ? PFEM_OK : fail(ctx, PFEM_ERR_LINSOLVE, "Krylov solve did not reach its tolerance");
}

int pfem_amg_apply(pfem_ctx* ctx, const double* r, double* z) {
  if (!ctx || !r || !z) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  const long long n = ctx->ndof;
  if (ctx->tangent_prec == PFEM_FP64 && ctx->amg64.built) {
    CK(h2d(ctx, ctx->kw64.r, r, n * sizeof(double)));
    vcycle<double>(ctx, 0, ctx->kw64.r, ctx->kw64.z);
    CKL();
    CK(d2h(ctx, z, ctx->kw64.z, n * sizeof(double)));
  } else if (ctx->tangent_prec == PFEM_MIXED && ctx->amg32.built) {
    std::vector<float> f(r, r + n);
    CK(h2d(ctx, ctx->kw32.r, f.data(), n * sizeof(float)));
    vcycle<float>(ctx, 0, ctx->kw32.r, ctx->kw32.z);
    CKL();
    CK(d2h(ctx, f.data(), ctx->kw32.z, n * sizeof(float)));
    for (long long i = 0; i < n; ++i) z[i] = f[i];
  } else {
    return fail(ctx, PFEM_ERR_STATE, "no AMG hierarchy built for the resident tangent");
  }
  return PFEM_OK;
}

int pfem_amg_dense(pfem_ctx* ctx, int32_t level, int32_t what, double* out, int64_t* dims) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  if (ctx->tangent_prec == PFEM_MIXED) return amg_dense_t<float>(ctx, level, what, out, dims);
  return amg_dense_t<double>(ctx, level, what, out, dims);
}

namespace {
// Component-major device state (c * ngp + gp) to the caller's per-GP layout
// (gp * 6 + c), optionally divided by a per-GP factor.
__global__ void soa_to_aos_kernel(long long ngp, const double* __restrict__ src, double* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ngp * 6; i += (long long)gridDim.x * blockDim.x) {
    const long long g = i / 6;
    const int c = (int)(i - g * 6);
    dst[i] = src[(long long)c * ngp + g];
  }
}

// Cauchy stress tau / det F with the standard F at every Gauss point
// (gauss_stress, Model.jl:188-208), one thread per Gauss point, written in the
// caller's per-GP layout.  det F <= 0 leaves tau unscaled, as the host rule did.
__global__ void cauchy_kernel(long long ne, const double* __restrict__ X, const int* __restrict__ elem,
                              const double* __restrict__ U, const double* __restrict__ tau,
                              double* __restrict__ out) {
  const long long ngp = ne * 8;
  const double gc = 0.57735026918962576451;
  for (long long gp = blockIdx.x * (long long)blockDim.x + threadIdx.x; gp < ngp; gp += (long long)gridDim.x * blockDim.x) {
    const long long e = gp >> 3;
    const int g = (int)(gp & 7);
    const double sgx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, sgy[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
                 sgz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    const double xi = sgx[g] * gc, et = sgy[g] * gc, ze = sgz[g] * gc;
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const double d0 = 0.125 * sgx[a] * (1 + sgy[a] * et) * (1 + sgz[a] * ze);
      const double d1 = 0.125 * sgy[a] * (1 + sgx[a] * xi) * (1 + sgz[a] * ze);
      const double d2 = 0.125 * sgz[a] * (1 + sgx[a] * xi) * (1 + sgy[a] * et);
      const long long n = elem[e * 8 + a];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double x = X[n * 3 + i], u = U[n * 3 + i];
        J[3 * i] += x * d0; J[3 * i + 1] += x * d1; J[3 * i + 2] += x * d2;
        H[3 * i] += u * d0; H[3 * i + 1] += u * d1; H[3 * i + 2] += u * d2;
      }
    }
    double Ji[9], F[9];
    pfem::inv3(J, Ji);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        F[3 * i + j] = (i == j ? 1.0 : 0.0) + H[3 * i] * Ji[j] + H[3 * i + 1] * Ji[3 + j] + H[3 * i + 2] * Ji[6 + j];
    const double dF = pfem::det3(F);
    const double inv = dF > 0 ? 1.0 / dF : 1.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) out[gp * 6 + c] = tau[(long long)c * ngp + gp] * inv;
  }
}

// Copy a component-major 6 x ngp device array to a host buffer in per-GP
// layout through the device scratch (one transpose on the device, one copy).
int download_aos(pfem_ctx* ctx, const double* d, double* h) {
  const long long ngp = ctx->ngp;
  if (!ctx->dOut) CK(dalloc(ctx, &ctx->dOut, (size_t)6 * ngp));
  pfem::count_launch();
  soa_to_aos_kernel<<<1024, 256, 0, ctx->st>>>(ngp, d, ctx->dOut);
  CKL();
  CK(cudaMemcpyAsync(h, ctx->dOut, (size_t)6 * ngp * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
  CK(cudaStreamSynchronize(ctx->st));
  return PFEM_OK;
}
}  // namespace

int pfem_get_state(const pfem_ctx* ctx, double* U, double* tau, double* alpha, double* cpi, double* epsp,
                   uint8_t* flags) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return PFEM_ERR_STATE;
  pfem_ctx* c = const_cast<pfem_ctx*>(ctx);
  cudaSetDevice(ctx->device);
  if (cudaStreamSynchronize(ctx->st) != cudaSuccess) return PFEM_ERR_CUDA;
  const long long ngp = ctx->ngp;
  if (U && d2h(ctx, U, ctx->dU, ctx->ndof * sizeof(double)) != cudaSuccess) return PFEM_ERR_CUDA;
  if (alpha && d2h(ctx, alpha, ctx->dAlpha, ngp * sizeof(double)) != cudaSuccess) return PFEM_ERR_CUDA;
  if (flags && d2h(ctx, flags, ctx->dFlags, ngp) != cudaSuccess) return PFEM_ERR_CUDA;
  if (tau && download_aos(c, ctx->dTau, tau)) return PFEM_ERR_CUDA;
  if (cpi && download_aos(c, ctx->dCpi, cpi)) return PFEM_ERR_CUDA;
  if (epsp && download_aos(c, ctx->dEpsp, epsp)) return PFEM_ERR_CUDA;
  return PFEM_OK;
}

int pfem_gauss_stress(const pfem_ctx* ctx, double* sigma) {
  if (!ctx || !sigma) return PFEM_ERR_BAD_ARG;
  // the small-strain kind stores sigma itself (Model.jl:188-208, small branch)
  if (ctx->kind == PFEM_HEX8_SMALL) return pfem_get_state(ctx, nullptr, sigma, nullptr, nullptr, nullptr, nullptr);
  if (ctx->device < 0) return PFEM_ERR_STATE;
  pfem_ctx* c = const_cast<pfem_ctx*>(ctx);
  cudaSetDevice(ctx->device);
  // tau / det F at each Gauss point with the standard F (Model.jl:188-208), on the device
  if (!c->dOut) {
    const cudaError_t e__ = dalloc(c, &c->dOut, (size_t)6 * ctx->ngp);
    if (e__ != cudaSuccess) { pfem_set_cuda_error(e__, "dOut", __FILE__, __LINE__); return cuda_fail(c); }
  }
  pfem::count_launch();
  cauchy_kernel<<<1024, 256, 0, ctx->st>>>(ctx->ne, ctx->dX, ctx->dElem, ctx->dU, ctx->dTau, c->dOut);
  {
    cudaError_t e__ = cudaGetLastError();
    if (e__ != cudaSuccess) { pfem_set_cuda_error(e__, "kernel launch", __FILE__, __LINE__); return cuda_fail(c); }
  }
  if (cudaMemcpyAsync(sigma, c->dOut, (size_t)6 * ctx->ngp * sizeof(double), cudaMemcpyDeviceToHost, ctx->st) !=
          cudaSuccess ||
      cudaStreamSynchronize(ctx->st) != cudaSuccess)
    return PFEM_ERR_CUDA;
  return PFEM_OK;
}

int pfem_profile(pfem_ctx* ctx, int32_t what, int32_t reps, double* ms) {
  if (!ctx || !ms || reps <= 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc;
  if (what == 0 || what == 1) {
    const int prec = what == 0 ? PFEM_FP64 : PFEM_MIXED;
    rc = ensure_tangent(ctx, prec);
    if (rc) return rc;
    rc = assemble_dev(ctx, prec, false);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->e0, ctx->st));
    for (int i = 0; i < reps; ++i) {
      rc = assemble_dev(ctx, prec, false);
      if (rc) return rc;
    }
    CK(cudaEventRecord(ctx->e1, ctx->st));
  } else if (what == 2 || what == 3) {
    if (!ctx->amg_struct) build_amg_structure(ctx);
    if (what == 2) {
      rc = ensure_tangent(ctx, PFEM_MIXED); if (rc) return rc;
      rc = amg_alloc<float>(ctx); if (rc) return rc;
      rc = krylov_alloc<float>(ctx); if (rc) return rc;
      BsrMat<float> A = ctx->amg32.lv[0].A;
      A.val = ctx->dK32;
      fill<float>(ctx->ndof, ctx->kw32.p, 1.0f, ctx->st);
      bsr_spmv<float>(A, ctx->kw32.p, ctx->kw32.q, ctx->st);
      CK(cudaEventRecord(ctx->e0, ctx->st));
      for (int i = 0; i < reps; ++i) bsr_spmv<float>(A, ctx->kw32.p, ctx->kw32.q, ctx->st);
      CK(cudaEventRecord(ctx->e1, ctx->st));
    } else {
      rc = ensure_tangent(ctx, PFEM_FP64); if (rc) return rc;
      rc = amg_alloc<double>(ctx); if (rc) return rc;
      rc = krylov_alloc<double>(ctx); if (rc) return rc;
      BsrMat<double> A = ctx->amg64.lv[0].A;
      A.val = ctx->dK64;
      fill<double>(ctx->ndof, ctx->kw64.p, 1.0, ctx->st);
      bsr_spmv<double>(A, ctx->kw64.p, ctx->kw64.q, ctx->st);
      CK(cudaEventRecord(ctx->e0, ctx->st));
      for (int i = 0; i < reps; ++i) bsr_spmv<double>(A, ctx->kw64.p, ctx->kw64.q, ctx->st);
      CK(cudaEventRecord(ctx->e1, ctx->st));
    }
  } else if (what == 4) {
    // one cycle of the resident FP32 hierarchy as it runs inside the CG loop: captured
    // once into a CUDA graph, replayed reps times
    if (!ctx->amg32.built) return fail(ctx, PFEM_ERR_STATE, "no FP32 AMG hierarchy built");
    KrylovWork<float>& w = ctx->kw32;
    fill<float>(ctx->ndof, w.r, 1.0f, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
    const long long c0 = pfem::launch_counter();
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
    vcycle<float>(ctx, 0, w.r, w.z);
    cudaError_t e = cudaStreamEndCapture(ctx->st, &g);
    pfem::launch_counter() = c0;  // counted when replayed below, not when captured
    if (e != cudaSuccess) return fail(ctx, PFEM_ERR_CUDA, std::string("cycle capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ge, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(ctx, PFEM_ERR_CUDA, std::string("cycle graph instantiate: ") + cudaGetErrorString(e));
    }
    size_t nodes = 0;
    cudaGraphGetNodes(g, nullptr, &nodes);
    e = cudaGraphLaunch(ge, ctx->st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->e0, ctx->st);
    for (int i = 0; i < reps && e == cudaSuccess; ++i) e = cudaGraphLaunch(ge, ctx->st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->e1, ctx->st);
    if (e == cudaSuccess) e = cudaEventSynchronize(ctx->e1);
    pfem::launch_counter() += (long long)nodes * (reps + 1);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ctx, PFEM_ERR_CUDA, std::string("cycle graph replay: ") + cudaGetErrorString(e));
  } else {
    return PFEM_ERR_BAD_ARG;
  }
  CKL();
  CK(cudaEventSynchronize(ctx->e1));
  float t = 0;
  CK(cudaEventElapsedTime(&t, ctx->e0, ctx->e1));
  *ms = t / reps;
  return PFEM_OK;
}

int64_t pfem_kernel_launches(void) { return (int64_t)g_launches; }

int pfem_tangent_index_bytes(pfem_ctx* ctx, int32_t* bytes) {
  if (!ctx || !bytes) return PFEM_ERR_BAD_ARG;
  *bytes = ctx->dBcol16 ? 2 : 4;
  return PFEM_OK;
}

int pfem_mlp_init(pfem_ctx* ctx, uint64_t seed) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = mlp_alloc(ctx);
  if (rc) return rc;
  // He-uniform weights (fan-in of the real inputs), zero biases; padding stays zero.
  std::vector<float> p(MLP_NPARAMS, 0.0f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (double)((st >> 11) & ((1ull << 53) - 1)) / (double)(1ull << 53) * 2.0 - 1.0;
  };
  const int H = 128;
  for (int h = 0; h < H; ++h)
    for (int i = 0; i < MLP_NFEAT; ++i) p[h * 16 + i] = (float)(uni() * std::sqrt(6.0 / MLP_NFEAT));
  const int oW2 = H * 16 + H;
  for (int i = 0; i < H * H; ++i) p[oW2 + i] = (float)(uni() * std::sqrt(6.0 / H));
  const int oW3 = oW2 + H * H + H;
  for (int o = 0; o < 3; ++o)
    for (int h = 0; h < H; ++h) p[oW3 + o * H + h] = (float)(uni() * std::sqrt(6.0 / H) * 0.1);
  CK(h2d(ctx, ctx->mlp.w, p.data(), p.size() * sizeof(float)));
  CK(cudaMemset(ctx->mlp.m, 0, MLP_NPARAMS * sizeof(float)));
  CK(cudaMemset(ctx->mlp.v, 0, MLP_NPARAMS * sizeof(float)));
  ctx->mlp.adam_t = 0;
  ctx->mlp.ready = false;
  return PFEM_OK;
}

int pfem_mlp_params(pfem_ctx* ctx, int32_t op, float* p, int64_t n) {
  if (!ctx || !p || n != MLP_NPARAMS) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = mlp_alloc(ctx);
  if (rc) return rc;
  if (op == 0) {
    CK(d2h(ctx, p, ctx->mlp.w, MLP_NPARAMS * sizeof(float)));
  } else {
    CK(h2d(ctx, ctx->mlp.w, p, MLP_NPARAMS * sizeof(float)));
    ctx->mlp.ready = true;
  }
  return PFEM_OK;
}

int pfem_mlp_forward(pfem_ctx* ctx, const float* feats, int64_t n, float* out) {
  if (!ctx || !feats || !out || n <= 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = mlp_alloc(ctx);
  if (rc) return rc;
  float *df = nullptr, *dy = nullptr;
  char* db = nullptr;
  TmpDev tmp;
  CK(tmp.alloc(&df, (size_t)n * MLP_NFEAT * sizeof(float)));
  CK(tmp.alloc(&db, (size_t)n * 32));
  CK(tmp.alloc(&dy, (size_t)n * 3 * sizeof(float)));
  CK(h2d(ctx, df, feats, (size_t)n * MLP_NFEAT * sizeof(float)));
  mlp_pack_features(df, n, db, ctx->st);
  rc = mlp_launch(false, ctx->mlp.w, db, nullptr, nullptr, n, dy, nullptr, nullptr, ctx->mlp.err, 148, ctx->st);
  CK(cudaStreamSynchronize(ctx->st));
  CK(d2h(ctx, out, dy, (size_t)n * 3 * sizeof(float)));
  if (rc) return fail(ctx, PFEM_ERR_CUDA, "predictor kernel launch failed");
  return mlp_check_err(ctx);
}

int pfem_mlp_loss_grad(pfem_ctx* ctx, const float* feats, const float* targets, int64_t n, float* grad, float* loss) {
  if (!ctx || !feats || !targets || n <= 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = mlp_alloc(ctx);
  if (rc) return rc;
  float *df = nullptr, *dt = nullptr;
  char* db = nullptr;
  TmpDev tmp;
  CK(tmp.alloc(&df, (size_t)n * MLP_NFEAT * sizeof(float)));
  CK(tmp.alloc(&db, (size_t)n * 32));
  CK(tmp.alloc(&dt, (size_t)n * 3 * sizeof(float)));
  CK(h2d(ctx, df, feats, (size_t)n * MLP_NFEAT * sizeof(float)));
  CK(h2d(ctx, dt, targets, (size_t)n * 3 * sizeof(float)));
  mlp_pack_features(df, n, db, ctx->st);
  CK(cudaMemsetAsync(ctx->mlp.g, 0, MLP_NPARAMS * sizeof(float), ctx->st));
  CK(cudaMemsetAsync(ctx->mlp.loss, 0, sizeof(float), ctx->st));
  rc = mlp_launch(true, ctx->mlp.w, db, dt, nullptr, n, nullptr, ctx->mlp.g, ctx->mlp.loss, ctx->mlp.err, 148,
                  ctx->st);
  CK(cudaStreamSynchronize(ctx->st));
  if (grad) CK(d2h(ctx, grad, ctx->mlp.g, MLP_NPARAMS * sizeof(float)));
  float l = 0;
  CK(d2h(ctx, &l, ctx->mlp.loss, sizeof(float)));
  if (loss) *loss = l / (3.0f * (float)n);
  if (rc) return fail(ctx, PFEM_ERR_CUDA, "predictor kernel launch failed");
  return mlp_check_err(ctx);
}

int pfem_mlp_record(pfem_ctx* ctx, int32_t op, int64_t capacity, int64_t* size) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  int rc = mlp_alloc(ctx);
  if (rc) return rc;
  MlpState& m = ctx->mlp;
  if (op == 0) {
    if (capacity > m.ds_cap) {
      if (m.ds_x) { cudaFree(m.ds_x); cudaFree(m.ds_t); }
      m.ds_x = nullptr; m.ds_t = nullptr;
      CK(cudaMalloc(&m.ds_x, (size_t)capacity * 32));
      CK(cudaMalloc((void**)&m.ds_t, (size_t)capacity * 3 * sizeof(float)));
      m.ds_cap = capacity;
    }
    m.recording = true;
  } else if (op == 1) {
    m.recording = false;
  } else if (op == 2) {
    m.ds_n = 0;
  }
  if (size) *size = m.ds_n;
  return PFEM_OK;
}

int pfem_mlp_train(pfem_ctx* ctx, int32_t steps, int32_t batch, float lr, uint64_t seed, float* losses) {
  if (!ctx || steps <= 0 || batch <= 0) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  MlpState& m = ctx->mlp;
  if (!m.alloc || m.ds_n <= 0) return fail(ctx, PFEM_ERR_STATE, "no recorded training samples");
  if (batch > m.rows_cap) {
    int* r = nullptr;
    CK(dalloc(ctx, &r, (size_t)batch));
    m.rows = r;
    m.rows_cap = batch;
  }
  float* dl = nullptr;
  TmpDev tmp;
  CK(tmp.alloc(&dl, (size_t)steps * sizeof(float)));
  int rc = 0;
  for (int k = 0; k < steps; ++k) {
    mlp_random_rows(batch, m.ds_n, seed * 1000003ull + (uint64_t)k, m.rows, ctx->st);
    CK(cudaMemsetAsync(m.g, 0, MLP_NPARAMS * sizeof(float), ctx->st));
    CK(cudaMemsetAsync(dl + k, 0, sizeof(float), ctx->st));
    rc |= mlp_launch(true, m.w, m.ds_x, m.ds_t, m.rows, batch, nullptr, m.g, dl + k, m.err, 148, ctx->st);
    mlp_adam(m.w, m.m, m.v, m.g, lr, ++m.adam_t, ctx->st);
  }
  CK(cudaStreamSynchronize(ctx->st));
  if (losses) {
    std::vector<float> h(steps);
    CK(d2h(ctx, h.data(), dl, (size_t)steps * sizeof(float)));
    for (int k = 0; k < steps; ++k) losses[k] = h[k] / (3.0f * (float)batch);
  }
  if (rc) return fail(ctx, PFEM_ERR_CUDA, "predictor training kernel launch failed");
  rc = mlp_check_err(ctx);
  if (rc) return rc;
  m.ready = true;
  return PFEM_OK;
}

int pfem_timer(pfem_ctx* ctx, int32_t op, double* ms) {
  if (!ctx) return PFEM_ERR_BAD_ARG;
  if (ctx->device < 0) return fail(ctx, PFEM_ERR_STATE, "topology-only context (device < 0)");
  cudaSetDevice(ctx->device);
  if (op == 0) {
    CK(cudaEventRecord(ctx->t0, ctx->st));
    return PFEM_OK;
  }
  CK(cudaEventRecord(ctx->t1, ctx->st));
  CK(cudaEventSynchronize(ctx->t1));
  float t = 0;
  CK(cudaEventElapsedTime(&t, ctx->t0, ctx->t1));
  if (ms) *ms = t;
  return PFEM_OK;
}

}  // extern "C"
