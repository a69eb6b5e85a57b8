// topology.cu -- one-time mesh set-up on the device: the block pattern of the
// tangent (node adjacency through shared elements, lagrangian/src/
// Assembly.jl:62-82 and the pattern of build_sparsity :99-111, here at 3 x 3
// block granularity) and the per-element rank table the colored scatter uses
// instead of the reference's per-entry binary searches (:210-224).
#include <cstdint>

#include "common.cuh"
#include "pfem_internal.h"

namespace pfem {

constexpr int TOPO_WARPS = 8;    // warps per block
constexpr int TOPO_CAP = 512;    // candidates staged per warp: 64 incident elements

// A warp per node n.  Its candidates are the eight nodes of each incident
// element (8 m of them, duplicates included), staged in shared memory; a
// candidate is kept when no earlier one has the same value.  Count pass
// (col == null): deg[n] = number of distinct nodes.  Fill pass: each distinct
// node goes to rowptr[n] + (number of distinct nodes below it), so the row
// comes out sorted without a sort.  A node with more than TOPO_CAP / 8
// incident elements sets *err and is skipped (the caller then builds the
// pattern on the host).
__global__ void __launch_bounds__(32 * TOPO_WARPS)
node_rows_kernel(int nn, const int* __restrict__ nptr, const int* __restrict__ nel, const int* __restrict__ elem,
                 const int* __restrict__ rowptr, int* __restrict__ deg, int* __restrict__ col, int* __restrict__ err) {
  __shared__ int buf[TOPO_WARPS][TOPO_CAP];
  __shared__ unsigned char first[TOPO_WARPS][TOPO_CAP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (long long n = (long long)blockIdx.x * TOPO_WARPS + w; n < nn; n += (long long)gridDim.x * TOPO_WARPS) {
    const int k0 = nptr[n];
    const int m = 8 * (nptr[n + 1] - k0);
    if (m > TOPO_CAP) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    for (int i = lane; i < m; i += 32) buf[w][i] = elem[(long long)nel[k0 + (i >> 3)] * 8 + (i & 7)];
    __syncwarp();
    int cnt = 0;
    for (int i = lane; i < m; i += 32) {
      const int v = buf[w][i];
      bool f = true;
      for (int j = 0; j < i && f; ++j) f = buf[w][j] != v;
      first[w][i] = f ? 1 : 0;
      cnt += f ? 1 : 0;
    }
    __syncwarp();
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (!col) {
      if (lane == 0) deg[n] = cnt;
    } else {
      const int base = rowptr[n];
      for (int i = lane; i < m; i += 32) {
        if (!first[w][i]) continue;
        const int v = buf[w][i];
        int pos = 0;
        for (int j = 0; j < m; ++j) pos += (first[w][j] && buf[w][j] < v) ? 1 : 0;
        col[base + pos] = v;
      }
    }
    __syncwarp();
  }
}

// rank[e][a][b] = position of node b of element e in node a's block row
// (lower bound in the sorted row), one thread per (e, a).
__global__ void rank_table_kernel(long long ne, const int* __restrict__ elem, const int* __restrict__ rowptr,
                                  const int* __restrict__ col, uint8_t* __restrict__ rank) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ne * 8;
       t += (long long)gridDim.x * blockDim.x) {
    const long long e = t >> 3;
    const int a = (int)(t & 7);
    const int na = elem[e * 8 + a];
    const int lo0 = rowptr[na], hi0 = rowptr[na + 1];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int v = elem[e * 8 + b];
      int lo = lo0, hi = hi0;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (col[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      rank[e * 64 + a * 8 + b] = (uint8_t)(lo - lo0);
    }
  }
}

void launch_node_rows(int nn, const int* nptr, const int* nel, const int* elem, const int* rowptr, int* deg,
                      int* col, int* err, cudaStream_t st) {
  if (nn <= 0) return;
  const long long want = ((long long)nn + TOPO_WARPS - 1) / TOPO_WARPS;
  const int blocks = (int)(want < 148 * 16 ? want : 148 * 16);
  count_launch();
  node_rows_kernel<<<blocks, 32 * TOPO_WARPS, 0, st>>>(nn, nptr, nel, elem, rowptr, deg, col, err);
}

void launch_rank_table(long long ne, const int* elem, const int* rowptr, const int* col, uint8_t* rank,
                       cudaStream_t st) {
  if (ne <= 0) return;
  const long long want = (ne * 8 + 255) / 256;
  const int blocks = (int)(want < 148 * 16 ? want : 148 * 16);
  count_launch();
  rank_table_kernel<<<blocks, 256, 0, st>>>(ne, elem, rowptr, col, rank);
}

}  // namespace pfem
