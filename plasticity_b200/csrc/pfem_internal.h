// pfem_internal.h -- device-side data structures shared by the CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>
#include "common.cuh"
#include "../../include/pfem_b200.h"

namespace pfem {

template <typename KT>
struct ElemArgs {
  const double* X;         // nn x 3 node coordinates (node-major)
  const int* elem;         // ne x 8 node ids (0-based)
  const double* U;         // ndof displacements
  double* cpi;             // 6 x ngp committed Cp^-1 (component-major SoA)
  double* alpha;           // ngp committed equivalent plastic strain
  double* epsp;            // 6 x ngp accumulated plastic strain (diagnostic)
  double* beta;            // 6 x ngp committed back stress (HARD_KIN only; reference
                           // configuration for the finite kinds), else null
  const double* sigy0_e;   // ne per-element initial yield stress, or null
  double* tau;             // 6 x ngp Kirchhoff stress of the last evaluation
  uint8_t* flags;          // ngp elastic(0)/plastic(1) of the last evaluation
  double* R;               // ndof internal force (accumulated)
  KT* Kval;                // nnzb x 9 block-CSR tangent values (accumulated)
  const int* browptr;      // nn+1 block row pointers
  const uint8_t* rank;     // ne x 64: position of node b in node a's block row
  // Element-ordered outputs (the gathered assembly): when set, the kernel writes
  // K_e as Kbuf[e][a][i][(b,k)] (576 values: rows of node a together) and F_e as
  // Fbuf[e][a][i] (24 doubles) instead of adding into Kval and R.
  KT* Kbuf;
  double* Fbuf;
  long long ngp;
  MatParams mat;
  DevStatus* status;
};

template <typename KT>
void launch_element_color(const ElemArgs<KT>& a, const int* elist, int n, bool commit, bool fbar,
                          int hard, cudaStream_t st);
// Small-strain kind (Elements.jl:323-360): epsp holds the committed plastic
// strain, tau receives sigma; cpi is unused.
template <typename KT>
void launch_element_small(const ElemArgs<KT>& a, const int* elist, int n, bool commit, int hard,
                          cudaStream_t st);

// Row-owned gather (element.cu): block row a of K and R[a] are the sums, over
// the elements incident to node a in increasing element order (nptr/nel, with
// nloc the node's position in the element), of the element buffers' (a, b)
// blocks and force rows.  Every block of K and every entry of R is written once.
template <typename KT>
void launch_gather_rows(int nn, const int* nptr, const int* nel, const uint8_t* nloc, const int* browptr,
                        const uint8_t* rank, const KT* Kbuf, const double* Fbuf, KT* Kval, double* R, int maxlen,
                        cudaStream_t st);

// One-time topology on the device (topology.cu): per-node block rows
// (count pass with col = null, fill pass with rowptr) and the rank table.
void launch_node_rows(int nn, const int* nptr, const int* nel, const int* elem, const int* rowptr, int* deg,
                      int* col, int* err, cudaStream_t st);
void launch_rank_table(long long ne, const int* elem, const int* rowptr, const int* col, uint8_t* rank,
                       cudaStream_t st);

// ---------------- block-CSR matrices ----------------
template <typename VT>
struct BsrMat {
  int nbrow = 0;     // block rows (== block cols)
  int bs = 0;        // block size
  long long nnzb = 0;
  int* rowptr = nullptr;  // device, nbrow+1
  int* col = nullptr;     // device, nnzb
  VT* val = nullptr;      // device, nnzb*bs*bs (row-major blocks)
  // optional, device: col[k] - row as 16-bit offsets (set when every offset fits),
  // read by the SpMV in place of col
  const int16_t* col16 = nullptr;
};

// One level of smoothed-aggregation AMG.  Every fine block row n belongs to
// one aggregate agg[n] and carries the tentative bs x 6 block T_n (the six
// rigid-body modes, orthonormalised per aggregate).  The prolongator is
// P = (I - w D^-1 A) T in block-CSR form (bs x 6 blocks, columns = aggregates);
// AP is kept for the Galerkin product P^T A P that forms the next level.
template <typename VT>
struct AmgLevel {
  BsrMat<VT> A;
  VT* dinv = nullptr;     // nbrow x bs x bs inverse diagonal blocks
  VT lmax = 0;            // spectral radius estimate of D^-1 A (x 1.1)
  int nagg = 0;
  int* agg = nullptr;     // nbrow aggregate of each block row
  VT* T = nullptr;        // nbrow x bs x 6
  int nnzP = 0;
  int *p_rp = nullptr, *p_cl = nullptr, *p_row = nullptr;  // P pattern (+ row of each block)
  VT* p_val = nullptr;
  int* pslot = nullptr;   // per A block: the P block of its row whose column is agg(col)
  int *pt_rp = nullptr, *pt_blk = nullptr;  // P^T: P blocks of each aggregate
  int* pt_row = nullptr;  // P^T order: the fine block row of each block
  VT* pt_val = nullptr;   // P^T order: a copy of the P blocks, streamed by the restriction
  int nnzAP = 0;
  int *ap_rp = nullptr, *ap_cl = nullptr, *ap_row = nullptr;
  VT* ap_val = nullptr;
  int *c_row = nullptr, *c_cl = nullptr;    // next level's pattern with the row of each block
  // work vectors (length nbrow*bs)
  VT *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *t = nullptr;
  // second coarse iteration of a W-cycle visit (levels >= 2): its right-hand side and result
  VT *b2 = nullptr, *x2 = nullptr;
};

template <typename VT>
struct Amg {
  std::vector<AmgLevel<VT>> lv;
  int coarse_n = 0;          // dofs of the coarsest level
  long long coarse_nnzb = 0;
  VT* coarse_val = nullptr;  // Galerkin operator of the coarsest level (6 x 6 blocks)
  int *coarse_rp = nullptr, *coarse_cl = nullptr;  // its block pattern (device)
  VT* coarse_inv = nullptr;  // coarse_n x coarse_n dense inverse (row-major)
  VT *cx = nullptr, *cb = nullptr;
  bool built = false;
  int cheb_degree = 2;
  long long version = 0;     // bumped by every numeric set-up (captured solver graphs key on it)
};

}  // namespace pfem
