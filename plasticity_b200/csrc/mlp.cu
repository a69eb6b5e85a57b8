// mlp.cu -- learned per-node Newton predictor: 12 -> 128 -> 128 -> 3 MLP (GELU)
// on BF16 tensor cores (tcgen05.mma kind::f16, FP32 accumulation in TMEM).
//
// One CTA (8 warps: two threads per tile row, each taking half of the row's
// columns in the epilogues) loops over tiles of 128 samples.  The forward-only
// kernel keeps H2 in H1's tile and allocates 256 TMEM columns, so two CTAs share
// an SM and one's epilogue overlaps the other's MMAs.
// Forward:  Z1 = X W1^T + b1, H1 = gelu(Z1); Z2 = H1 W2^T + b2, H2 = gelu(Z2);
//           Y = H2 W3^T + b3.
// Backward (mean squared error over the 3 outputs):
//           dY = 2 (Y - T) / (3B); dH2 = dY W3; dZ2 = dH2 * gelu'(Z2);
//           dH1 = dZ2 W2; dZ1 = dH1 * gelu'(Z1);
//           dW3^T += H2^T dY, dW2 += dZ2^T H1, dW1 += dZ1^T X (TMEM accumulators),
//           bias gradients are column sums of dY, dZ2, dZ1.
// Every GEMM is one tcgen05.mma chain issued by thread 0 with M = 128 (the
// tile rows, or the hidden width for the weight gradients); the transposed
// operands of the backward pass are the same shared-memory tiles read through
// MN-major descriptors.  Shared-memory tiles use the no-swizzle canonical
// layout: 8-row x 16-byte core matrices, core (row group g, column chunk c)
// at ((c * R/8) + g) * 128 bytes for an R-row tile.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "mlp.cuh"

namespace pfem {

namespace {

constexpr int TR = 128;  // tile rows
constexpr int HID = 128;
constexpr int INP = 16;  // 12 features padded to 16
constexpr int OUTP = 16; // 3 outputs padded to 16
constexpr long long WAIT_LIMIT = 1ll << 22;

// parameter offsets in the flat FP32 vector
constexpr int OFF_W1 = 0;                       // [HID][INP]
constexpr int OFF_B1 = OFF_W1 + HID * INP;      // [HID]
constexpr int OFF_W2 = OFF_B1 + HID;            // [HID][HID]
constexpr int OFF_B2 = OFF_W2 + HID * HID;      // [HID]
constexpr int OFF_W3 = OFF_B2 + HID;            // [OUTP][HID]
constexpr int OFF_B3 = OFF_W3 + OUTP * HID;     // [OUTP]
static_assert(OFF_B3 + OUTP == MLP_NPARAMS, "parameter layout");

constexpr int NT = 256;   // threads per CTA: row = tid % 128, column half = tid / 128

// shared-memory map (bytes); the forward-only kernel writes H2 over H1 (the
// MMA that reads H1 has completed by then) and has no backward tiles
template <bool TRAIN>
struct Lay {
  static constexpr int W1 = 0;                               // 128 x 16
  static constexpr int W2 = W1 + HID * INP * 2;              // 128 x 128
  static constexpr int W3 = W2 + HID * HID * 2;              // 16 x 128
  static constexpr int X = W3 + OUTP * HID * 2;              // 128 x 16
  static constexpr int H1 = X + TR * INP * 2;                // 128 x 128
  static constexpr int H2 = TRAIN ? H1 + TR * HID * 2 : H1;
  static constexpr int DY = H2 + TR * HID * 2;               // 128 x 16
  static constexpr int DZ2 = DY + (TRAIN ? TR * OUTP * 2 : 0);
  static constexpr int DZ1 = DZ2 + (TRAIN ? TR * HID * 2 : 0);
  static constexpr int BIAS = DZ1 + (TRAIN ? TR * HID * 2 : 0);  // b1, b2, b3 floats
  static constexpr int DB = BIAS + (HID + HID + OUTP) * 4;       // db1, db2, db3 partials
  static constexpr int MISC = DB + (HID + HID + OUTP) * 4;       // mbarrier, tmem base, abort, loss
  static constexpr int TOTAL = MISC + 64;
  static constexpr uint32_t COLS = TRAIN ? 512 : 256;            // TMEM columns allocated
};

// TMEM columns
constexpr uint32_t T_DA = 0, T_DB = 128, T_G2 = 256, T_G1 = 384, T_G3 = 400;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// byte offset of element (r, c) in an R-row no-swizzle tile
__device__ __forceinline__ uint32_t tile_off(int r, int c, int R) {
  return (uint32_t)(((c >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}
// UMMA shared-memory descriptor (no swizzle): start, leading / stride byte
// offsets, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// K-major operand: R rows (M or N), K step s of 16 columns.
__device__ __forceinline__ uint64_t desc_k(uint32_t base, int R, int s) {
  return smem_desc(base + (uint32_t)(2 * s * (R >> 3) * 128), (uint32_t)((R >> 3) * 128), 128);
}
// MN-major view of a tile stored with rows = K and columns = M or N: K step s
// covers tile rows 16s..16s+15.
__device__ __forceinline__ uint64_t desc_mn(uint32_t base, int R, int s) {
  return smem_desc(base + (uint32_t)(2 * s * 128), 128, (uint32_t)((R >> 3) * 128));
}
// instruction descriptor: BF16 x BF16 -> F32, M = 128, N, operand majors
__device__ __forceinline__ uint32_t idesc(int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TR >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem), "l"(a), "l"(b),
      "r"(id), "r"(acc));
}
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}
// Bounded wait on the mbarrier phase; returns false after WAIT_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// store 16 floats (columns c0..c0+15 of row r) as BF16 into an R-row tile
__device__ __forceinline__ void store16(unsigned char* tile, int r, int c0, int R, const float* v) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] = __floats2bfloat162_rn(v[h * 8 + 2 * i], v[h * 8 + 2 * i + 1]);
    *reinterpret_cast<uint4*>(tile + tile_off(r, c0 + 8 * h, R)) = *reinterpret_cast<uint4*>(p);
  }
}

// Column sums over the warp's 32 rows of 16 per-lane values, by halving
// exchanges (8 + 4 + 2 + 1 + 1 shuffles): afterwards the even lane 2m holds the
// sum of column colsum16_col(2m); returns it (odd lanes hold the same value).
__device__ __forceinline__ int colsum16_col(int lane) {
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}
__device__ __forceinline__ float colsum16(const float* v16, int lane) {
  float v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = v16[i];
#pragma unroll
  for (int o = 16, m = 16; o >= 2; o >>= 1, m >>= 1) {
    const bool lower = (lane & o) == 0;
    const int half = m >> 1;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (i < half) {
        const float send = lower ? v[i + half] : v[i];
        const float recv = __shfl_xor_sync(0xffffffffu, send, o);
        v[i] = (lower ? v[i] : v[i + half]) + recv;
      }
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

struct Ctl {
  uint32_t mbar;
  uint32_t phase;
  bool ok;
};
// thread 0 commits, every thread waits; a timeout sets the device error flag
__device__ __forceinline__ void sync_mma(Ctl& c, int* err, int* abort_flag) {
  if (threadIdx.x == 0) commit(c.mbar);
  if (!mbar_wait(c.mbar, c.phase)) {
    atomicExch(err, 1);
    *abort_flag = 1;
  }
  c.phase ^= 1u;
  fence_after();
}
__device__ __forceinline__ void sync_threads_tc() {
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
}

template <bool TRAIN>
__global__ void __launch_bounds__(NT, 1)
mlp_tile_kernel(const float* __restrict__ params, const __nv_bfloat16* __restrict__ X, const float* __restrict__ T,
                const int* __restrict__ rows, long long nrows, float* __restrict__ Y, float* __restrict__ grad,
                float* __restrict__ loss, float inv_scale, int* __restrict__ err) {
  using LY = Lay<TRAIN>;
  extern __shared__ __align__(1024) unsigned char sm[];
  const int tid = threadIdx.x;
  const int row = tid & (TR - 1);         // tile row = TMEM lane
  const int half = tid >> 7;              // which 64 of the 128 hidden columns this thread handles
  const int lane = tid & 31;
  float* bias = reinterpret_cast<float*>(sm + LY::BIAS);
  float* dbias = reinterpret_cast<float*>(sm + LY::DB);
  uint64_t* mbar_p = reinterpret_cast<uint64_t*>(sm + LY::MISC);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + LY::MISC + 8);
  int* abort_flag = reinterpret_cast<int*>(sm + LY::MISC + 12);
  float* loss_s = reinterpret_cast<float*>(sm + LY::MISC + 16);

  // ---- weights (BF16, K-major tiles) and biases into shared memory ----
  for (int i = tid; i < HID * INP; i += NT) {
    const int r = i / INP, c = i % INP;
    *reinterpret_cast<__nv_bfloat16*>(sm + LY::W1 + tile_off(r, c, HID)) = __float2bfloat16_rn(params[OFF_W1 + i]);
  }
  for (int i = tid; i < HID * HID; i += NT) {
    const int r = i / HID, c = i % HID;
    *reinterpret_cast<__nv_bfloat16*>(sm + LY::W2 + tile_off(r, c, HID)) = __float2bfloat16_rn(params[OFF_W2 + i]);
  }
  for (int i = tid; i < OUTP * HID; i += NT) {
    const int r = i / HID, c = i % HID;
    *reinterpret_cast<__nv_bfloat16*>(sm + LY::W3 + tile_off(r, c, OUTP)) = __float2bfloat16_rn(params[OFF_W3 + i]);
  }
  for (int i = tid; i < HID + HID + OUTP; i += NT) {
    bias[i] = i < HID ? params[OFF_B1 + i] : (i < 2 * HID ? params[OFF_B2 + i - HID] : params[OFF_B3 + i - 2 * HID]);
    dbias[i] = 0.0f;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar_p)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *abort_flag = 0;
    *loss_s = 0.0f;
  }
  if (tid < 32) {  // warp 0 allocates TMEM
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(LY::COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  sync_threads_tc();
  const uint32_t tbase = *tmem_slot;
  const uint32_t lane_off = (uint32_t)((row & ~31) << 16);  // this warp's TMEM lanes
  Ctl ctl{smem_addr(mbar_p), 0u, true};
  const uint32_t aW1 = smem_addr(sm + LY::W1), aW2 = smem_addr(sm + LY::W2), aW3 = smem_addr(sm + LY::W3);
  const uint32_t aX = smem_addr(sm + LY::X), aH1 = smem_addr(sm + LY::H1), aH2 = smem_addr(sm + LY::H2);
  const uint32_t aDY = smem_addr(sm + LY::DY), aDZ2 = smem_addr(sm + LY::DZ2), aDZ1 = smem_addr(sm + LY::DZ1);
  const int c_lo = half * (HID / 2), c_hi = c_lo + HID / 2;  // this thread's hidden columns
  bool first_tile = true;
  const long long ntiles = (nrows + TR - 1) / TR;
  float lsum = 0.0f;

  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // every thread reads the flag between the same two barriers
    __syncthreads();
    if (*abort_flag) break;
    const long long row0 = tile * TR;
    const long long gr = row0 + row;
    const bool valid = gr < nrows;
    const long long src = valid ? (rows ? (long long)rows[gr] : gr) : 0;
    // ---- X tile ----
    if (half == 0) {
      uint4 a = make_uint4(0, 0, 0, 0), b = make_uint4(0, 0, 0, 0);
      if (valid) {
        const uint4* p = reinterpret_cast<const uint4*>(X + src * INP);
        a = p[0];
        b = p[1];
      }
      *reinterpret_cast<uint4*>(sm + LY::X + tile_off(row, 0, TR)) = a;
      *reinterpret_cast<uint4*>(sm + LY::X + tile_off(row, 8, TR)) = b;
    }
    sync_threads_tc();
    // ---- Z1 = X W1^T ----
    if (tid == 0) mma(tbase + T_DA, desc_k(aX, TR, 0), desc_k(aW1, HID, 0), idesc(HID, 0, 0), 0);
    sync_mma(ctl, err, abort_flag);
    for (int c = c_lo; c < c_hi; c += 16) {
      float v[16];
      tmem_ld16(tbase + lane_off + T_DA + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + bias[c + i]);
      store16(sm + LY::H1, row, c, TR, v);
    }
    sync_threads_tc();
    // ---- Z2 = H1 W2^T ----
    if (tid == 0)
      for (int s = 0; s < HID / 16; ++s) mma(tbase + T_DB, desc_k(aH1, TR, s), desc_k(aW2, HID, s), idesc(HID, 0, 0), s > 0);
    sync_mma(ctl, err, abort_flag);
    for (int c = c_lo; c < c_hi; c += 16) {
      float v[16];
      tmem_ld16(tbase + lane_off + T_DB + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + bias[HID + c + i]);
      store16(sm + LY::H2, row, c, TR, v);
    }
    sync_threads_tc();
    // ---- Y = H2 W3^T ----
    if (tid == 0)
      for (int s = 0; s < HID / 16; ++s) mma(tbase + T_DA, desc_k(aH2, TR, s), desc_k(aW3, OUTP, s), idesc(OUTP, 0, 0), s > 0);
    sync_mma(ctl, err, abort_flag);
    float y[16];
    tmem_ld16(tbase + lane_off + T_DA, y);
#pragma unroll
    for (int i = 0; i < 16; ++i) y[i] += bias[2 * HID + i];
    if constexpr (!TRAIN) {
      if (valid && half == 0) {
        Y[gr * 3 + 0] = y[0];
        Y[gr * 3 + 1] = y[1];
        Y[gr * 3 + 2] = y[2];
      }
      sync_threads_tc();
    } else {
    // ---- backward ----
    float dy[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) dy[i] = 0.0f;
    if (valid && half == 0) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float e = y[j] - T[src * 3 + j];
        lsum += e * e;
        dy[j] = 2.0f * e * inv_scale;
      }
    }
    {
      const float cs = colsum16(dy, lane);  // warps of the upper half contribute zeros
      if (half == 0 && (lane & 1) == 0 && colsum16_col(lane) < 3) atomicAdd(&dbias[2 * HID + colsum16_col(lane)], cs);
    }
    if (half == 0) store16(sm + LY::DY, row, 0, TR, dy);
    sync_threads_tc();
    // dH2 = dY W3 (W3 as MN-major B), dW3^T += H2^T dY
    if (tid == 0) {
      mma(tbase + T_DA, desc_k(aDY, TR, 0), desc_mn(aW3, OUTP, 0), idesc(HID, 0, 1), 0);
      for (int s = 0; s < TR / 16; ++s)
        mma(tbase + T_G3, desc_mn(aH2, TR, s), desc_mn(aDY, TR, s), idesc(OUTP, 1, 1), (s > 0) || !first_tile);
    }
    sync_mma(ctl, err, abort_flag);
    for (int c = c_lo; c < c_hi; c += 16) {
      float g[16], z[16];
      tmem_ld16(tbase + lane_off + T_DA + c, g);
      tmem_ld16(tbase + lane_off + T_DB + c, z);
#pragma unroll
      for (int i = 0; i < 16; ++i) g[i] = valid ? g[i] * gelu_d(z[i] + bias[HID + c + i]) : 0.0f;
      const float cs = colsum16(g, lane);
      if ((lane & 1) == 0) atomicAdd(&dbias[HID + c + colsum16_col(lane)], cs);
      store16(sm + LY::DZ2, row, c, TR, g);
    }
    sync_threads_tc();
    // dH1 = dZ2 W2, dW2 += dZ2^T H1, Z1 again = X W1^T
    if (tid == 0) {
      for (int s = 0; s < HID / 16; ++s) mma(tbase + T_DB, desc_k(aDZ2, TR, s), desc_mn(aW2, HID, s), idesc(HID, 0, 1), s > 0);
      for (int s = 0; s < TR / 16; ++s)
        mma(tbase + T_G2, desc_mn(aDZ2, TR, s), desc_mn(aH1, TR, s), idesc(HID, 1, 1), (s > 0) || !first_tile);
      mma(tbase + T_DA, desc_k(aX, TR, 0), desc_k(aW1, HID, 0), idesc(HID, 0, 0), 0);
    }
    sync_mma(ctl, err, abort_flag);
    for (int c = c_lo; c < c_hi; c += 16) {
      float g[16], z[16];
      tmem_ld16(tbase + lane_off + T_DB + c, g);
      tmem_ld16(tbase + lane_off + T_DA + c, z);
#pragma unroll
      for (int i = 0; i < 16; ++i) g[i] = valid ? g[i] * gelu_d(z[i] + bias[c + i]) : 0.0f;
      const float cs = colsum16(g, lane);
      if ((lane & 1) == 0) atomicAdd(&dbias[c + colsum16_col(lane)], cs);
      store16(sm + LY::DZ1, row, c, TR, g);
    }
    sync_threads_tc();
    // dW1 += dZ1^T X
    if (tid == 0)
      for (int s = 0; s < TR / 16; ++s)
        mma(tbase + T_G1, desc_mn(aDZ1, TR, s), desc_mn(aX, TR, s), idesc(INP, 1, 1), (s > 0) || !first_tile);
    sync_mma(ctl, err, abort_flag);
    first_tile = false;
    }
  }

  if (TRAIN && !first_tile && !*abort_flag) {
    // weight gradients: TMEM lane = hidden unit (row of W1 / W2, column of W3)
    for (int c = c_lo; c < c_hi; c += 16) {
      float g[16];
      tmem_ld16(tbase + lane_off + T_G2 + c, g);
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(&grad[OFF_W2 + row * HID + c + i], g[i]);
    }
    {
      float g[16];
      tmem_ld16(tbase + lane_off + (half == 0 ? T_G1 : T_G3), g);
      if (half == 0) {
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(&grad[OFF_W1 + row * INP + i], g[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(&grad[OFF_W3 + i * HID + row], g[i]);
      }
    }
    __syncthreads();
    for (int i = tid; i < HID + HID + OUTP; i += NT) {
      const int off = i < HID ? OFF_B1 + i : (i < 2 * HID ? OFF_B2 + i - HID : OFF_B3 + i - 2 * HID);
      atomicAdd(&grad[off], dbias[i]);
    }
    atomicAdd(loss_s, lsum);
    __syncthreads();
    if (tid == 0) atomicAdd(loss, *loss_s);
  }
  fence_before();
  __syncthreads();
  if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(LY::COLS));
}

// Adam (FP32 master weights); bias-corrected step.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// FP32 host features (n x 12) -> BF16 rows of 16
__global__ void pack_features_kernel(const float* __restrict__ f, long long n, __nv_bfloat16* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n * INP) return;
  const long long r = i / INP;
  const int c = (int)(i % INP);
  out[i] = __float2bfloat16_rn(c < MLP_NFEAT ? f[r * MLP_NFEAT + c] : 0.0f);
}

// ---- solver-side kernels ----
__global__ void nodal_alpha_kernel(long long ne, const int* __restrict__ elem, const double* __restrict__ agp,
                                   const float* __restrict__ val, double* __restrict__ an) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double s = 0.0;
#pragma unroll
  for (int g = 0; g < 8; ++g) s += agp[e * 8 + g];
  s *= 0.125;
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int n = elem[e * 8 + a];
    atomicAdd(&an[n], s / (double)val[n]);
  }
}
constexpr int SCALE_BLOCKS = 1024;
// per-block maxima of |dU_n| and |dU_n - rho dU_{n-1}| (dU_n = U0 - U1, dU_{n-1} = U1 - U2)
__global__ void scales_kernel(long long n, const double* __restrict__ U0, const double* __restrict__ U1,
                              const double* __restrict__ U2, double rho, double* __restrict__ part) {
  __shared__ double sh[2][32];
  double m1 = 0.0, m2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d1 = U0[i] - U1[i];
    m1 = fmax(m1, fabs(d1));
    m2 = fmax(m2, fabs(d1 - rho * (U1[i] - U2[i])));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = m1;
    sh[1][threadIdx.x >> 5] = m2;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool in = threadIdx.x < (blockDim.x >> 5);
    m1 = in ? sh[0][threadIdx.x] : 0.0;
    m2 = in ? sh[1][threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
      m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    if (threadIdx.x == 0) {
      part[blockIdx.x] = m1;
      part[SCALE_BLOCKS + blockIdx.x] = m2;
    }
  }
}
// scale[1] is floored at 1e-6 scale[0] so a purely linear response (zero
// second difference) cannot blow the normalised features up.
__global__ void scales_final_kernel(int np, const double* __restrict__ part, double* __restrict__ scale) {
  double m1 = 0.0, m2 = 0.0;
  for (int i = 0; i < np; ++i) {
    m1 = fmax(m1, part[i]);
    m2 = fmax(m2, part[SCALE_BLOCKS + i]);
  }
  m1 = fmax(m1, 1e-300);
  scale[0] = m1;
  scale[1] = fmax(m2, 1e-6 * m1);
}
// features of node n for the step to lam: position in the bounding box,
// dU_n / scale[0], (dU_n - rho dU_{n-1}) / scale[1], nodal equivalent plastic
// strain, load-step size, load factor
__global__ void features_kernel(long long nn, const double* __restrict__ X, double lx, double ly, double lz,
                                double ex, double ey, double ez, const double* __restrict__ U0,
                                const double* __restrict__ U1, const double* __restrict__ U2,
                                const double* __restrict__ an, double dlam, double lam, double rho,
                                const double* __restrict__ scale, __nv_bfloat16* __restrict__ out) {
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const double is1 = 1.0 / scale[0], is2 = 1.0 / scale[1];
  float f[INP];
  f[0] = (float)((X[n * 3 + 0] - lx) / ex - 0.5);
  f[1] = (float)((X[n * 3 + 1] - ly) / ey - 0.5);
  f[2] = (float)((X[n * 3 + 2] - lz) / ez - 0.5);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double d1 = U0[n * 3 + d] - U1[n * 3 + d];
    f[3 + d] = (float)(d1 * is1);
    f[6 + d] = (float)((d1 - rho * (U1[n * 3 + d] - U2[n * 3 + d])) * is2);
  }
  f[9] = (float)(10.0 * an[n]);
  f[10] = (float)(10.0 * dlam);
  f[11] = (float)lam;
#pragma unroll
  for (int i = 12; i < INP; ++i) f[i] = 0.0f;
#pragma unroll
  for (int i = 0; i < INP; ++i) out[n * INP + i] = __float2bfloat16_rn(f[i]);
}
__global__ void targets_kernel(long long nn, const double* __restrict__ Un, const double* __restrict__ U0,
                               const double* __restrict__ U1, double r, const double* __restrict__ scale,
                               float* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nn * 3) return;
  out[i] = (float)((Un[i] - U0[i] - r * (U0[i] - U1[i])) / scale[1]);
}
__global__ void apply_kernel(long long nn, const double* __restrict__ U0, const double* __restrict__ U1, double r,
                             const double* __restrict__ scale, const float* __restrict__ Y, double* __restrict__ U) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nn * 3) return;
  U[i] = U0[i] + r * (U0[i] - U1[i]) + scale[1] * (double)Y[i];
}
__global__ void random_rows_kernel(int n, long long nrows, unsigned long long seed, int* __restrict__ rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long h = seed ^ ((unsigned long long)i * 0x9E3779B97F4A7C15ull);
  h ^= h >> 31; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 27; h *= 0x94D049BB133111EBull; h ^= h >> 31;
  rows[i] = (int)(h % (unsigned long long)nrows);
}

}  // namespace

void mlp_nodal_alpha(long long ne, long long nn, const int* elem, const double* alpha_gp, const float* valence,
                     double* anode, cudaStream_t st) {
  cudaMemsetAsync(anode, 0, nn * sizeof(double), st);
  count_launch();
  nodal_alpha_kernel<<<(int)((ne + 255) / 256), 256, 0, st>>>(ne, elem, alpha_gp, valence, anode);
}
void mlp_features(long long nn, const double* X, const double* lo, const double* ext, const double* U0,
                  const double* U1, const double* U2, const double* anode, double dlam, double lam, double rho,
                  double* scale, double* part, void* feat, cudaStream_t st) {
  const long long n3 = nn * 3;
  const int blocks = (int)std::min<long long>((n3 + 255) / 256, SCALE_BLOCKS);
  count_launch();
  scales_kernel<<<blocks, 256, 0, st>>>(n3, U0, U1, U2, rho, part);
  count_launch();
  scales_final_kernel<<<1, 1, 0, st>>>(blocks, part, scale);
  count_launch();
  features_kernel<<<(int)((nn + 255) / 256), 256, 0, st>>>(nn, X, lo[0], lo[1], lo[2], ext[0], ext[1], ext[2], U0,
                                                           U1, U2, anode, dlam, lam, rho, scale,
                                                           static_cast<__nv_bfloat16*>(feat));
}

void mlp_targets(long long nn, const double* Unew, const double* U0, const double* U1, double r,
                 const double* scale, float* out, cudaStream_t st) {
  count_launch();
  targets_kernel<<<(int)((nn * 3 + 255) / 256), 256, 0, st>>>(nn, Unew, U0, U1, r, scale, out);
}
void mlp_apply(long long nn, const double* U0, const double* U1, double r, const double* scale, const float* Y,
               double* U, cudaStream_t st) {
  count_launch();
  apply_kernel<<<(int)((nn * 3 + 255) / 256), 256, 0, st>>>(nn, U0, U1, r, scale, Y, U);
}
void mlp_random_rows(int n, long long nrows, unsigned long long seed, int* rows, cudaStream_t st) {
  count_launch();
  random_rows_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, nrows, seed, rows);
}

size_t mlp_smem_bytes() { return (size_t)Lay<true>::TOTAL; }

int mlp_launch(bool train, const float* params, const void* X, const float* T, const int* rows, long long nrows,
               float* Y, float* grad, float* loss, int* err, int max_ctas, cudaStream_t st) {
  if (nrows <= 0) return 0;
  const long long ntiles = (nrows + TR - 1) / TR;
  // max_ctas is a count of SMs: the training kernel (512 TMEM columns, ~178 KB of
  // shared memory) runs one CTA per SM, the forward kernel (256 columns, ~80 KB) two
  const int grid = (int)std::min<long long>(ntiles, (long long)max_ctas * (train ? 1 : 2));
  const float inv_scale = 1.0f / (3.0f * (float)nrows);
  const __nv_bfloat16* Xb = static_cast<const __nv_bfloat16*>(X);
  count_launch();
  if (train) {
    cudaFuncSetAttribute(mlp_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay<true>::TOTAL);
    mlp_tile_kernel<true><<<grid, NT, Lay<true>::TOTAL, st>>>(params, Xb, T, rows, nrows, Y, grad, loss, inv_scale,
                                                              err);
  } else {
    cudaFuncSetAttribute(mlp_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay<false>::TOTAL);
    mlp_tile_kernel<false><<<grid, NT, Lay<false>::TOTAL, st>>>(params, Xb, T, rows, nrows, Y, grad, loss, inv_scale,
                                                                err);
  }
  return (int)cudaGetLastError();
}

void mlp_adam(float* w, float* m, float* v, const float* g, float lr, long long t, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  count_launch();
  adam_kernel<<<(MLP_NPARAMS + 255) / 256, 256, 0, st>>>(w, m, v, g, MLP_NPARAMS, lr, b1, b2, eps, c1, c2);
}

void mlp_pack_features(const float* f, long long n, void* out, cudaStream_t st) {
  const long long tot = n * INP;
  count_launch();
  pack_features_kernel<<<(int)((tot + 255) / 256), 256, 0, st>>>(f, n, static_cast<__nv_bfloat16*>(out));
}

}  // namespace pfem
