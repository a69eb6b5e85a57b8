// mlp.cuh -- learned per-node Newton predictor: device state and launchers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pfem {

constexpr int MLP_NFEAT = 12;
constexpr int MLP_NPARAMS = 128 * 16 + 128 + 128 * 128 + 128 + 16 * 128 + 16;  // 20752

struct MlpState {
  bool alloc = false;
  bool ready = false;        // trained / loaded weights present
  int used_count = 0;        // load steps where the learned guess won
  long long adam_t = 0;
  float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;  // FP32 params, Adam moments, grads
  float* loss = nullptr;     // device scalar
  int* err = nullptr;        // device flag set by a timed-out wait
  // per-step prediction buffers (nn rows)
  void* feat = nullptr;      // BF16 nn x 16
  float* out = nullptr;      // nn x 3
  double* anode = nullptr;   // nodal equivalent plastic strain
  double* scale = nullptr;   // device scalar: max |dU_n|
  double* U3 = nullptr;      // U_{n-2}
  float* valence = nullptr;  // elements per node
  // recorded training set
  void* ds_x = nullptr;      // BF16 cap x 16
  float* ds_t = nullptr;     // cap x 3
  long long ds_n = 0, ds_cap = 0;
  bool recording = false;
  bool have_feat = false;    // features of the current step computed
  double r_ratio = 1.0;      // dlam_{n+1} / dlam_n of the current step
  double last_r_ex = -1.0;   // FP64 residuals of the last prediction (-1: not evaluated)
  double last_r_ml = -1.0;
  bool last_used = false;    // the last prediction kept the learned guess
  int* rows = nullptr;       // batch row indices
  int rows_cap = 0;
};

size_t mlp_smem_bytes();
int mlp_launch(bool train, const float* params, const void* X, const float* T, const int* rows, long long nrows,
               float* Y, float* grad, float* loss, int* err, int max_ctas, cudaStream_t st);
void mlp_adam(float* w, float* m, float* v, const float* g, float lr, long long t, cudaStream_t st);
void mlp_pack_features(const float* f, long long n, void* out, cudaStream_t st);

// solver-side helpers (mlp.cu)
void mlp_nodal_alpha(long long ne, long long nn, const int* elem, const double* alpha_gp, const float* valence,
                     double* anode, cudaStream_t st);
// scale[0] = max |dU_n|, scale[1] = max |dU_n - rho dU_{n-1}| (the second
// difference); part needs 2048 doubles.
void mlp_features(long long nn, const double* X, const double* lo, const double* ext, const double* U0,
                  const double* U1, const double* U2, const double* anode, double dlam, double lam, double rho,
                  double* scale, double* part, void* feat, cudaStream_t st);
void mlp_targets(long long nn, const double* Unew, const double* U0, const double* U1, double r,
                 const double* scale, float* out, cudaStream_t st);
void mlp_apply(long long nn, const double* U0, const double* U1, double r, const double* scale, const float* Y,
               double* U, cudaStream_t st);
void mlp_random_rows(int n, long long nrows, unsigned long long seed, int* rows, cudaStream_t st);

}  // namespace pfem
