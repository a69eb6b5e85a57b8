/*
 * pfem_b200.h -- C ABI of the B200 finite-strain F-bar J2 plasticity path.
 *
 * Drop-in for the per-Newton-iteration path of vinaysrao1/plasticity,
 * lagrangian/ (Julia).  A Julia shim binds these symbols with `ccall`, passing
 * its own arrays (GC.@preserve'd for the call); the Python package
 * `plasticity_b200` binds them with ctypes.
 *
 * Conventions (same as the reference):
 *   - node coordinates: 3 x nn, column-major (nodes[3*n + d]), Mesh.jl:17-22
 *   - element connectivity: 8 x ne, column-major, 1-based Int64, VTK Hex8 order
 *   - dof(n, c) = 3(n-1) + c (1-based), Mesh.jl:111; U is node-major
 *   - per-Gauss-point arrays: 6 x ngp column-major, gp = 8(e-1) + g, Mesh.jl:124-130
 *   - Voigt [xx,yy,zz,xy,yz,zx]; strain engineering shear, stress physical shear
 *   - sparsity exported as 1-based CSC (colptr/rowval), Assembly.jl:99-148
 *
 * Ownership: host buffers are read/written only during a call.  The library
 * owns one device context per pfem_ctx (device memory + one CUDA stream);
 * calls on one context are synchronous and must not run concurrently.
 * Errors: every call returns a pfem_status; no C++ exception crosses the ABI.
 * There is no CPU fallback: every call that computes runs on the GPU and
 * returns PFEM_ERR_CUDA when no usable device is present.
 */
#ifndef PFEM_B200_H
#define PFEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfem_ctx pfem_ctx;

enum pfem_status {
  PFEM_OK = 0,
  PFEM_ERR_BAD_ARG = -1,          /* ArgumentError guards, Materials.jl:90-103 */
  PFEM_ERR_CUDA = -2,             /* CUDA runtime failure (message in pfem_last_error) */
  PFEM_ERR_INVERTED_ELEMENT = -3, /* ElementInversionError, FiniteStrain.jl:42-52 */
  PFEM_ERR_LINSOLVE = -4,         /* Krylov solve missed its tolerance, Solver.jl:268-287 */
  PFEM_ERR_NOT_CONVERGED = -5,    /* Newton non-convergence, Solver.jl:463-467 */
  PFEM_ERR_STATE = -6             /* call made in the wrong state (e.g. no tangent yet) */
};

/* Element kinds, FiniteStrain.jl:62-65 (Hex8Finite / Hex8FiniteFbar). */
/* Element kinds (Model(...; element=:small / :finite / :finite_fbar), Model.jl:63-75).
 * PFEM_HEX8_SMALL: small strain (Elements.jl:323-360); the committed plastic strain lives in
 * the eps_p state array and the stress outputs are sigma. */
enum pfem_kind { PFEM_HEX8_SMALL = 0, PFEM_HEX8_FINITE = 1, PFEM_HEX8_FINITE_FBAR = 2 };
/* Tangent / inner-solve precision: FP64 throughout, or FP32 tangent + FP32
 * Krylov/AMG inside the FP64 Newton residual loop. */
enum pfem_precision { PFEM_FP64 = 0, PFEM_MIXED = 1 };
/* Newton predictor for each load step: previous converged U (the reference,
 * Solver.jl:321-323), linear extrapolation of the last two increments, or the
 * learned per-node MLP with extrapolation as fallback. */
enum pfem_predictor { PFEM_PRED_PREVIOUS = 0, PFEM_PRED_EXTRAPOLATE = 1, PFEM_PRED_LEARNED = 2 };
enum pfem_krylov { PFEM_KRYLOV_CG = 0, PFEM_KRYLOV_BICGSTAB = 1 };

/* J2Material(; E, nu, sigy0, Hiso, Hkin, sigsat, delta), Materials.jl:82-108.
 * Isotropic hardening sigma_y(a) = sigy0 + (sigsat - sigy0)(1 - exp(-delta a)) +
 * Hiso a (linear when delta = 0 or sigsat = sigy0), plus linear kinematic
 * hardening Hkin.  sigsat = 0 stands for the reference's default sigsat = sigy0.
 * Guards as the reference: E > 0, -1 < nu < 0.5, sigy0 > 0, Hiso >= 0,
 * Hkin >= 0, sigsat >= sigy0, delta >= 0, and saturation together with Hkin > 0
 * is rejected (PFEM_ERR_BAD_ARG).  With a per-element sigy0 the saturation
 * amplitude stays sigsat - sigy0 of this struct. */
typedef struct pfem_material {
  double E, nu, sigy0, Hiso, Hkin;
  double sigsat, delta;
} pfem_material;

/* Keyword arguments of solve!, Solver.jl:419-422, and LinearSolveState,
 * Solver.jl:103-108. */
typedef struct pfem_solve_opts {
  int32_t nsteps;        /* load steps, lambda = n/nsteps */
  int32_t maxiter;       /* Newton iterations per load step */
  double tol;            /* Newton relative residual tolerance */
  int32_t precision;     /* pfem_precision */
  int32_t krylov;        /* pfem_krylov */
  double lin_rtol;       /* > 0: fixed Krylov rtol; <= 0: Eisenstat-Walker forcing */
  double eta_min, eta_max, ew_gamma, ew_alpha;
  int32_t krylov_itmax;  /* cg_itmax */
  int32_t predictor;     /* pfem_predictor */
  int32_t amg_rebuild;   /* 0: once per load step (reference policy); 1: every Newton iteration;
                            2 (default): adaptive -- keep the numeric hierarchy across load
                            steps and rebuild when a Krylov solve needs more than
                            amg_stale_ratio times the iterations per decade of the first solve
                            after the last rebuild (or after reset / a new constrained set) */
  int32_t cheb_degree;   /* Chebyshev smoother degree */
  int32_t verbose;
  int32_t line_search;   /* 0: full Newton steps (the reference); 1: backtrack (halving, at
                            most 8 times) until the FP64 residual norm decreases -- the
                            accepted trial assembly is the next iterate, so a full step
                            costs nothing extra */
  int32_t predictor_smooth; /* learned predictor only: degree of the block-Jacobi Chebyshev
                            smoothing applied to the network's correction, on the tangent
                            at the extrapolated guess (0 = none) */
  int32_t max_cuts;      /* pfem_solve only: a load step that does not converge (or inverts an
                            element) is retried from the last converged state with half the
                            increment, at most max_cuts times per load step; 0 = the
                            reference (solve! stops, Solver.jl:455-466) */
  double eta_first;      /* Eisenstat-Walker forcing only: while no load step of the path has
                            converged yet (the first increment, from U = 0 and the full
                            boundary-value jump), the inner tolerance is capped at eta_first;
                            <= 0 = the reference's forcing term throughout */
  double amg_stale_ratio; /* amg_rebuild = 2 only (default 1.5) */
  int32_t ew_need;       /* Eisenstat-Walker forcing only: 1 (default) never asks an inner solve
                            for more than the Newton test needs, eta >= 0.5 tol
                            max(|R_1|, |F_ext|, 1) / |R_k| (no oversolving in the last
                            iteration); 0 = the reference's forcing term (Solver.jl:159-171) */
} pfem_solve_opts;

typedef struct pfem_solve_result {
  int32_t converged;
  int32_t steps_done;
  int32_t newton_iters_total;   /* sum of SolveResult.iters (each counts the final check) */
  int32_t krylov_iters_total;
  int32_t predictor_learned_used; /* load steps where the learned guess won */
  double time_total_ms;
  double time_assembly_ms;      /* element kernels incl. scatter, device time */
  double time_amg_setup_ms;
  double time_krylov_ms;
  double time_predictor_ms;
  int32_t load_step_cuts;       /* increments halved under pfem_solve_opts.max_cuts */
} pfem_solve_result;

void pfem_default_opts(pfem_solve_opts* o);

/* Model(mesh, material; element=:finite_fbar), Model.jl:63-75, plus
 * build_sparsity / element_colors (Assembly.jl:99-206) and
 * precompute_cache (Elements.jl:291-308).  sigy0_e: optional per-element
 * initial yield stress (ne values) replacing mat->sigy0.  device < 0 builds a
 * topology-only context (pattern and colors; compute calls return
 * PFEM_ERR_STATE) that needs no GPU. */
int pfem_create(pfem_ctx** out, const double* nodes, int64_t nn, const int64_t* elements,
                int64_t ne, int32_t kind, const pfem_material* mat, const double* sigy0_e,
                int32_t device);
void pfem_destroy(pfem_ctx* ctx);
const char* pfem_last_error(const pfem_ctx* ctx);
/* ElementInversionError fields (e, g 1-based; J = det Fbar), FiniteStrain.jl:42-46. */
int pfem_inversion_info(const pfem_ctx* ctx, int64_t* e, int32_t* g, double* J);

/* SparsityPattern.K structure (Assembly.jl:99-148): nnz, then 1-based
 * colptr (3nn+1) / rowval (nnz) when the pointers are non-null. */
int pfem_pattern(const pfem_ctx* ctx, int64_t* nnz, int64_t* colptr, int64_t* rowval);
/* element_colors (Assembly.jl:172-206): count and 0-based color per element. */
int pfem_colors(const pfem_ctx* ctx, int32_t* ncolors, int64_t* color_of_element);

/* fix!/prescribe!/load! accumulators frozen by _freeze_bcs (Solver.jl:192-218):
 * Dirichlet dofs (1-based, duplicates: last wins), values, ramp flags; Neumann
 * dofs and nodal forces (ramped by lambda). */
int pfem_set_bcs(pfem_ctx* ctx, const int64_t* dir_dofs, const double* dir_vals,
                 const uint8_t* dir_ramp, int64_t ndir, const int64_t* neu_dofs,
                 const double* neu_vals, int64_t nneu);

/* reset! (Model.jl:157-162): U = 0, Cp^-1 = I, alpha = 0, eps_p = 0. */
int pfem_reset(pfem_ctx* ctx);

/* assemble! (Assembly.jl:238-257) at displacement U (host, ndof) against the
 * committed state: writes F_int into R (ndof) and, if Kvals is non-null, the
 * tangent values in the order of the exported pattern read as CSR (row r,
 * columns rowval[colptr[r]..]); tau (6 x ngp) / flags (ngp) of the evaluation.
 * commit != 0 advances the committed state (Elements.jl:483-491).
 * precision selects the tangent storage (FP64 or FP32). */
int pfem_assemble(pfem_ctx* ctx, const double* U, int32_t commit, int32_t precision, double* R,
                  double* Kvals, double* tau, uint8_t* flags);

/* newton! (Solver.jl:317-389) for one load step at load factor lambda from
 * the context's current U and committed state, followed by the commit pass
 * (Solver.jl:470-471) when it converges.  res_hist / krylov_hist (capacity
 * maxiter) receive the residual norms and Krylov iteration counts. */
int pfem_newton(pfem_ctx* ctx, double lambda, const pfem_solve_opts* o, int32_t* iters,
                double* res_hist, int32_t* krylov_hist);

/* The Newton predictor alone for the load step to lambda (no counterpart in
 * the reference, whose predictor is the previous converged U, Solver.jl:321-323):
 * o->predictor selects extrapolation or the learned guess; the chosen guess is
 * left in the context's U (copied to U, ndof, when non-null), so a following
 * pfem_newton with predictor PFEM_PRED_PREVIOUS starts from it.  r_extrap /
 * r_learned receive the imposed FP64 residual norms of the two guesses
 * (r_learned = -1 when the learned guess was not evaluated: no trained
 * weights, or fewer than two converged steps); learned_used = 1 when the
 * learned guess was kept. */
int pfem_predict(pfem_ctx* ctx, double lambda, const pfem_solve_opts* o, double* U, double* r_extrap,
                 double* r_learned, int32_t* learned_used);

/* solve! (Solver.jl:419-475): reset, load loop, Newton, commit.
 * iters_per_step (nsteps), residuals (nsteps x maxiter, row per step) and
 * krylov_per_iter (nsteps x maxiter) may be null. */
int pfem_solve(pfem_ctx* ctx, const pfem_solve_opts* o, pfem_solve_result* res,
               int32_t* iters_per_step, double* residuals, int32_t* krylov_per_iter);

/* One Newton iteration's assembly at the context's current U against the
 * committed state: K and R (Assembly.jl:238-257), R -= lambda Fext, Dirichlet
 * imposition of both BC sets (Solver.jl:349-355), ||R|| (Solver.jl:358).  The
 * imposed tangent stays resident for pfem_linear_solve; R (ndof) is copied
 * out when non-null. */
int pfem_residual(pfem_ctx* ctx, double lambda, int32_t precision, double* rnorm, double* R);

/* _linear_solve! (Solver.jl:235-290) on the tangent left by the last Newton
 * iteration (Dirichlet rows imposed): x = K^-1 b to relative tolerance rtol. */
int pfem_linear_solve(pfem_ctx* ctx, const double* b, double* x, double rtol, int32_t rebuild_pc,
                      const pfem_solve_opts* o, int32_t* niter);

/* One cycle of the AMG hierarchy last built by pfem_linear_solve / Newton
 * (precision of the resident tangent; a V on the finest level, a W on the
 * levels between it and the dense coarsest level): z = M^-1 r, host vectors
 * of ndof. */
int pfem_amg_apply(pfem_ctx* ctx, const double* r, double* z);

/* Inspection of the resident AMG hierarchy (small problems): the dense
 * operator of `level` (what = 0, n_l x n_l, row-major), its smoothed
 * prolongator (what = 1, n_l x n_{l+1}), or, for the coarsest level L, the
 * dense inverse the cycle applies (what = 2, n_L x n_L); dims receives
 * (rows, cols). */
int pfem_amg_dense(pfem_ctx* ctx, int32_t level, int32_t what, double* out, int64_t* dims);

/* Read-out: nodal_displacements / gauss_kirchhoff / equivalent_plastic_strain /
 * Cp^-1 / eps_p / last elastic-plastic flags (Model.jl:169-232).  Null pointers
 * are skipped.  Per-GP arrays are 6 x ngp column-major. */
int pfem_get_state(const pfem_ctx* ctx, double* U, double* tau, double* alpha, double* cpi,
                   double* epsp, uint8_t* flags);
/* Overwrite the committed per-GP state (6 x ngp Cp^-1, ngp alpha, optional
 * 6 x ngp eps_p; null pointers keep the current values). */
int pfem_set_state(pfem_ctx* ctx, const double* cpi, const double* alpha, const double* epsp);
/* Overwrite U (host ndof) -- e.g. to evaluate a predictor guess. */
int pfem_set_displacement(pfem_ctx* ctx, const double* U);
/* Committed back stress beta (state_committed.beta: Model.jl:38, GaussState Mesh.jl:124-130), 6 x ngp
 * column-major (physical-shear Voigt).  For the finite kinds it is the
 * rotation-neutralised back stress of the reference configuration
 * (FiniteStrain.jl:292-346).  get writes zeros when Hkin = 0; set needs
 * Hkin > 0. */
int pfem_get_back_stress(const pfem_ctx* ctx, double* beta);
int pfem_set_back_stress(pfem_ctx* ctx, const double* beta);
/* gauss_stress (Model.jl:188-208): Cauchy = tau / det F_gp (standard F). */
int pfem_gauss_stress(const pfem_ctx* ctx, double* sigma);

/* Device timing of one hot-path kernel family on the resident data, CUDA
 * events on the context's stream, averaged over reps launches.
 * what: 0 = element kernels of one full assembly (all colors, FP64 tangent),
 *       1 = same with the FP32 tangent, 2 = level-0 SpMV FP32, 3 = SpMV FP64,
 *       4 = one cycle of the resident FP32 AMG hierarchy, captured once in a CUDA
 *           graph and replayed (as inside the CG loop). */
int pfem_profile(pfem_ctx* ctx, int32_t what, int32_t reps, double* ms_per_launch);

/* CUDA-event timer on the context's stream (the stream every kernel of this
 * context is launched on): op 0 records the start event; op 1 records the
 * stop event, synchronizes and returns the elapsed milliseconds in *ms. */
int pfem_timer(pfem_ctx* ctx, int32_t op, double* ms);
/* Euclidean norm sqrt(sum x_i^2) of a device vector, allocating nothing.  It
 * has no counterpart in the reference.  It serves callers that cannot call
 * cudaMalloc -- code running inside a framework that owns every device
 * allocation through its own pool, or a caller that must keep cudaMalloc and
 * cudaFree out of its steady state.  x (n doubles) and result (one double) are
 * device pointers the caller owns.  The per-block partial sums live in a
 * file-scope device array of 65,536 doubles (512 KiB on every device that
 * loads the library, held until the process exits), so n is limited to
 * 134,217,728 elements; a larger n returns PFEM_ERR_BAD_ARG and
 * pfem_last_error(NULL) says why.  The call is asynchronous on `stream` (a
 * cudaStream_t; NULL means the legacy default stream).  The first call on a
 * device, made with that device current, looks up the scratch address; make
 * it before any stream capture.  All calls share the scratch array, so calls
 * that overlap on the GPU race. */
int pfem_norm2_noalloc(const double* x, int64_t n, double* result, void* stream);

/* ---- Learned Newton predictor (no counterpart in the reference) ----
 * Per-node MLP 12 -> 128 -> 128 -> 3 (GELU) on BF16 tensor cores with FP32
 * accumulation.  Features of node n for the step to lambda_{k+1}, from the two
 * previous converged increments dU_k and dU_{k-1}: coordinates scaled to the
 * bounding box minus 1/2 (3), dU_k / s1 (3) with s1 = max |dU_k|, the second
 * difference d2 = dU_k - rho dU_{k-1} over s2 = max |d2| (3; rho the ratio of
 * the two previous load-step sizes), 10 x nodal-mean alpha (1), 10 x
 * load-step size (1), lambda_{k+1} (1).  Output y: U_{k+1} = U_k + r dU_k +
 * s2 y, r the step ratio -- the extrapolation predictor plus a learned
 * correction measured in units of the second difference, so BF16 resolution
 * applies to the correction itself.  With predictor = PFEM_PRED_LEARNED the
 * network's correction is smoothed (pfem_solve_opts.predictor_smooth) and the
 * guess with the smaller FP64 residual (learned or extrapolated) starts
 * Newton.  Parameters are MLP_NPARAMS = 20752 FP32 values:
 * W1 [128][16], b1 [128], W2 [128][128], b2 [128], W3 [16][128], b3 [16]
 * (columns 12..15 of W1 and rows 3..15 of W3 are padding, kept zero). */
int pfem_mlp_init(pfem_ctx* ctx, uint64_t seed);
/* op 0: copy the parameters out; op 1: load them (the predictor becomes usable). */
int pfem_mlp_params(pfem_ctx* ctx, int32_t op, float* params, int64_t n);
/* Forward pass on host features (n x 12) -> outputs (n x 3). */
int pfem_mlp_forward(pfem_ctx* ctx, const float* feats, int64_t n, float* out);
/* Mean-squared-error loss and its gradient (MLP_NPARAMS) on host data. */
int pfem_mlp_loss_grad(pfem_ctx* ctx, const float* feats, const float* targets, int64_t n, float* grad,
                       float* loss);
/* Training-set recording from converged load steps: op 0 start (capacity
 * samples), 1 stop, 2 clear; *size receives the number of recorded samples. */
int pfem_mlp_record(pfem_ctx* ctx, int32_t op, int64_t capacity, int64_t* size);
/* Adam (beta 0.9/0.999) on random batches of the recorded samples. */
int pfem_mlp_train(pfem_ctx* ctx, int32_t steps, int32_t batch, float lr, uint64_t seed, float* losses);

/* Number of CUDA kernels this library has launched in this process. */
int64_t pfem_kernel_launches(void);

/* Bytes per block column index that the level-0 SpMV reads (inspection; no
 * counterpart in the reference): 2 when every column id of the tangent lies
 * within +-32767 of its row (offsets stored in 16 bits; node-ordered meshes up to
 * about 180^3), else 4. */
int pfem_tangent_index_bytes(pfem_ctx* ctx, int32_t* bytes);

#ifdef __cplusplus
}
#endif
#endif /* PFEM_B200_H */
