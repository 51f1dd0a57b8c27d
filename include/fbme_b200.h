/*
 * fbme_b200.h -- C ABI of the B200 (sm_100a) FBME plan-replay hot path.
 *
 * Plain C types only: device pointers, sizes, a CUDA stream handle.  The
 * caller (the Python host layer, or any C/C++/FFI host) owns every device
 * buffer, including the plan workspace whose size fbme_plan_workspace_bytes
 * reports; the library allocates no device memory.  No exception crosses
 * this boundary: every entry point returns an FBME_* error code and
 * fbme_last_error() describes the last failure of the calling thread.
 *
 * Thread-safety: one plan per stream; a plan must not be replayed
 * concurrently with itself.  Plans share no mutable global state.
 *
 * Reference interfaces replaced (FBME-SBL v1.1, paths inside that project):
 *   fbme_plan_create / replay  <-> torch_sbl/cuda_graph.py:22-107
 *                                  (CUDAGraphSBLPlan.__init__ / .replay) and
 *                                  torch_sbl_fastest_stable/profiles.py:35-148
 *   fbme_dft_forward           <-> torch_sbl/operators.py:237-253 (forward_flat)
 *   fbme_dft_adjoint           <-> torch_sbl/operators.py:255-280 (adjoint_flat)
 *   fbme_uamp_run              <-> torch_sbl/solver.py:1063-1189, 1295-1798,
 *                                  1907-1925 (fast_sbl uamp init/loop/E-step),
 *                                  solver.py:2726-2870 (_uamp_posterior) and the
 *                                  Triton kernels torch_sbl/triton_kernels.py:
 *                                  476-547, 550-667, 806-904
 *   fbme_polish_run            <-> torch_sbl/solver.py:1926-2021, 3961-4510
 *                                  (top-K + _uamp_active_em_polish + fixed-
 *                                  budget diagnostics), 2081-2126
 */
#ifndef FBME_B200_H
#define FBME_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same handle as cudaStream_t. */
typedef struct CUstream_st* fbme_stream_t;

/* Return codes. */
enum {
  FBME_OK = 0,
  FBME_ERR_INVALID = 1,     /* bad argument, shape or config (-> ValueError) */
  FBME_ERR_UNSUPPORTED = 2, /* valid request outside what is built */
  FBME_ERR_CUDA = 3,        /* a CUDA runtime call failed (-> RuntimeError) */
  FBME_ERR_WORKSPACE = 4    /* workspace too small or misaligned */
};

/* Per-scene status bits written to FbmeOutputs.status. */
enum {
  FBME_STATUS_NONFINITE = 1,   /* NaN/Inf reached the reduced posterior */
  FBME_STATUS_CHOLESKY = 2,    /* reduced Cholesky pivot <= 0 after loading */
  FBME_STATUS_TIMEOUT = 4,     /* a bounded device wait ran out */
  FBME_STATUS_PCG_BREAKDOWN = 8,
  FBME_STATUS_ITER_CAP = 16
};

/* One scene: reconstruction grid N1 x N2, observed prefix M1 x M2. */
typedef struct {
  int32_t n1, n2, m1, m2;
} FbmeShape;

/* Hot-path fields of SBLConfig (torch_sbl/solver.py:34-176), resolved by
 * the host layer (e.g. the UAMP iteration budget of solver.py:1295-1309). */
typedef struct {
  int32_t uamp_iterations;           /* T_u */
  float uamp_damping;                /* message/denoiser damping */
  float damping;                     /* prior and noise damping ("keep") */
  float initialization_blend;        /* backprojection blend; < 0 => uniform */
  float initial_noise_fraction;
  float fixed_noise_variance;        /* <= 0 => estimated */
  float min_variance;
  float max_precision;
  float hyper_shape, hyper_rate, noise_shape, noise_rate;
  int32_t noise_update;              /* 0 = "em", 1 = "evidence" */
  int32_t polish_size;               /* K, 0 disables the active-set polish */
  int32_t polish_iterations;         /* P */
  int32_t polish_prune_tail;
  int32_t polish_reinitialize;
  int32_t polish_evidence_gate;
  float polish_damping;
  float evidence_margin_factor;
  int32_t exchange_size;             /* residual support exchange size */
  int32_t fixed_budget_diagnostics;
  float cholesky_jitter_multiplier;  /* reduced Cholesky loading, x eps */
  float support_false_alarm_budget;  /* <= 0 => no support mask */
  int32_t dft_terms;                 /* split-BF16 products: 3 or 6 */
} FbmeConfig;

/* Caller-owned device output buffers for B scenes (N = n1*n2 per scene).
 * Pointers marked optional may be NULL. */
typedef struct {
  void* x;                                 /* [B,N] complex64 */
  float* posterior_variance;               /* [B,N] */
  float* precision;                        /* [B,N] */
  uint8_t* support_mask;                   /* [B,N] bool, optional */
  float* noise_variance;                   /* [B] */
  float* effective_dof;                    /* [B] */
  float* negative_log_evidence;            /* [B] */
  float* evidence_trace;                   /* [B,P] */
  int64_t* support_exchanges_accepted;     /* [B], optional */
  float* fixed_budget_gamma_residual;      /* [B], optional */
  float* fixed_budget_noise_residual;      /* [B], optional */
  float* fixed_budget_objective_decrease;  /* [B], optional */
  uint8_t* fixed_budget_monotone;          /* [B], optional */
  float* support_score_threshold;          /* [B], optional */
  int64_t* active_indices;                 /* [B,K], optional */
  void* active_values;                     /* [B,K] complex64, optional: x at
                                              active_indices (x is zero
                                              elsewhere, so the pair is the
                                              whole reconstruction) */
  int32_t* status;                         /* [B] */
} FbmeOutputs;

/* Device pointers into a plan's resident UAMP state (for tests/tools). */
typedef struct {
  void* mean;              /* [B,N] complex64 */
  float* variance;         /* [B,N] */
  float* prior_variance;   /* [B,N] */
  void* message;           /* [B,M] complex64 */
  void* prediction;        /* [B,M] complex64 */
  void* backprojection;    /* [B,N] complex64 (A^H y) */
  float* noise_variance;   /* [B] */
  float* data_variance;    /* [B] */
} FbmeState;

typedef struct FbmePlan FbmePlan;

/* Bytes of device workspace a plan for these scenes needs (0 on error). */
size_t fbme_plan_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes,
                                 const FbmeConfig* cfg);

/* Build a plan: validate, bind the caller's workspace (256-byte aligned)
 * and fill its constant tables on `stream`.  Launches kernels and waits
 * for them; call it outside stream capture. */
int fbme_plan_create(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                     void* workspace, size_t workspace_bytes, fbme_stream_t stream,
                     FbmePlan** plan);

/* Solve every scene.  Equal shapes: y is [B, M1*M2] complex64 (row-major
 * prefix blocks, scenes back to back) and the outputs are as FbmeOutputs
 * lists them.  Scenes of different shapes (an uneven plan): y holds each
 * scene's M1*M2 samples back to back in scene order, and the per-pixel
 * outputs (x, posterior_variance, precision, support_mask) each scene's
 * N1*N2 values back to back; per-scene outputs stay [B], [B,P], [B,K].
 * Asynchronous on `stream`; capturable (an uneven plan forks its shape
 * buckets onto plan-owned streams and joins them back on `stream`). */
int fbme_plan_replay(FbmePlan* plan, const void* y, const FbmeOutputs* out,
                     fbme_stream_t stream);

int fbme_plan_destroy(FbmePlan* plan);

/* ------------------------------------------------------------------------
 * Uneven batches (no counterpart in the reference, which batches only
 * equal shapes through leading dimensions, torch_sbl/solver.py:966-1001).
 * A plan may hold scenes of different shapes: it groups them into one
 * bucket per shape, in order of first appearance; each bucket is solved
 * as an equal-shape batch with its own tables and state, the buckets run
 * concurrently, and a gather / scatter kernel pair maps the scene-order
 * buffers to bucket order and back.  Values that depend on the shape are
 * set per bucket by FbmeShapeParams (the host resolves them from N and M
 * as torch_sbl/solver.py:1183-1189 and 1295-1309 do); the solve of a
 * scene stops after its own bucket's T_u sweeps.
 * ---------------------------------------------------------------------- */
typedef struct {
  FbmeShape shape;            /* scenes of this shape use the values below */
  int32_t uamp_iterations;    /* T_u; <= 0 keeps FbmeConfig.uamp_iterations */
  float uamp_damping;         /* < 0 keeps FbmeConfig.uamp_damping */
  int32_t exchange_size;      /* < 0 keeps FbmeConfig.exchange_size */
  int32_t dft_n_tile;         /* DFT stage tile width in real columns: 64,
                                 128 or 256 with 3 terms (128 with 6); 0 =
                                 default (256, or 128 with 6 terms) */
} FbmeShapeParams;

size_t fbme_plan_workspace_bytes_ex(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                                    const FbmeShapeParams* params, int32_t n_params);
int fbme_plan_create_ex(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                        const FbmeShapeParams* params, int32_t n_params, void* workspace,
                        size_t workspace_bytes, fbme_stream_t stream, FbmePlan** plan);
/* Buckets of a plan (1 for equal shapes) and the resolved values of one. */
int32_t fbme_plan_bucket_count(const FbmePlan* plan);
int fbme_plan_bucket(const FbmePlan* plan, int32_t bucket, FbmeShapeParams* resolved, int32_t* n_scenes);

/* Stage entry points (same plan, same stream rules; equal-shape plans
 * only: an uneven plan returns FBME_ERR_UNSUPPORTED). */
int fbme_dft_forward(FbmePlan* plan, const void* coefficients, void* data, fbme_stream_t stream);
int fbme_dft_adjoint(FbmePlan* plan, const void* data, void* coefficients, fbme_stream_t stream);
/* UAMP initialisation, T_u sweeps and the final E-step; the state is left
 * in the plan (read it with fbme_plan_state). */
int fbme_uamp_run(FbmePlan* plan, const void* y, fbme_stream_t stream);
/* Top-K, reduced evidence-gated polish and outputs, from the plan's state
 * after fbme_uamp_run. */
int fbme_polish_run(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream);
int fbme_plan_state(FbmePlan* plan, FbmeState* state);

/* Observation mask (non-rectangular sampling), replacing the
 * observation_mask of PrefixFourierOperator (torch_sbl/operators.py:57-75,
 * 473-496) and of sbl_2d (torch_sbl/solver.py:986-1021) on the plan path.
 * `mask` is a device array of M1*M2 bytes (nonzero = observed), shared by
 * every scene of an equal-shape plan; NULL restores the full block.  The
 * observations keep the M1 x M2 layout; unobserved samples are ignored.
 * Builds the masked Gram table and reads the observed count back, so it
 * synchronises `stream`: call it after fbme_plan_create and before replays
 * are captured.  The caller resolves the config's sweep budget from the
 * observed count (as solver.py does from operator.n_samples).  An uneven
 * plan returns FBME_ERR_UNSUPPORTED; an all-zero mask FBME_ERR_INVALID. */
int fbme_plan_set_observation_mask(FbmePlan* plan, const uint8_t* mask, fbme_stream_t stream);

/* Global certificate and support repairs of the active-set polish
 * (uamp_polish_global_certificate / uamp_polish_support_repairs, the
 * certified_hybrid_uamp configuration), replacing _inactive_evidence_certificate
 * (torch_sbl/solver.py:3522-3588), _active_evidence_certificate (3219-3317),
 * the repair loop (4511-4628) and the final coordinate diagnostics
 * (4851-4870, 5388-5460) of _uamp_active_em_polish.  After the polish the
 * plan scores every grid atom j by its one-coordinate Type-II ratio
 * |a_j^H C^-1 y|^2 / a_j^H C^-1 a_j, lets the best inactive atom replace the
 * active atom of largest deletion gain up to `support_repairs` times (kept
 * when the exact evidence does not rise), and writes the certificate of the
 * final model.  Every output is a device array of B entries; the evidence
 * trace of FbmeOutputs then holds P + support_repairs entries per scene.
 * The tolerance-to-ratio threshold is computed by the caller.  Call before
 * replays are captured; NULL switches the certificate off.  An uneven plan
 * returns FBME_ERR_UNSUPPORTED. */
typedef struct {
  int32_t support_repairs;                  /* R in [0, 4], P + R <= 8 */
  float coordinate_tolerance;               /* gains <= tolerance are stationary */
  float familywise_ratio_threshold;         /* > 0: familywise_no_discovery is written */
  float* inactive_max_evidence_ratio;
  int64_t* inactive_best_index;
  float* inactive_evidence_gain;
  float* inactive_optimal_variance;
  int64_t* support_repairs_accepted;        /* residual exchanges + repairs kept */
  float* active_max_evidence_gain;
  int64_t* active_best_index;
  float* active_optimal_variance;
  float* active_max_deletion_gain;
  float* active_penalized_evidence_gain;
  uint8_t* coordinate_stationary;
  uint8_t* type2_map_coordinate_stationary;
  uint8_t* familywise_no_discovery;         /* required when the threshold > 0 */
  void* workspace;                          /* device scratch, 256-byte aligned */
  size_t workspace_bytes;                   /* >= fbme_plan_certificate_workspace_bytes() */
} FbmeCertificate;
size_t fbme_plan_certificate_workspace_bytes(const FbmePlan* plan);
int fbme_plan_set_certificate(FbmePlan* plan, const FbmeCertificate* cert);

/* Unfused variational ARD prior update, replacing uamp_prior_update /
 * _uamp_prior_kernel (torch_sbl/triton_kernels.py:670-735, 196-235; taken
 * at torch_sbl/solver.py:1605-1625 when the UAMP posterior has not already
 * damped the prior).  For `batch` scenes of `n` coefficients:
 *   cand  = clamp((|mean|^2 + posterior_variance + hyper_rate)
 *                 / (1 + hyper_shape), prior_floor[b], maximum)
 *   out   = max(damping * old_prior + (1 - damping) * cand, prior_floor[b])
 * with |mean|^2 = re^2 + im^2 and every float32 operation rounded on its
 * own.  mean is complex64 [batch, n]; posterior_variance, old_prior, out
 * float32 [batch, n]; prior_floor float32 [batch].  batch <= 65535. */
int fbme_uamp_prior_update(const void* mean, const float* posterior_variance, const float* old_prior,
                           const float* prior_floor, int32_t batch, int64_t n, float hyper_shape,
                           float hyper_rate, float damping, float maximum, float* out,
                           fbme_stream_t stream);

/* Top-k (k <= 32) of each of `batch` rows of `n` float scores: values
 * largest first, ties by lower index, as torch.topk(scores, k) at
 * torch_sbl/solver.py:1931 and 4410.  `indices` / `values` are [batch, k].
 * batch <= 65535 (rows run on a grid dimension of that limit), k <= n and
 * ceil(n/8192) * k <= 2048; other sizes return FBME_ERR_INVALID.
 * The caller provides fbme_topk_workspace_bytes(n, k, batch) bytes of
 * 16-byte aligned device workspace for the per-slice candidates. */
size_t fbme_topk_workspace_bytes(int64_t n, int32_t k, int32_t batch);
int fbme_topk(const float* scores, int64_t n, int32_t k, int32_t batch, void* workspace,
              size_t workspace_bytes, int64_t* indices, float* values, fbme_stream_t stream);

/* Allocation-free top-k; no counterpart in the reference.  Same result as
 * fbme_topk, for callers that cannot allocate device memory when they need
 * it: code running while another component captures a CUDA graph (no
 * allocation during global-mode capture), real-time hosts that freeze their
 * memory budget after start-up, FFI hosts that only receive device pointers.
 * The candidate scratch is a library-owned static device array of
 * FBME_TOPK_STATIC_SCRATCH_BYTES (1 MiB), held by every GPU that loads the
 * library until the process exits.  Requests needing more than that
 * (batch * ceil(n/8192) * k * 8 bytes) return FBME_ERR_INVALID, as do the
 * sizes fbme_topk rejects.  The first call on a device (and the first after
 * cudaDeviceReset, which gives the device a new context) looks up the
 * array's device address with that device current: make it before any
 * stream capture.  All calls share the array (nothing in it needs to start
 * at zero); calls that overlap on the GPU race on it, so the caller must
 * order them.  An error left pending by an earlier launch is returned as
 * FBME_ERR_CUDA before anything is launched.  Allocates nothing.  Error
 * text: fbme_topk_static_error(). */
#define FBME_TOPK_STATIC_SCRATCH_BYTES (1u << 20)
int fbme_topk_static(const float* scores, int64_t n, int32_t k, int32_t batch, int64_t* indices,
                     float* values, fbme_stream_t stream);
const char* fbme_topk_static_error(void);

/* ------------------------------------------------------------------------
 * mode="cg": PCG + Hutchinson SBL for a batch of equally shaped scenes
 * (and mode="dense" with `dense` set: the same EM loop, exact posterior).
 *
 * Replaces (FBME-SBL v1.1):
 *   fbme_cg_solve     <-> torch_sbl/solver.py:925-2393 (fast_sbl) with
 *                         mode="cg": initialisation 1063-1159, probe setup
 *                         1191-1221, EM loop 1315-1904 (_posterior cg
 *                         branch 2991-3036, relevance 3156-3181, MacKay
 *                         update 1669-1677, noise update 1737-1791,
 *                         convergence 1800-1904), final posterior 2023-2080
 *   fbme_pcg_solve    <-> torch_sbl/solver.py:5582-5723 (_pcg) with the
 *                         low-rank preconditioner 5786-5848
 *   fbme_cg_matvec    <-> torch_sbl/operators.py:299-371 (Q = noise I +
 *                         A diag(prior) A^H; toeplitz_matvec / matvec)
 * A single-scene plan with active_set_start > 0 also runs the active-set
 * switch (solver.py:1316-1341): from that EM iteration, every
 * active_set_check_interval iterations until it switches, the ARD set is
 * selected (_select_active_indices, 3184-3216) and, once selected, the
 * remaining iterations and the final posterior use the exact reduced
 * posterior on it (_active_posterior, 3897-3920) with the omitted prior
 * variances fixed (1684-1693).
 * ---------------------------------------------------------------------- */
typedef struct {
  int32_t max_iter, min_iter;           /* outer EM iterations */
  int32_t cg_min_iter;
  float tol;                            /* relative change tolerance (0: off) */
  int32_t convergence_patience, convergence_check_interval;
  float hyper_shape, hyper_rate, noise_shape, noise_rate;
  float initial_noise_fraction;
  float initialization_blend;           /* < 0: uniform initialisation */
  float fixed_noise_variance;           /* > 0: fixed noise variance */
  int32_t noise_update;                 /* 0 = EM, 1 = evidence */
  float damping, cg_damping;            /* keep = max(damping, cg_damping) */
  float min_variance, max_precision;
  float cg_tolerance, cg_initial_tolerance;
  int32_t cg_max_iter, cg_check_interval, cg_fixed_iterations;
  int32_t preconditioner_rank;          /* low-rank preconditioner atoms (<= 32) */
  int32_t probes;                       /* maximum Hutchinson probes P */
  int32_t initial_probes;               /* adaptive schedule: probes of iterations 1-5 */
  int32_t adaptive_cg, adaptive_probes, warm_start;
  float jitter_multiplier;              /* Cholesky loading: max(10, m) * eps * mean|diag| */
  int32_t dft_terms;                    /* 3 or 6 split-BF16 products */
  /* active-set switch (one scene only; 0 = off) */
  int32_t active_set_start;             /* first EM iteration that may switch */
  int32_t active_set_check_interval;
  int32_t active_set_min_size, active_set_max_size;  /* max <= 1024 */
  float active_set_tail_fraction;       /* in (0, 1) */
  /* 1: mode="dense" (solver.py:2962-2990): the exact posterior through the
   * M x M data covariance, in FP64, instead of PCG + Hutchinson (probes,
   * cg_* and the active set unused); M <= 4096 */
  int32_t dense;
} FbmeCgConfig;

/* Device outputs of fbme_cg_solve (shapes [B][N1][N2] / [B]). */
typedef struct {
  void* x;                       /* complex64 posterior mean */
  float* posterior_variance;
  float* precision;              /* 1 / prior variance */
  float* noise_variance;
  float* effective_dof;
  uint8_t* support_mask;         /* optional: |x|^2 / max(v, tiny) > support_threshold */
  float support_threshold;       /* used when support_mask is set (solver.py:2108-2126) */
  int32_t* status;               /* FBME_STATUS_* bits per scene */
} FbmeCgOutputs;

/* Host-side run summary.  `history`, if not NULL, receives max_iter rows of
 * {relative change (max over scenes), mean noise variance, mean effective
 * DOF, PCG iterations, probes, PCG tolerance} for the iterations run. */
typedef struct {
  int32_t iterations;
  int32_t converged;
  float relative_change;
  int32_t last_cg_iterations;
  float* history;
  int32_t active_set_size;       /* size of the switched-to active set (0: none) */
  int32_t active_set_iteration;  /* EM iteration of the switch (0: none) */
} FbmeCgInfo;

typedef struct FbmeCgPlan FbmeCgPlan;

size_t fbme_cg_workspace_bytes(const FbmeShape* shape, int32_t n_scenes, const FbmeCgConfig* cfg);
int fbme_cg_create(const FbmeShape* shape, int32_t n_scenes, const FbmeCgConfig* cfg,
                   void* workspace, size_t workspace_bytes, fbme_stream_t stream,
                   FbmeCgPlan** plan);
/* y: complex64 [B][M1][M2]; probes: float32 +-1 [B][P][M1][M2] (probe p of
 * scene b over the observed samples, the reference's probes[b, :, p]).
 * The PCG restart test runs on the device (a CUDA graph WHILE node repeats
 * chunks of cg_check_interval iterations while a right-hand side is active;
 * with cg_fixed_iterations or an odd check interval the host reads it).
 * Synchronises `stream` at the EM convergence checks and active-set checks,
 * as the reference reads those on the host. */
int fbme_cg_solve(FbmeCgPlan* plan, const void* y, const float* probes, const FbmeCgOutputs* out,
                  FbmeCgInfo* info, fbme_stream_t stream);
int fbme_cg_destroy(FbmeCgPlan* plan);
/* out = Q v for `rhs` vectors per scene: v, out complex64 [B][rhs][M1][M2];
 * prior float [B][N1][N2]; noise float [B]; rhs <= 1 + P. */
int fbme_cg_matvec(FbmeCgPlan* plan, const float* prior, const float* noise, const void* v,
                   int32_t rhs, void* out, fbme_stream_t stream);
/* One preconditioned solve Q X = RHS (rhs columns per scene, layout as
 * fbme_cg_matvec), initial guess `initial` (NULL: zero), with the plan's
 * cg_max_iter / cg_check_interval / cg_fixed_iterations / rank.  Writes the
 * solution and the iteration count of the last loop. */
int fbme_pcg_solve(FbmeCgPlan* plan, const float* prior, const float* noise, const void* rhs,
                   int32_t rhs_count, const void* initial, float tolerance, void* solution,
                   int32_t* iterations, fbme_stream_t stream);

/* ------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference: it is the learned
 * part of this implementation).  A 3-layer 3x3 convolutional network
 * (8 hidden channels, BF16 operands, FP32 accumulation) maps the features
 * of A^H y to the initial log prior variance that replaces the
 * backprojection initialisation of torch_sbl/solver.py:1072-1099.
 * Parameters are an FP32 vector of fbme_cnn_param_count() values; the
 * layout is W1[3][3][2][8], b1[8], W2[3][3][8][8], b2[8], W3[3][3][8][1],
 * b3[1] (809 values).  Grids need N1 % 8 == 0 and N2 % 16 == 0.
 * ---------------------------------------------------------------------- */
int32_t fbme_cnn_param_count(void);
size_t fbme_cnn_workspace_bytes(int32_t batch, int32_t n1, int32_t n2);
/* Features of the backprojection (complex64 [batch][n1][n2]) into the
 * workspace; forward / backward then read them from there. */
int fbme_cnn_features(const void* backprojection, int32_t batch, int32_t n1, int32_t n2, void* workspace,
                      fbme_stream_t stream);
/* out [batch][n1][n2] FP32 = network output (predicted log(prior / (P/N)),
 * P the data power).  Keeps the activations for fbme_cnn_backward. */
int fbme_cnn_forward(const float* params, int32_t batch, int32_t n1, int32_t n2, void* workspace, float* out,
                     fbme_stream_t stream);
/* Gradient of mean((out - target)^2) after fbme_cnn_forward on the same
 * workspace; writes grad[param_count] and the loss to *loss (device FP64,
 * may be NULL). */
int fbme_cnn_backward(const float* target, int32_t batch, int32_t n1, int32_t n2, void* workspace, float* grad,
                      double* loss, fbme_stream_t stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the FP32 parameters. */
int fbme_cnn_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                  fbme_stream_t stream);
/* Warm-started replays: from the next replay on, the plan's initial prior
 * is max(P/N * exp(network output), floor) instead of the backprojection
 * blend.  `params` (device, FP32) and `workspace` stay caller-owned and
 * must outlive the replays; params == NULL turns the warm start off. */
size_t fbme_plan_warm_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes);
int fbme_plan_set_warm_start(FbmePlan* plan, const float* params, void* workspace, size_t workspace_bytes);
/* Warm start from the caller's own predictor: from the next replay on, the
 * initial prior is max(P/N * exp(map), floor), map a device float array
 * [B, N1*N2] of log(prior / (P/N)) that the caller fills before each replay
 * (for example from A^H y, fbme_dft_adjoint).  Caller-owned, read at every
 * replay; NULL turns it off.  Replaces a network set by
 * fbme_plan_set_warm_start (and is replaced by it).  Any grid. */
int fbme_plan_set_warm_prior_map(FbmePlan* plan, const float* map);

/* Kernel groups timed by fbme_plan_profile. */
enum {
  FBME_GROUP_INIT = 0,        /* A^H y, data power, prior/noise initialisation */
  FBME_GROUP_ADJ_MESSAGE = 1, /* adjoint stage 1 (reads the updated message) */
  FBME_GROUP_ADJ_DENOISE = 2, /* denoiser / ARD update (elementwise, after adjoint stage 2) */
  FBME_GROUP_FWD_1 = 3,       /* forward stage 1 */
  FBME_GROUP_FWD_RESIDUAL = 4,/* forward stage 2 with the fused residual energy */
  FBME_GROUP_SCALARS = 5,     /* per-scene noise / variance updates */
  FBME_GROUP_SWEEP1 = 6,      /* first-sweep denoiser (reuses A^H y) */
  FBME_GROUP_TOPK = 7,        /* top-K selections */
  FBME_GROUP_POLISH = 8,      /* reduced posterior, gate, EM, diagnostics */
  FBME_GROUP_EXCHANGE = 9,    /* residual exchange scoring over the grid */
  FBME_GROUP_OUTPUT = 10,     /* dense outputs */
  FBME_GROUP_ADJ_2 = 11,      /* adjoint stage 2 of sweeps 2.. and the final E-step */
  FBME_GROUP_MESSAGE = 12,    /* UAMP message update (elementwise, before adjoint stage 1) */
  FBME_GROUP_CERTIFICATE = 13,/* global certificate and support repairs (fbme_plan_set_certificate) */
  FBME_NUM_GROUPS = 14
};

/* One replay with CUDA events around every kernel launch (not capturable;
 * synchronises `stream`).  group_ms[g] receives the summed device time of
 * group g and group_launches[g] its launch count, for g < n_groups. */
int fbme_plan_profile(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream,
                      float* group_ms, int32_t* group_launches, int32_t n_groups);
const char* fbme_profile_group_name(int32_t group);

/* Failure-detection self-test of the bounded device waits (no counterpart
 * in the reference, which has no device-side waits).  Launches one DFT
 * stage tile with its operand producer held back, so the tensor-core
 * issuer's wait for a full operand stage and the epilogue's wait for the
 * accumulator both run out after `wait_cycles` SM cycles (in [1e3, 2e9];
 * plans use 1e9).  The kernel then ORs FBME_STATUS_TIMEOUT into *status,
 * releases its tensor memory and returns, leaving the context usable.
 * `workspace` (fbme_selftest_workspace_bytes(), 256-byte aligned) holds
 * the tile's operands and output; nothing in it is read or written. */
size_t fbme_selftest_workspace_bytes(void);
int fbme_selftest_stage_timeout(void* workspace, size_t workspace_bytes, int32_t* status, int64_t wait_cycles,
                                fbme_stream_t stream);

/* Thread-local description of the last failure ("" if none). */
const char* fbme_last_error(void);
/* Library version string. */
const char* fbme_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FBME_B200_H */
