// Internal interfaces shared by the FBME .cu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../../include/fbme_b200.h"

namespace fbme {

#define FBME_TIMED(prof, g, launch) \
  do {                              \
    if (prof) (prof)->begin(g);     \
    launch;                         \
    if (prof) (prof)->end();        \
  } while (0)

constexpr int kMaxTilesPerScene = 64;  // partial-sum slots per scene and stage
constexpr int kPartWarps = 8;          // per-warp partial sums kept per tile and reduction
constexpr int kPartSlots = 4 * kPartWarps;  // 4 reductions x 8 warps per tile
constexpr int kMaxPolish = 32;         // active-set capacity of the warp polish

// Per-scene scalar state, structure of arrays of length B (device).
struct Scalars {
  float* data_power;  // max(mean |y|^2, eps)
  float* floor_;      // variance floor = prior floor
  float* noise;       // noise variance sigma^2
  float* dvar;        // UAMP data variance (sum of coefficient variances)
  float* pv;          // pseudo variance of the current sweep
  float* prec;        // 1 / (dvar + noise)
  float* ebp;         // sum |A^H y|^2
  float* dof;         // UAMP effective DOF of the last sweep
  float* energy;      // last residual energy
  float* data_energy; // sum |y|^2
};

// Geometry of one equal-shape batch.
struct BatchShape {
  int B, n1, n2, m1, m2;
  __host__ __device__ long long n() const { return static_cast<long long>(n1) * n2; }
  __host__ __device__ long long m() const { return static_cast<long long>(m1) * m2; }
};

// Resolved numeric configuration used by device code.
struct DevConfig {
  float uamp_damping, damping, blend, init_noise, fixed_noise, min_var, max_prec;
  float hyper_shape, hyper_rate, noise_shape, noise_rate;
  int noise_evidence;
  int polish_size, polish_iters, prune_tail, reinit, gate;
  float polish_damping, margin_factor;
  int exchange;
  int fixed_budget;
  float jitter;
  float false_alarm;
  int terms;
  int uamp_iters;
  // observed samples per scene under an observation mask (0: the whole
  // M1 x M2 block is observed)
  float m_obs;
  // support repairs after the polish (global certificate on), whose
  // evidence extends the trace
  int repairs;
};

// Samples a scene's data terms count: the observed ones under a mask.
__host__ __device__ inline double observed_samples(const BatchShape& s, const DevConfig& c) {
  return c.m_obs > 0.f ? static_cast<double>(c.m_obs) : static_cast<double>(s.m());
}

// Optional per-launch event timing (fbme_plan_profile); nullptr otherwise.
struct Profiler {
  static constexpr int kMax = 512;
  cudaEvent_t ev[2 * kMax];
  int group[kMax];
  int n = 0;
  cudaStream_t st = nullptr;
  void begin(int g) {
    if (n < kMax) {
      group[n] = g;
      cudaEventRecord(ev[2 * n], st);
    }
  }
  void end() {
    if (n < kMax) {
      cudaEventRecord(ev[2 * n + 1], st);
      ++n;
    }
  }
};

// ---------------------------------------------------------------------------
// launchers (all asynchronous on `st`)
// ---------------------------------------------------------------------------
void launch_twiddle_table(uint8_t* dst, int L, int sign, int n_tile, int col_tiles, int kchunks,
                          int parts, cudaStream_t st);
void launch_dirichlet(float2* dst, int M, int L, cudaStream_t st);

struct DftTables {
  const uint8_t* fwd_n2;  // L = N2, sign -1
  const uint8_t* fwd_n1;  // L = N1, sign -1
  const uint8_t* adj_n2;  // L = N2, sign +1
  const uint8_t* adj_n1;  // L = N1, sign +1
  int kchunks_n1, kchunks_n2;
  int n_tile;  // real output columns per stage tile the tables are laid out for
  // FP32 FFT mode (dft_terms = 0): the FP64-evaluated twiddles of lengths
  // N1 and N2, in the layout of fft.cu (fft_twiddle_kernel)
  const float2* fft_n1;
  const float2* fft_n2;
};

// FP32 FFT stages (fft.cu).  mode 0 store, 1 store + sum |out|^2 (slot 1),
// 2 store + masked sum |y - out|^2 (slot 2); ysum: sum |in|^2 (slot 3).
int fft_length_ok(int L);
int fft_stage_tiles(int rows, int L);
cudaError_t set_fft_attributes();
void launch_fft_twiddles(float2* dst, int L, cudaStream_t st);

// Buffers of the UAMP stage.
struct UampBuffers {
  const float2* y;
  float2 *mu, *bp, *msg, *pred, *tmp;
  float2* lift;  // [B][N] adjoint output A^H m (the denoiser's input)
  float *var, *gamma;
  double* part;  // [B][kMaxTilesPerScene][kPartSlots]
  uint32_t* keys;  // [B][N] order-preserving score keys (final E-step)
  Scalars sc;
  int* status;   // launch status word
  // observation mask [M1*M2] (nullptr: all observed); y is then the masked
  // copy of the caller's data
  const uint8_t* mask;
  // nonzero: tmp holds the two-stage intermediates as the second stage's
  // pre-split operand (split_unit_bytes per scene; 3-term products only)
  int split;
  // learned warm start (optional): FP32 network parameters and its workspace
  const float* warm_params;
  void* warm_ws;
  // caller-supplied warm start (optional): [B][N] log(prior / (P/N)) map
  const float* warm_map;
};

cudaError_t set_dft_attributes();
cudaError_t set_polish_attributes();
void dft_forward(const BatchShape& s, const DftTables& t, int terms, const float2* coeff,
                 float2* data, float2* tmp, int* status, cudaStream_t st);
void dft_adjoint(const BatchShape& s, const DftTables& t, int terms, const float2* data,
                 float2* coeff, float2* tmp, int* status, cudaStream_t st);
// plain_prior = false stops after the data power, floors and initial noise
// (a warm start supplies the prior).
void sbl_init(const BatchShape& s, const DftTables& t, const DevConfig& c, const UampBuffers& u,
              cudaStream_t st, Profiler* prof = nullptr, bool plain_prior = true);
void uamp_run(const BatchShape& s, const DftTables& t, const DevConfig& c, const UampBuffers& u,
              cudaStream_t st, Profiler* prof = nullptr);
// One shape bucket of uamp_run_multi.
struct UampJob {
  BatchShape s;
  DftTables t;
  DevConfig c;
  UampBuffers u;
};
// uamp_run over several shape buckets with merged launches (no warm start).
// FP32 FFT buckets of different transform lengths run their per-length
// launches of a step on `st` and the `naux` side streams, forked and joined
// through `ev` (naux + 1 events), when no profiler is given.
void uamp_run_multi(const UampJob* jobs, int n, cudaStream_t st, Profiler* prof = nullptr,
                    const cudaStream_t* aux = nullptr, const cudaEvent_t* ev = nullptr, int naux = 0);

// Active-set stage.
struct PolishBuffers {
  const float2* y;
  const float2* bp;
  const float2 *mu, *dir1, *dir2;
  // under an observation mask: the Gram table G(d) = sum over observed
  // samples m of exp(2 pi i m.d / N), [N1][N2] (replaces dir1 x dir2)
  const float2* gram2d;
  const float *var, *gamma;
  Scalars sc;
  // per-scene state
  int* active;        // [B][K] current active set
  float* score;       // [B][K] UAMP second moments of the active set
  float* gamma_init;  // [B][K] prior variances of the active set before reinit
  unsigned char* pstate;  // opaque per-scene polish state
  float* xcand_val;   // exchange candidates [B][E]
  int* xcand_idx;
  uint32_t* keys;     // [B][N] score keys scratch
  uint32_t* cand_key; // [B][max candidates] top-k candidate keys
  int* cand_idx;      // [B][max candidates] their grid indices
  int* status;        // [B] per-scene status
};
// `cert` (host copy; null: off) adds the global certificate and support
// repairs between the polish and its outputs.
void polish_run(const BatchShape& s, const DevConfig& c, const PolishBuffers& p,
                const FbmeOutputs& out, cudaStream_t st, Profiler* prof = nullptr,
                const FbmeCertificate* cert = nullptr);
size_t polish_state_bytes();
size_t cert_scratch_bytes(const BatchShape& s);
int topk_slices(long long n);

// Several shape buckets' top-k in one launch each (uneven plans): bucket i
// is blockIdx.z = i, its scenes and slices in blockIdx.y / x.
constexpr int kBucketSetMax = 64;
struct TopkJob {
  const uint32_t* keys;  // [B][n]
  long long n;
  int k, B;
  uint32_t* cand_key;
  int* cand_idx;
};
struct TopkJobs {
  int n;
  TopkJob j[kBucketSetMax];
};
struct TopkMergeJob {
  const uint32_t* cand_key;
  const int* cand_idx;
  int ncand, k, B;
  int* out_idx;
  float* out_val;
};
struct TopkMergeJobs {
  int n;
  TopkMergeJob j[kBucketSetMax];
};
void launch_topk_blocks_multi(const TopkJobs& J, int max_slices, int max_b, cudaStream_t st);
void launch_topk_merge_multi(const TopkMergeJobs& J, int max_b, cudaStream_t st);
// The polish of several equal-config shape buckets (an uneven plan's) as
// one launch per step: results equal polish_run per bucket.
struct PolishBucket {
  BatchShape s;
  DevConfig c;
  PolishBuffers p;
  FbmeOutputs out;
};
void polish_run_multi(const PolishBucket* b, int n, cudaStream_t st);
// Observation masks (mask.cu): set-up (normalised mask, observed count,
// 2-D Gram table; synchronises `st`) and the masked copy of the data.
size_t mask_gram_scratch_bytes(const BatchShape& s);
cudaError_t mask_setup(const BatchShape& s, const uint8_t* mask_in, uint8_t* mask, float2* gram, void* scratch,
                       long long* observed, cudaStream_t st);
void mask_data(const BatchShape& s, const float2* y, const uint8_t* mask, float2* out, cudaStream_t st);
// Stage-kernel wait-timeout self-test (uamp.cu).
size_t stage_selftest_bytes();
cudaError_t stage_selftest(void* ws, int* status, long long wait_cycles, cudaStream_t st);
// Unfused variational ARD prior update (prior.cu).
void uamp_prior_update(const float2* mean, const float* var, const float* old_prior, const float* floor_,
                       int batch, long long n, float hyper_shape, float hyper_rate, float damping,
                       float maximum, float* out, cudaStream_t st);
size_t topk_scratch_bytes(long long n, int k, int batch);
const char* topk_check(long long n, int k, int batch);
void topk_scores(const float* scores, long long n, int k, int batch, void* scratch,
                 int64_t* indices, float* values, cudaStream_t st);
int exchange_blocks(const BatchShape& s);

// Learned warm start (csrc/cnn.cu).
int cnn_param_count();
size_t cnn_workspace_bytes(long long B, long long H, long long W);
const char* cnn_check(long long B, long long H, long long W);
void cnn_features(const float2* bp, int B, int H, int W, void* ws, cudaStream_t st);
void cnn_forward(const float* params, int B, int H, int W, void* ws, float* out, cudaStream_t st);
void cnn_backward(const float* target, int B, int H, int W, void* ws, float* grad, double* loss_out,
                  cudaStream_t st);
void cnn_adam(float* params, const float* grad, float* m, float* v, int step, float lr, cudaStream_t st);
// ebp (optional): sum |bp|^2 per scene, from the initialisation
void cnn_warm_prior(const float* params, const float2* bp, int B, int H, int W, void* ws,
                    const float* data_power, const float* floor_, float* gamma, double* upart,
                    int nblocks, cudaStream_t st, const float* ebp = nullptr);
// The same initial prior from a caller-supplied [B][N] log(prior / (P/N)) map.
void warm_prior_from_map(const float* map, int B, int H, int W, const float* data_power, const float* floor_,
                         float* gamma, double* upart, int nblocks, cudaStream_t st);
cudaError_t set_cnn_attributes();

// Active-set switch of single-scene cg runs (cg_active.cu).
struct ActiveBufs {
  int* sel;        // [0] selected size (0: no switch), [1] non-finite flag
  int* idx;        // [kmax] selected grid indices, largest prior first
  uint8_t* mask;   // [N] 1 on the active set
  float2* E;       // [kmax * kmax] equilibrated system / Cholesky factor (column-major)
  float2* X;       // [kmax * kmax] L^-1 (column-major, lower)
};
struct ActiveArgs {
  long long N;
  int n1, n2;      // grid
  int K;           // active-set size
  int nb;          // tiles of the EM kernels' relevance partials
  const int* idx;
  const float* gamma;
  const float2* bp;    // A^H y
  const float* noise;  // [1]
  const float2 *d1, *d2;  // Dirichlet tables of the prefix
  float jitter;        // Cholesky loading multiplier
  float2 *E, *X;
  float2* mean;        // [N] out
  float* relc;         // [N] out: clipped relevance
  float* pv_out;       // [N] out (optional): posterior variance
  double* part;        // partial slots of scene 0
  int* status;
};
constexpr int kActiveMax = 1024;  // largest active_set_max_size built
size_t cg_active_bytes(long long N, int kmax);
ActiveBufs cg_active_bind(uint8_t* w, long long N, int kmax);
void cg_active_select(const float* gamma, long long N, int kmax, int min_size, float tail, const ActiveBufs& ab,
                      cudaStream_t st);
void cg_active_mask(const ActiveBufs& ab, long long N, int kmax, cudaStream_t st);
void cg_active_posterior(const ActiveArgs& a, cudaStream_t st);

// mode="dense": the exact posterior through the M x M data covariance in
// FP64 (dense.cu).
struct DenseBufs {
  double2 *Q, *X;      // [B][M][M] Cholesky factor, then Q^-1 / L^-1 (column-major)
  double2 *lag, *lsum; // [B][2M1-1][2M2-1] lags of the prior, lag sums of Q^-1
  double2* pass;       // separable-transform pass buffer
  double2* z;          // [B][M] Q^-1 y
  double2* lift;       // [B][N] A^H Q^-1 y
  double* dd;          // [B][N] diag(A^H Q^-1 A)
  double2 *tw1, *tw2;  // FP64 twiddles of N1, N2
};
size_t dense_bytes(const BatchShape& s);
DenseBufs dense_bind(uint8_t* w, const BatchShape& s, cudaStream_t st);
void dense_posterior(const BatchShape& s, const DenseBufs& d, const float* gamma, const float* noise,
                     const float2* y, float jitter, float2* mean, float* relc, float* pv_out, double* part, int nb,
                     int* status, cudaStream_t st);

// Shared by the C ABI translation units.
int api_fail(int code, const std::string& msg);
size_t dft_table_bytes(int L, int terms);
cudaError_t set_cg_attributes();

}  // namespace fbme
