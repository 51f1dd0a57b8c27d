// C ABI of the FBME B200 library: plan creation over a caller-owned
// workspace, replay, and stage entry points.  See include/fbme_b200.h.
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <vector>

#include "kernels.cuh"
#include "stage.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Bytes of one split-BF16 twiddle table for axis length L laid out for
// stage tiles of nt real columns.
size_t table_bytes(int L, int terms, int nt) {
  if (terms == 0) return 0;  // the FP32 FFT mode has no tensor-core tables
  const int parts = terms == 6 ? 3 : 2;
  return static_cast<size_t>(ceil_div(2LL * L, nt)) * ceil_div(2LL * L, 64) * parts * nt * 128;
}
int default_n_tile(int terms) { return terms == 6 ? 128 : 256; }

struct Layout {
  size_t tab_f2, tab_f1, tab_a2, tab_a1, dir1, dir2;
  size_t mu, bp, var, gamma, msg, pred, tmp, lift, keys, part, scal;
  size_t active, score, pstate, xval, xidx, status, ckey, cidx;
  size_t mask, ymask, gram, gscr;  // observation mask (fbme_plan_set_observation_mask)
  size_t fft1, fft2;               // FP32 FFT twiddles (dft_terms 0)
  size_t total;
};

Layout make_layout(const fbme::BatchShape& s, const FbmeConfig& c, int nt) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align256(off + bytes);
    return o;
  };
  const size_t B = s.B, N = s.n(), M = s.m();
  const size_t K = c.polish_size > 0 ? c.polish_size : 1;
  const size_t E = c.exchange_size > 0 ? c.exchange_size : 1;
  L.tab_f2 = take(table_bytes(s.n2, c.dft_terms, nt));
  L.tab_a2 = take(table_bytes(s.n2, c.dft_terms, nt));
  if (s.n1 != s.n2) {
    L.tab_f1 = take(table_bytes(s.n1, c.dft_terms, nt));
    L.tab_a1 = take(table_bytes(s.n1, c.dft_terms, nt));
  } else {
    L.tab_f1 = L.tab_f2;
    L.tab_a1 = L.tab_a2;
  }
  L.dir1 = take(s.n1 * sizeof(float2));
  L.dir2 = take(s.n2 * sizeof(float2));
  L.mu = take(B * N * sizeof(float2));
  L.bp = take(B * N * sizeof(float2));
  L.var = take(B * N * sizeof(float));
  L.gamma = take(B * N * sizeof(float));
  L.msg = take(2 * B * M * sizeof(float2));
  L.pred = take(B * M * sizeof(float2));
  // the two-stage intermediates: FP32 complex, or (3-term products) the
  // second stage's pre-split operand, whose rows and K are tile-padded
  size_t tmp1 = static_cast<size_t>(s.m2) * s.n1 * sizeof(float2);
  size_t tmp2 = static_cast<size_t>(s.n2) * s.m1 * sizeof(float2);
  if (c.dft_terms == 3) {
    tmp1 = static_cast<size_t>(fbme::split_unit_bytes(s.m2, s.n1));
    tmp2 = static_cast<size_t>(fbme::split_unit_bytes(s.n2, s.m1));
  }
  L.tmp = take(B * (tmp1 > tmp2 ? tmp1 : tmp2));
  L.lift = take(B * N * sizeof(float2));
  L.keys = take(B * N * sizeof(uint32_t));
  L.part = take(B * fbme::kMaxTilesPerScene * fbme::kPartSlots * sizeof(double));
  L.scal = take(10 * B * sizeof(float));
  L.active = take(B * K * sizeof(int));
  L.score = take(B * K * sizeof(float));
  L.pstate = take(B * fbme::polish_state_bytes());
  L.xval = take(B * E * sizeof(float));
  L.xidx = take(B * E * sizeof(int));
  L.status = take(B * sizeof(int));
  const size_t c1 = static_cast<size_t>(fbme::topk_slices(s.n())) * K;
  const size_t c2 = static_cast<size_t>(fbme::exchange_blocks(s)) * E;
  const size_t nc = c1 > c2 ? c1 : c2;
  L.ckey = take(B * nc * sizeof(uint32_t));
  L.cidx = take(B * nc * sizeof(int));
  L.mask = take(M);
  L.ymask = take(B * M * sizeof(float2));
  L.gram = take(N * sizeof(float2));
  L.gscr = take(fbme::mask_gram_scratch_bytes(s));
  L.fft1 = take(c.dft_terms == 0 ? s.n1 * sizeof(float2) : 0);
  L.fft2 = take(c.dft_terms == 0 ? s.n2 * sizeof(float2) : 0);
  L.total = off;
  return L;
}

int check_shape(const FbmeShape& s) {
  if (s.n1 < 1 || s.n2 < 1 || s.m1 < 1 || s.m2 < 1 || s.m1 > s.n1 || s.m2 > s.n2)
    return fail(FBME_ERR_INVALID, "Each sample dimension must satisfy 0 < M <= N.");
  return FBME_OK;
}

// Checks of one bucket: its shape s (s.B scenes) under its resolved config.
int check_bucket(const fbme::BatchShape& s, const FbmeConfig* c, int nt) {
  const long long N = s.n();
  if (c->dft_terms != 0 && c->dft_terms != 3 && c->dft_terms != 6)
    return fail(FBME_ERR_INVALID, "dft_terms must be 0 (FP32 FFT), 3 or 6");
  if (c->dft_terms == 0 && (!fbme::fft_length_ok(s.n1) || !fbme::fft_length_ok(s.n2)))
    return fail(FBME_ERR_UNSUPPORTED, "the FP32 FFT mode needs N1 and N2 of the form 2^a or 3 * 2^a, at most 512");
  if (c->uamp_iterations < 1) return fail(FBME_ERR_INVALID, "uamp_iterations must be positive");
  if (c->polish_size < 1 || !c->polish_prune_tail)
    return fail(FBME_ERR_UNSUPPORTED,
                "the device path implements the zero-tail active-set polish (polish_size >= 1, "
                "prune_tail)");
  if (c->polish_size > fbme::kMaxPolish)
    return fail(FBME_ERR_UNSUPPORTED, "polish_size above 32 is not built");
  if (c->polish_size > N) return fail(FBME_ERR_INVALID, "polish_size exceeds the grid size");
  if (c->polish_iterations < 1 || c->polish_iterations > 8)
    return fail(FBME_ERR_INVALID, "polish_iterations must be in [1, 8]");
  if (c->exchange_size < 0 || c->exchange_size > 32)
    return fail(FBME_ERR_INVALID, "exchange size must be in [0, 32]");
  if (c->exchange_size > 0) {
    const long long lim1 = c->polish_size - 1, lim2 = N - c->polish_size;
    if (c->exchange_size > lim1 || c->exchange_size > lim2)
      return fail(FBME_ERR_INVALID, "exchange size must be resolved to min(E, K-1, N-K)");
    if (!c->polish_evidence_gate)
      return fail(FBME_ERR_INVALID, "residual exchange requires the evidence gate");
  }
  if (!(c->uamp_damping >= 0.f && c->uamp_damping < 1.f) || !(c->damping >= 0.f && c->damping < 1.f))
    return fail(FBME_ERR_INVALID, "damping values must be in [0, 1)");
  if (N * s.B > (1LL << 40)) return fail(FBME_ERR_INVALID, "batch too large");
  // Elementwise, top-k and polish launches put the scenes of a bucket on
  // gridDim.y / gridDim.z, whose limit is 65535.
  if (s.B > 65535)
    return fail(FBME_ERR_UNSUPPORTED, "more than 65535 scenes of one shape in a plan are not built");
  if (N > 524288 || s.n2 > 512)
    return fail(FBME_ERR_UNSUPPORTED, "grids above 524288 points or N2 > 512 are not built");
  if (static_cast<long long>((s.n1 + 15) / 16) * c->exchange_size > 2048)
    return fail(FBME_ERR_UNSUPPORTED, "exchange candidate count above 2048");
  if (c->dft_terms != 0 && !fbme::dft_n_tile_ok(c->dft_terms, nt, s))
    return fail(FBME_ERR_INVALID, "dft_n_tile must be 64, 128 or 256 with 3 terms (128 with 6) and give at "
                                  "most 64 tiles per scene in every stage");
  return FBME_OK;
}

fbme::DevConfig dev_config(const FbmeConfig& c) {
  fbme::DevConfig d{};
  d.uamp_damping = c.uamp_damping;
  d.damping = c.damping;
  d.blend = c.initialization_blend;
  d.init_noise = c.initial_noise_fraction;
  d.fixed_noise = c.fixed_noise_variance;
  d.min_var = c.min_variance;
  d.max_prec = c.max_precision;
  d.hyper_shape = c.hyper_shape;
  d.hyper_rate = c.hyper_rate;
  d.noise_shape = c.noise_shape;
  d.noise_rate = c.noise_rate;
  d.noise_evidence = c.noise_update == 1;
  d.polish_size = c.polish_size;
  d.polish_iters = c.polish_iterations;
  d.prune_tail = c.polish_prune_tail;
  d.reinit = c.polish_reinitialize;
  d.gate = c.polish_evidence_gate;
  d.polish_damping = c.polish_damping;
  d.margin_factor = c.evidence_margin_factor;
  d.exchange = c.exchange_size;
  d.fixed_budget = c.fixed_budget_diagnostics;
  d.jitter = c.cholesky_jitter_multiplier;
  d.false_alarm = c.support_false_alarm_budget;
  d.terms = c.dft_terms;
  d.uamp_iters = c.uamp_iterations;
  return d;
}

}  // namespace

namespace fbme {
// Error reporting and table sizing shared with the cg translation unit.
int api_fail(int code, const std::string& msg) { return fail(code, msg); }
size_t dft_table_bytes(int L, int terms) { return table_bytes(L, terms, default_n_tile(terms)); }
}  // namespace fbme

// One shape bucket: an equal-shape batch with its own tables, state and
// resolved config, placed at `base` in the plan workspace.
struct Bucket {
  fbme::BatchShape s;
  FbmeConfig cfg;
  fbme::DevConfig dc;
  fbme::DftTables tables;
  fbme::UampBuffers u;
  fbme::PolishBuffers p;
  int* status;
  Layout L;
  size_t base;
  int first;       // first scene in bucket order
  long long pix0;  // first pixel in bucket order
  long long smp0;  // first sample in bucket order
  float2* ymask;   // masked copy of the observations (under an observation mask)
  bool certify = false;  // global certificate + support repairs after the polish
  FbmeCertificate cert{};
};

// Where scene i (caller order) lives: samples and pixels in the caller's
// packed buffers and in bucket order, and its bucket-order index.
struct SceneMap {
  long long caller_smp, bucket_smp, caller_pix, bucket_pix;
  int m, n, bucket_scene, pad;
};

// Bucket-order staging of an uneven plan (workspace offsets).
struct Staging {
  size_t map, y, x, var, prec, mask, noise, dof, nle, trace, exch, fbg, fbn, fbd, fbm, thr, active, aval, status;
  size_t total;
};

struct FbmePlan {
  std::vector<Bucket> bk;
  FbmeConfig cfg;  // the caller's config
  int B = 0;
  bool uneven = false;
  uint8_t* ws = nullptr;
  Staging stg{};
  SceneMap* map = nullptr;  // device [B]
  std::vector<cudaStream_t> streams;  // buckets 1.. of an uneven plan
  std::vector<cudaEvent_t> events;    // fork, then one join per bucket 1..
  ~FbmePlan() {
    for (cudaStream_t s : streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
  }
};

namespace {

// Buckets of a scene list: shapes in order of first appearance, with the
// scenes' bucket and rank.
struct Grouping {
  std::vector<FbmeShape> shape;
  std::vector<int> count, scene_bucket, scene_rank;
};

bool same(const FbmeShape& a, const FbmeShape& b) {
  return a.n1 == b.n1 && a.n2 == b.n2 && a.m1 == b.m1 && a.m2 == b.m2;
}

Grouping group_scenes(const FbmeShape* shapes, int n) {
  Grouping G;
  G.scene_bucket.resize(n);
  G.scene_rank.resize(n);
  for (int i = 0; i < n; ++i) {
    int b = 0;
    while (b < static_cast<int>(G.shape.size()) && !same(G.shape[b], shapes[i])) ++b;
    if (b == static_cast<int>(G.shape.size())) {
      G.shape.push_back(shapes[i]);
      G.count.push_back(0);
    }
    G.scene_bucket[i] = b;
    G.scene_rank[i] = G.count[b]++;
  }
  return G;
}

// The bucket's config: the caller's with the matching FbmeShapeParams
// applied; its stage tile width in *nt.
FbmeConfig bucket_config(const FbmeConfig& c, const FbmeShape& shape, const FbmeShapeParams* params,
                         int n_params, int* nt) {
  FbmeConfig r = c;
  *nt = default_n_tile(c.dft_terms);
  for (int i = 0; params && i < n_params; ++i) {
    const FbmeShapeParams& q = params[i];
    if (!same(q.shape, shape)) continue;
    if (q.uamp_iterations > 0) r.uamp_iterations = q.uamp_iterations;
    if (q.uamp_damping >= 0.f) r.uamp_damping = q.uamp_damping;
    if (q.exchange_size >= 0) r.exchange_size = q.exchange_size;
    if (q.dft_n_tile > 0) *nt = q.dft_n_tile;
  }
  return r;
}

// Everything plan creation needs to know before touching the device.
struct PlanSpec {
  Grouping G;
  std::vector<Bucket> bk;
  Staging stg{};
  size_t total = 0;
};

int plan_spec(const FbmeShape* shapes, int n, const FbmeConfig* c, const FbmeShapeParams* params,
              int n_params, PlanSpec* out) {
  if (!shapes || !c || n < 1) return fail(FBME_ERR_INVALID, "shapes, config and n_scenes >= 1 are required");
  if (n_params < 0 || (n_params > 0 && !params)) return fail(FBME_ERR_INVALID, "bad shape parameter list");
  for (int i = 0; i < n; ++i) {
    const int rc = check_shape(shapes[i]);
    if (rc != FBME_OK) return rc;
  }
  PlanSpec& P = *out;
  P.G = group_scenes(shapes, n);
  const int nb = static_cast<int>(P.G.shape.size());
  size_t off = 0;
  int first = 0;
  long long pix = 0, smp = 0;
  for (int b = 0; b < nb; ++b) {
    Bucket k{};
    const FbmeShape& sh = P.G.shape[b];
    k.s = fbme::BatchShape{P.G.count[b], sh.n1, sh.n2, sh.m1, sh.m2};
    int nt = 0;
    k.cfg = bucket_config(*c, sh, params, n_params, &nt);
    const int rc = check_bucket(k.s, &k.cfg, nt);
    if (rc != FBME_OK) return rc;
    if (nb > 1 && (k.cfg.polish_size != c->polish_size || k.cfg.polish_iterations != c->polish_iterations))
      return fail(FBME_ERR_INVALID, "an uneven plan needs one polish size and iteration count");
    k.tables.n_tile = nt;
    k.L = make_layout(k.s, k.cfg, nt);
    k.base = off;
    off = align256(off + k.L.total);
    // each bucket's staging starts on a 256-byte boundary
    pix = (pix + 255) & ~255LL;
    smp = (smp + 31) & ~31LL;
    k.first = first;
    k.pix0 = pix;
    k.smp0 = smp;
    first += k.s.B;
    pix += k.s.B * k.s.n();
    smp += k.s.B * k.s.m();
    P.bk.push_back(k);
  }
  if (nb > 1) {
    if (n > 65535) return fail(FBME_ERR_UNSUPPORTED, "an uneven plan holds at most 65535 scenes");
    Staging& S = P.stg;
    auto take = [&](size_t bytes) {
      const size_t o = off;
      off = align256(off + bytes);
      return o;
    };
    const size_t B = n, Pn = c->polish_iterations, K = c->polish_size;
    S.map = take(B * sizeof(SceneMap));
    S.y = take(smp * sizeof(float2));
    S.x = take(pix * sizeof(float2));
    S.var = take(pix * sizeof(float));
    S.prec = take(pix * sizeof(float));
    S.mask = take(pix);
    S.noise = take(B * 4);
    S.dof = take(B * 4);
    S.nle = take(B * 4);
    S.trace = take(B * Pn * 4);
    S.exch = take(B * 8);
    S.fbg = take(B * 4);
    S.fbn = take(B * 4);
    S.fbd = take(B * 4);
    S.fbm = take(B);
    S.thr = take(B * 4);
    S.active = take(B * K * 8);
    S.aval = take(B * K * 8);
    S.status = take(B * 4);
    S.total = off;
  }
  P.total = off;
  return FBME_OK;
}

// Pointers of one bucket inside the workspace; tables filled on `st`.
void bind_bucket(Bucket& k, uint8_t* ws, cudaStream_t st) {
  uint8_t* w = ws + k.base;
  const Layout& L = k.L;
  const fbme::BatchShape& s = k.s;
  k.dc = dev_config(k.cfg);
  const int nt = k.tables.n_tile, parts = k.cfg.dft_terms == 6 ? 3 : 2;
  auto build_table = [&](size_t off, int Lx, int sign) {
    if (k.cfg.dft_terms == 0) return;
    fbme::launch_twiddle_table(w + off, Lx, sign, nt, ceil_div(2LL * Lx, nt), ceil_div(2LL * Lx, 64), parts, st);
  };
  build_table(L.tab_f2, s.n2, -1);
  build_table(L.tab_a2, s.n2, +1);
  if (s.n1 != s.n2) {
    build_table(L.tab_f1, s.n1, -1);
    build_table(L.tab_a1, s.n1, +1);
  }
  k.tables.fwd_n2 = w + L.tab_f2;
  k.tables.adj_n2 = w + L.tab_a2;
  k.tables.fwd_n1 = w + L.tab_f1;
  k.tables.adj_n1 = w + L.tab_a1;
  k.tables.kchunks_n1 = ceil_div(2LL * s.n1, 64);
  k.tables.kchunks_n2 = ceil_div(2LL * s.n2, 64);
  k.tables.fft_n1 = k.tables.fft_n2 = nullptr;
  if (k.cfg.dft_terms == 0) {
    float2* f1 = reinterpret_cast<float2*>(w + L.fft1);
    float2* f2 = reinterpret_cast<float2*>(w + L.fft2);
    fbme::launch_fft_twiddles(f1, s.n1, st);
    fbme::launch_fft_twiddles(f2, s.n2, st);
    k.tables.fft_n1 = f1;
    k.tables.fft_n2 = f2;
  }
  float2* dir1 = reinterpret_cast<float2*>(w + L.dir1);
  float2* dir2 = reinterpret_cast<float2*>(w + L.dir2);
  fbme::launch_dirichlet(dir1, s.m1, s.n1, st);
  fbme::launch_dirichlet(dir2, s.m2, s.n2, st);

  fbme::UampBuffers& u = k.u;
  u = fbme::UampBuffers{};
  u.mu = reinterpret_cast<float2*>(w + L.mu);
  u.bp = reinterpret_cast<float2*>(w + L.bp);
  u.msg = reinterpret_cast<float2*>(w + L.msg);
  u.pred = reinterpret_cast<float2*>(w + L.pred);
  u.tmp = reinterpret_cast<float2*>(w + L.tmp);
  u.split = k.cfg.dft_terms == 3;
  u.lift = reinterpret_cast<float2*>(w + L.lift);
  u.mask = nullptr;
  k.ymask = reinterpret_cast<float2*>(w + L.ymask);
  u.var = reinterpret_cast<float*>(w + L.var);
  u.gamma = reinterpret_cast<float*>(w + L.gamma);
  u.part = reinterpret_cast<double*>(w + L.part);
  u.keys = reinterpret_cast<uint32_t*>(w + L.keys);
  float* sc = reinterpret_cast<float*>(w + L.scal);
  const int B = s.B;
  u.sc = fbme::Scalars{sc, sc + B, sc + 2 * B, sc + 3 * B, sc + 4 * B,
                       sc + 5 * B, sc + 6 * B, sc + 7 * B, sc + 8 * B, sc + 9 * B};
  k.status = reinterpret_cast<int*>(w + L.status);
  u.status = k.status;

  fbme::PolishBuffers& p = k.p;
  p = fbme::PolishBuffers{};
  p.bp = u.bp;
  p.mu = u.mu;
  p.dir1 = dir1;
  p.dir2 = dir2;
  p.var = u.var;
  p.gamma = u.gamma;
  p.sc = u.sc;
  p.active = reinterpret_cast<int*>(w + L.active);
  p.score = reinterpret_cast<float*>(w + L.score);
  p.pstate = w + L.pstate;
  p.xcand_val = reinterpret_cast<float*>(w + L.xval);
  p.xcand_idx = reinterpret_cast<int*>(w + L.xidx);
  p.keys = u.keys;
  p.cand_key = reinterpret_cast<uint32_t*>(w + L.ckey);
  p.cand_idx = reinterpret_cast<int*>(w + L.cidx);
  p.status = k.status;
}

// Gather: the caller's scene-order samples into bucket order.
__global__ void gather_samples_kernel(const SceneMap* map, const float2* y, float2* ybuf) {
  const SceneMap m = map[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.m; i += gridDim.x * blockDim.x)
    ybuf[m.bucket_smp + i] = y[m.caller_smp + i];
}

// Output fields moved by the scatter: per-pixel ones (count 0) and
// per-scene ones of `count` elements; NULL destinations are skipped.
struct ScatterField {
  const void* src;
  void* dst;
  int elem_bytes;  // 1, 4 or 8
  int count;       // 0 = one element per pixel
};
constexpr int kScatterFields = 20;
struct ScatterArgs {
  ScatterField f[kScatterFields];
  int n;
};

template <typename T>
__device__ void copy_elems(const ScatterField& f, long long src0, long long dst0, long long n, long long i0,
                           long long step) {
  const T* s = static_cast<const T*>(f.src) + src0;
  T* d = static_cast<T*>(f.dst) + dst0;
  for (long long i = i0; i < n; i += step) d[i] = s[i];
}

// Scatter: bucket-order outputs back to the caller's scene order.  Block
// (x, scene, field) copies a strided part of one field of one scene.
__global__ void scatter_outputs_kernel(const SceneMap* map, const __grid_constant__ ScatterArgs a) {
  const ScatterField& f = a.f[blockIdx.z];
  if (!f.dst) return;
  const SceneMap m = map[blockIdx.y];
  long long src0, dst0, n;
  if (f.count == 0) {
    src0 = m.bucket_pix;
    dst0 = m.caller_pix;
    n = m.n;
  } else {
    src0 = static_cast<long long>(m.bucket_scene) * f.count;
    dst0 = static_cast<long long>(blockIdx.y) * f.count;
    n = f.count;
  }
  const long long i0 = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  if (f.elem_bytes == 8)
    copy_elems<unsigned long long>(f, src0, dst0, n, i0, step);
  else if (f.elem_bytes == 4)
    copy_elems<unsigned int>(f, src0, dst0, n, i0, step);
  else
    copy_elems<unsigned char>(f, src0, dst0, n, i0, step);
}

int check_outputs(const FbmeConfig& c, const FbmeOutputs* out) {
  if (!out->x || !out->posterior_variance || !out->precision || !out->noise_variance ||
      !out->effective_dof || !out->negative_log_evidence || !out->evidence_trace || !out->status)
    return fail(FBME_ERR_INVALID, "required output buffer is NULL");
  if (c.fixed_budget_diagnostics &&
      (!out->fixed_budget_gamma_residual || !out->fixed_budget_noise_residual ||
       !out->fixed_budget_objective_decrease || !out->fixed_budget_monotone))
    return fail(FBME_ERR_INVALID, "fixed-budget diagnostics need their four output buffers");
  return FBME_OK;
}

// Bucket b's outputs inside the uneven plan's bucket-order staging; an
// optional field stays NULL where the caller's is.
FbmeOutputs bucket_outputs(const FbmePlan* P, const Bucket& k, const FbmeOutputs& caller) {
  const Staging& S = P->stg;
  uint8_t* w = P->ws;
  const long long f = k.first, px = k.pix0;
  const long long Pn = P->cfg.polish_iterations, K = P->cfg.polish_size;
  auto at = [&](size_t off, long long elems, int bytes) { return w + off + elems * bytes; };
  FbmeOutputs o{};
  o.x = at(S.x, px, 8);
  o.posterior_variance = reinterpret_cast<float*>(at(S.var, px, 4));
  o.precision = reinterpret_cast<float*>(at(S.prec, px, 4));
  o.support_mask = caller.support_mask ? at(S.mask, px, 1) : nullptr;
  o.noise_variance = reinterpret_cast<float*>(at(S.noise, f, 4));
  o.effective_dof = reinterpret_cast<float*>(at(S.dof, f, 4));
  o.negative_log_evidence = reinterpret_cast<float*>(at(S.nle, f, 4));
  o.evidence_trace = reinterpret_cast<float*>(at(S.trace, f * Pn, 4));
  o.support_exchanges_accepted =
      caller.support_exchanges_accepted ? reinterpret_cast<int64_t*>(at(S.exch, f, 8)) : nullptr;
  o.fixed_budget_gamma_residual =
      caller.fixed_budget_gamma_residual ? reinterpret_cast<float*>(at(S.fbg, f, 4)) : nullptr;
  o.fixed_budget_noise_residual =
      caller.fixed_budget_noise_residual ? reinterpret_cast<float*>(at(S.fbn, f, 4)) : nullptr;
  o.fixed_budget_objective_decrease =
      caller.fixed_budget_objective_decrease ? reinterpret_cast<float*>(at(S.fbd, f, 4)) : nullptr;
  o.fixed_budget_monotone = caller.fixed_budget_monotone ? at(S.fbm, f, 1) : nullptr;
  o.support_score_threshold =
      caller.support_score_threshold ? reinterpret_cast<float*>(at(S.thr, f, 4)) : nullptr;
  o.active_indices = caller.active_indices ? reinterpret_cast<int64_t*>(at(S.active, f * K, 8)) : nullptr;
  o.active_values = caller.active_values ? at(S.aval, f * K, 8) : nullptr;
  o.status = reinterpret_cast<int32_t*>(at(S.status, f, 4));
  return o;
}

// The scatter moves only the fields the polish writes for this config (the
// support mask and threshold need the false-alarm budget, the four
// fixed-budget diagnostics their switch), so the caller's other buffers
// stay untouched, as with an equal-shape plan.
ScatterArgs scatter_args(const FbmePlan* P, const FbmeOutputs& c) {
  const Staging& S = P->stg;
  const uint8_t* w = P->ws;
  const int Pn = P->cfg.polish_iterations, K = P->cfg.polish_size;
  const bool mask = P->cfg.support_false_alarm_budget > 0.f, fb = P->cfg.fixed_budget_diagnostics != 0;
  ScatterArgs a{};
  auto add = [&](size_t off, void* dst, int bytes, int count, bool written = true) {
    a.f[a.n++] = ScatterField{w + off, written ? dst : nullptr, bytes, count};
  };
  add(S.x, c.x, 8, 0);
  add(S.var, c.posterior_variance, 4, 0);
  add(S.prec, c.precision, 4, 0);
  add(S.mask, c.support_mask, 1, 0, mask);
  add(S.noise, c.noise_variance, 4, 1);
  add(S.dof, c.effective_dof, 4, 1);
  add(S.nle, c.negative_log_evidence, 4, 1);
  add(S.trace, c.evidence_trace, 4, Pn);
  add(S.exch, c.support_exchanges_accepted, 8, 1);
  add(S.fbg, c.fixed_budget_gamma_residual, 4, 1, fb);
  add(S.fbn, c.fixed_budget_noise_residual, 4, 1, fb);
  add(S.fbd, c.fixed_budget_objective_decrease, 4, 1, fb);
  add(S.fbm, c.fixed_budget_monotone, 1, 1, fb);
  add(S.thr, c.support_score_threshold, 4, 1, mask);
  add(S.active, c.active_indices, 8, K);
  add(S.aval, c.active_values, 8, K);
  add(S.status, c.status, 4, 1);
  return a;
}

// Polish and outputs of one bucket on `st` (its UAMP stage done).  The
// status words of an uneven plan's buckets already live in the staging
// area the outputs point at.
void polish_bucket(const Bucket& k, const float2* y, const FbmeOutputs& out, cudaStream_t st,
                   fbme::Profiler* prof = nullptr) {
  fbme::PolishBuffers p = k.p;
  p.y = y;
  fbme::polish_run(k.s, k.dc, p, out, st, prof, k.certify ? &k.cert : nullptr);
  if (out.status != k.status)
    cudaMemcpyAsync(out.status, k.status, k.s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
}

// The whole solve of one bucket on `st`: status reset, UAMP, polish and
// outputs.
void run_bucket(const Bucket& k, const float2* y, const FbmeOutputs& out, cudaStream_t st,
                fbme::Profiler* prof = nullptr) {
  cudaMemsetAsync(k.status, 0, k.s.B * sizeof(int), st);
  fbme::UampBuffers u = k.u;
  if (k.u.mask) {  // the solve reads the masked copy of the observations
    fbme::mask_data(k.s, y, k.u.mask, k.ymask, st);
    y = k.ymask;
  }
  u.y = y;
  fbme::uamp_run(k.s, k.tables, k.dc, u, st, prof);
  polish_bucket(k, y, out, st, prof);
}

int create_plan(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                const FbmeShapeParams* params, int32_t n_params, void* workspace, size_t workspace_bytes,
                fbme_stream_t stream, FbmePlan** plan) {
  if (!plan) return fail(FBME_ERR_INVALID, "plan output pointer is NULL");
  *plan = nullptr;
  PlanSpec spec;
  int rc = plan_spec(shapes, n_scenes, cfg, params, n_params, &spec);
  if (rc != FBME_OK) return rc;
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return fail(FBME_ERR_WORKSPACE, "workspace must be a 256-byte aligned device pointer");
  if (workspace_bytes < spec.total)
    return fail(FBME_ERR_WORKSPACE, "workspace smaller than fbme_plan_workspace_bytes()");
  cudaError_t e = fbme::set_dft_attributes();
  if (e == cudaSuccess) e = fbme::set_polish_attributes();
  if (e == cudaSuccess) e = fbme::set_fft_attributes();
  if (e == cudaSuccess) e = fbme::set_cnn_attributes();
  if (e != cudaSuccess) return fail(FBME_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));

  FbmePlan* P = new (std::nothrow) FbmePlan();
  if (!P) return fail(FBME_ERR_INVALID, "out of host memory");
  P->cfg = *cfg;
  P->B = n_scenes;
  P->ws = static_cast<uint8_t*>(workspace);
  P->bk = spec.bk;
  P->uneven = P->bk.size() > 1;
  P->stg = spec.stg;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  for (Bucket& k : P->bk) bind_bucket(k, P->ws, st);
  if (P->uneven) {
    // status words in the bucket-order staging: one reset for all buckets
    for (Bucket& k : P->bk) {
      int* sw = reinterpret_cast<int*>(P->ws + P->stg.status) + k.first;
      k.status = k.u.status = k.p.status = sw;
    }
    std::vector<SceneMap> m(n_scenes);
    long long csmp = 0, cpix = 0;
    for (int i = 0; i < n_scenes; ++i) {
      const Bucket& k = P->bk[spec.G.scene_bucket[i]];
      const int r = spec.G.scene_rank[i];
      m[i].caller_smp = csmp;
      m[i].caller_pix = cpix;
      m[i].bucket_smp = k.smp0 + r * k.s.m();
      m[i].bucket_pix = k.pix0 + r * k.s.n();
      m[i].m = static_cast<int>(k.s.m());
      m[i].n = static_cast<int>(k.s.n());
      m[i].bucket_scene = k.first + r;
      csmp += k.s.m();
      cpix += k.s.n();
    }
    P->map = reinterpret_cast<SceneMap*>(P->ws + P->stg.map);
    e = cudaMemcpyAsync(P->map, m.data(), m.size() * sizeof(SceneMap), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // m is pageable host memory
    for (size_t b = 1; b < P->bk.size() && e == cudaSuccess; ++b) {
      cudaStream_t s2 = nullptr;
      e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
      if (e == cudaSuccess) P->streams.push_back(s2);
    }
    for (size_t i = 0; i < P->bk.size() && e == cudaSuccess; ++i) {
      cudaEvent_t ev = nullptr;
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) P->events.push_back(ev);
    }
    if (e != cudaSuccess) {
      delete P;
      return fail(FBME_ERR_CUDA, std::string("uneven plan setup: ") + cudaGetErrorString(e));
    }
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    delete P;
    return fail(FBME_ERR_CUDA, std::string("plan tables: ") + cudaGetErrorString(e));
  }
  *plan = P;
  return FBME_OK;
}

int single_bucket(const FbmePlan* plan) {
  if (!plan) return fail(FBME_ERR_INVALID, "plan is NULL");
  if (plan->uneven)
    return fail(FBME_ERR_UNSUPPORTED, "stage entry points need a plan whose scenes share one shape");
  return FBME_OK;
}

}  // namespace

extern "C" {

const char* fbme_last_error(void) { return g_last_error.c_str(); }
const char* fbme_version(void) { return "fbme-b200 0.2.0 (sm_100a)"; }

size_t fbme_plan_workspace_bytes_ex(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                                    const FbmeShapeParams* params, int32_t n_params) {
  PlanSpec spec;
  if (plan_spec(shapes, n_scenes, cfg, params, n_params, &spec) != FBME_OK) return 0;
  return spec.total;
}

size_t fbme_plan_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg) {
  return fbme_plan_workspace_bytes_ex(shapes, n_scenes, cfg, nullptr, 0);
}

int fbme_plan_create_ex(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                        const FbmeShapeParams* params, int32_t n_params, void* workspace,
                        size_t workspace_bytes, fbme_stream_t stream, FbmePlan** plan) {
  return create_plan(shapes, n_scenes, cfg, params, n_params, workspace, workspace_bytes, stream, plan);
}

int fbme_plan_create(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                     void* workspace, size_t workspace_bytes, fbme_stream_t stream,
                     FbmePlan** plan) {
  return create_plan(shapes, n_scenes, cfg, nullptr, 0, workspace, workspace_bytes, stream, plan);
}

int32_t fbme_plan_bucket_count(const FbmePlan* plan) {
  return plan ? static_cast<int32_t>(plan->bk.size()) : 0;
}

int fbme_plan_bucket(const FbmePlan* plan, int32_t bucket, FbmeShapeParams* resolved, int32_t* n_scenes) {
  if (!plan || !resolved || !n_scenes) return fail(FBME_ERR_INVALID, "NULL argument");
  if (bucket < 0 || bucket >= static_cast<int32_t>(plan->bk.size()))
    return fail(FBME_ERR_INVALID, "bucket index out of range");
  const Bucket& k = plan->bk[bucket];
  resolved->shape = FbmeShape{k.s.n1, k.s.n2, k.s.m1, k.s.m2};
  resolved->uamp_iterations = k.cfg.uamp_iterations;
  resolved->uamp_damping = k.cfg.uamp_damping;
  resolved->exchange_size = k.cfg.exchange_size;
  resolved->dft_n_tile = k.tables.n_tile;
  *n_scenes = k.s.B;
  return FBME_OK;
}

size_t fbme_plan_warm_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes) {
  if (!shapes || n_scenes < 1) return 0;
  if (fbme::cnn_check(n_scenes, shapes[0].n1, shapes[0].n2)) return 0;
  return fbme::cnn_workspace_bytes(n_scenes, shapes[0].n1, shapes[0].n2);
}

int fbme_plan_set_warm_start(FbmePlan* plan, const float* params, void* workspace,
                             size_t workspace_bytes) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  Bucket& k = plan->bk[0];
  if (!params) {
    k.u.warm_params = nullptr;
    k.u.warm_ws = nullptr;
    return FBME_OK;
  }
  if (const char* why = fbme::cnn_check(k.s.B, k.s.n1, k.s.n2))
    return fail(FBME_ERR_UNSUPPORTED, why);
  const size_t need = fbme::cnn_workspace_bytes(k.s.B, k.s.n1, k.s.n2);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0 || workspace_bytes < need)
    return fail(FBME_ERR_WORKSPACE, "warm-start workspace smaller than fbme_plan_warm_workspace_bytes() "
                                    "or not 256-byte aligned");
  k.u.warm_params = params;
  k.u.warm_ws = workspace;
  k.u.warm_map = nullptr;
  return FBME_OK;
}

int fbme_plan_set_warm_prior_map(FbmePlan* plan, const float* map) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (map && (reinterpret_cast<uintptr_t>(map) & 3u) != 0) return fail(FBME_ERR_INVALID, "misaligned map");
  Bucket& k = plan->bk[0];
  k.u.warm_map = map;
  if (map) {
    k.u.warm_params = nullptr;
    k.u.warm_ws = nullptr;
  }
  return FBME_OK;
}

int fbme_plan_destroy(FbmePlan* plan) {
  delete plan;
  return FBME_OK;
}

static int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(FBME_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FBME_OK;
}

int fbme_dft_forward(FbmePlan* plan, const void* coefficients, void* data, fbme_stream_t stream) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (!coefficients || !data) return fail(FBME_ERR_INVALID, "NULL argument");
  const Bucket& k = plan->bk[0];
  fbme::dft_forward(k.s, k.tables, k.cfg.dft_terms, static_cast<const float2*>(coefficients),
                    static_cast<float2*>(data), k.u.tmp, k.status, reinterpret_cast<cudaStream_t>(stream));
  return check_launch("dft_forward");
}

int fbme_dft_adjoint(FbmePlan* plan, const void* data, void* coefficients, fbme_stream_t stream) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (!coefficients || !data) return fail(FBME_ERR_INVALID, "NULL argument");
  const Bucket& k = plan->bk[0];
  fbme::dft_adjoint(k.s, k.tables, k.cfg.dft_terms, static_cast<const float2*>(data),
                    static_cast<float2*>(coefficients), k.u.tmp, k.status,
                    reinterpret_cast<cudaStream_t>(stream));
  return check_launch("dft_adjoint");
}

int fbme_uamp_run(FbmePlan* plan, const void* y, fbme_stream_t stream) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (!y) return fail(FBME_ERR_INVALID, "NULL argument");
  const Bucket& k = plan->bk[0];
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaMemsetAsync(k.status, 0, k.s.B * sizeof(int), st);
  fbme::UampBuffers u = k.u;
  u.y = static_cast<const float2*>(y);
  if (k.u.mask) {
    fbme::mask_data(k.s, u.y, k.u.mask, k.ymask, st);
    u.y = k.ymask;
  }
  fbme::uamp_run(k.s, k.tables, k.dc, u, st);
  return check_launch("uamp_run");
}

int fbme_polish_run(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (!y || !out) return fail(FBME_ERR_INVALID, "NULL argument");
  const Bucket& k = plan->bk[0];
  if ((rc = check_outputs(k.cfg, out)) != FBME_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  fbme::PolishBuffers p = k.p;
  p.y = static_cast<const float2*>(y);
  if (k.u.mask) {
    fbme::mask_data(k.s, p.y, k.u.mask, k.ymask, st);
    p.y = k.ymask;
  }
  fbme::polish_run(k.s, k.dc, p, *out, st, nullptr, k.certify ? &k.cert : nullptr);
  cudaMemcpyAsync(out->status, k.status, k.s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
  return check_launch("polish_run");
}

namespace {
// Gather, buckets, scatter of an uneven plan.  The UAMP stage of all
// buckets runs as merged launches on `st` (one launch per step for every
// bucket); then, with prof == nullptr, every polish step is one launch over
// all buckets (polish_run_multi); with a profiler the buckets' polishes run
// one after another on `st`.
void replay_uneven(FbmePlan* P, const float2* y, const FbmeOutputs& out, cudaStream_t st,
                   fbme::Profiler* prof) {
  float2* ybuf = reinterpret_cast<float2*>(P->ws + P->stg.y);
  const int gx = 8;
  FBME_TIMED(prof, FBME_GROUP_INIT, (gather_samples_kernel<<<dim3(gx, P->B), 256, 0, st>>>(P->map, y, ybuf)));
  const int nb = static_cast<int>(P->bk.size());
  cudaMemsetAsync(P->ws + P->stg.status, 0, static_cast<size_t>(P->B) * sizeof(int), st);
  std::vector<fbme::UampJob> jobs(nb);
  for (int b = 0; b < nb; ++b) {
    const Bucket& k = P->bk[b];
    jobs[b] = fbme::UampJob{k.s, k.tables, k.dc, k.u};
    jobs[b].u.y = ybuf + k.smp0;
  }
  fbme::uamp_run_multi(jobs.data(), nb, st, prof, P->streams.data(), P->events.data(),
                       static_cast<int>(P->streams.size()));
  if (!prof) {
    // every polish step is one launch over all buckets
    std::vector<fbme::PolishBucket> pb(nb);
    for (int b = 0; b < nb; ++b) {
      const Bucket& k = P->bk[b];
      pb[b].s = k.s;
      pb[b].c = k.dc;
      pb[b].p = k.p;
      pb[b].p.y = ybuf + k.smp0;
      pb[b].out = bucket_outputs(P, k, out);
    }
    fbme::polish_run_multi(pb.data(), nb, st);
  } else {
    for (int b = 0; b < nb; ++b) {
      const Bucket& k = P->bk[b];
      polish_bucket(k, ybuf + k.smp0, bucket_outputs(P, k, out), st, prof);
    }
  }
  const ScatterArgs a = scatter_args(P, out);
  FBME_TIMED(prof, FBME_GROUP_OUTPUT,
             (scatter_outputs_kernel<<<dim3(gx, P->B, a.n), 256, 0, st>>>(P->map, a)));
}
}  // namespace

int fbme_plan_replay(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream) {
  if (!plan || !y || !out) return fail(FBME_ERR_INVALID, "NULL argument");
  if (!plan->uneven) {
    int rc = fbme_uamp_run(plan, y, stream);
    if (rc != FBME_OK) return rc;
    return fbme_polish_run(plan, y, out, stream);
  }
  int rc = check_outputs(plan->cfg, out);
  if (rc != FBME_OK) return rc;
  replay_uneven(plan, static_cast<const float2*>(y), *out, reinterpret_cast<cudaStream_t>(stream), nullptr);
  return check_launch("uneven replay");
}

const char* fbme_profile_group_name(int32_t group) {
  static const char* names[FBME_NUM_GROUPS] = {
      "init", "adjoint_1", "adjoint_denoise", "forward_1", "forward_residual", "scalars",
      "sweep1_denoise", "topk", "polish", "exchange_score", "output", "adjoint_2", "message", "certificate"};
  return (group >= 0 && group < FBME_NUM_GROUPS) ? names[group] : "";
}

int fbme_plan_profile(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream,
                      float* group_ms, int32_t* group_launches, int32_t n_groups) {
  if (!plan || !y || !out || !group_ms || !group_launches)
    return fail(FBME_ERR_INVALID, "NULL argument");
  int rc = check_outputs(plan->cfg, out);
  if (rc != FBME_OK) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  fbme::Profiler* prof = new (std::nothrow) fbme::Profiler();
  if (!prof) return fail(FBME_ERR_INVALID, "out of host memory");
  prof->st = st;
  for (int i = 0; i < 2 * fbme::Profiler::kMax; ++i) cudaEventCreate(&prof->ev[i]);
  if (plan->uneven)
    replay_uneven(plan, static_cast<const float2*>(y), *out, st, prof);
  else
    run_bucket(plan->bk[0], static_cast<const float2*>(y), *out, st, prof);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    rc = fail(FBME_ERR_CUDA, std::string("profile: ") + cudaGetErrorString(e));
  } else {
    for (int g = 0; g < n_groups; ++g) {
      group_ms[g] = 0.f;
      group_launches[g] = 0;
    }
    for (int i = 0; i < prof->n; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, prof->ev[2 * i], prof->ev[2 * i + 1]);
      const int g = prof->group[i];
      if (g < n_groups) {
        group_ms[g] += ms;
        group_launches[g] += 1;
      }
    }
  }
  for (int i = 0; i < 2 * fbme::Profiler::kMax; ++i) cudaEventDestroy(prof->ev[i]);
  delete prof;
  return rc;
}

int fbme_uamp_prior_update(const void* mean, const float* posterior_variance, const float* old_prior,
                           const float* prior_floor, int32_t batch, int64_t n, float hyper_shape,
                           float hyper_rate, float damping, float maximum, float* out,
                           fbme_stream_t stream) {
  if (!mean || !posterior_variance || !old_prior || !prior_floor || !out)
    return fail(FBME_ERR_INVALID, "NULL argument");
  if (batch < 1 || batch > 65535 || n < 1)
    return fail(FBME_ERR_INVALID, "batch must be in [1, 65535] and n positive");
  if ((n + 1023) / 1024 > 0x7fffffffLL) return fail(FBME_ERR_INVALID, "n too large");
  if ((reinterpret_cast<uintptr_t>(mean) & 7u) != 0 || (reinterpret_cast<uintptr_t>(posterior_variance) & 3u) != 0 ||
      (reinterpret_cast<uintptr_t>(old_prior) & 3u) != 0 || (reinterpret_cast<uintptr_t>(out) & 3u) != 0)
    return fail(FBME_ERR_INVALID, "misaligned complex64 / float32 buffer");
  fbme::uamp_prior_update(static_cast<const float2*>(mean), posterior_variance, old_prior, prior_floor, batch, n,
                          hyper_shape, hyper_rate, damping, maximum, out,
                          reinterpret_cast<cudaStream_t>(stream));
  return check_launch("fbme_uamp_prior_update");
}

size_t fbme_selftest_workspace_bytes(void) { return fbme::stage_selftest_bytes(); }

int fbme_selftest_stage_timeout(void* workspace, size_t workspace_bytes, int32_t* status, int64_t wait_cycles,
                                fbme_stream_t stream) {
  if (!workspace || !status) return fail(FBME_ERR_INVALID, "NULL argument");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255u) != 0 || workspace_bytes < fbme::stage_selftest_bytes())
    return fail(FBME_ERR_WORKSPACE, "workspace smaller than fbme_selftest_workspace_bytes() or not 256-byte aligned");
  if (wait_cycles < 1000 || wait_cycles > 2000000000LL)
    return fail(FBME_ERR_INVALID, "wait_cycles must be in [1e3, 2e9]");
  const cudaError_t e = fbme::stage_selftest(workspace, status, wait_cycles, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(FBME_ERR_CUDA, std::string("fbme_selftest_stage_timeout: ") + cudaGetErrorString(e));
  return FBME_OK;
}

size_t fbme_topk_workspace_bytes(int64_t n, int32_t k, int32_t batch) {
  if (fbme::topk_check(n, k, batch)) return 0;
  return fbme::topk_scratch_bytes(n, k, batch);
}

int fbme_topk(const float* scores, int64_t n, int32_t k, int32_t batch, void* workspace,
              size_t workspace_bytes, int64_t* indices, float* values, fbme_stream_t stream) {
  if (!scores || !indices || !values) return fail(FBME_ERR_INVALID, "NULL argument");
  if (const char* why = fbme::topk_check(n, k, batch)) return fail(FBME_ERR_INVALID, why);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 15u) != 0 ||
      workspace_bytes < fbme::topk_scratch_bytes(n, k, batch))
    return fail(FBME_ERR_WORKSPACE, "workspace smaller than fbme_topk_workspace_bytes() or unaligned");
  fbme::topk_scores(scores, n, k, batch, workspace, indices, values,
                    reinterpret_cast<cudaStream_t>(stream));
  return check_launch("fbme_topk");
}

int fbme_plan_set_observation_mask(FbmePlan* plan, const uint8_t* mask, fbme_stream_t stream) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  Bucket& k = plan->bk[0];
  uint8_t* w = plan->ws + k.base;
  if (!mask) {  // back to the whole M1 x M2 block
    k.u.mask = nullptr;
    k.p.gram2d = nullptr;
    k.dc.m_obs = 0.f;
    return FBME_OK;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  uint8_t* dmask = w + k.L.mask;
  float2* gram = reinterpret_cast<float2*>(w + k.L.gram);
  long long observed = 0;
  const cudaError_t e = fbme::mask_setup(k.s, mask, dmask, gram, w + k.L.gscr, &observed, st);
  if (e != cudaSuccess)
    return fail(FBME_ERR_CUDA, std::string("fbme_plan_set_observation_mask: ") + cudaGetErrorString(e));
  if (observed == 0) return fail(FBME_ERR_INVALID, "observation_mask must retain at least one sample.");
  k.u.mask = dmask;
  k.p.gram2d = gram;
  k.dc.m_obs = static_cast<float>(observed);
  return FBME_OK;
}

size_t fbme_plan_certificate_workspace_bytes(const FbmePlan* plan) {
  if (!plan || plan->uneven || plan->bk.empty()) return 0;
  return fbme::cert_scratch_bytes(plan->bk[0].s);
}

int fbme_plan_set_certificate(FbmePlan* plan, const FbmeCertificate* cert) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  Bucket& k = plan->bk[0];
  if (!cert) {
    k.certify = false;
    k.dc.repairs = 0;
    return FBME_OK;
  }
  if (k.cfg.polish_size < 1)
    return fail(FBME_ERR_UNSUPPORTED, "the global certificate needs the active-set polish (polish_size >= 1)");
  if (cert->support_repairs < 0 || cert->support_repairs > 4)
    return fail(FBME_ERR_INVALID, "uamp_polish_support_repairs must be between 0 and 4.");
  if (k.cfg.polish_iterations + cert->support_repairs > 8)
    return fail(FBME_ERR_UNSUPPORTED, "polish iterations + support repairs above 8");
  if (!cert->inactive_max_evidence_ratio || !cert->inactive_best_index || !cert->inactive_evidence_gain ||
      !cert->inactive_optimal_variance || !cert->support_repairs_accepted || !cert->active_max_evidence_gain ||
      !cert->active_best_index || !cert->active_optimal_variance || !cert->active_max_deletion_gain ||
      !cert->active_penalized_evidence_gain || !cert->coordinate_stationary ||
      !cert->type2_map_coordinate_stationary ||
      (cert->familywise_ratio_threshold > 0.f && !cert->familywise_no_discovery))
    return fail(FBME_ERR_INVALID, "NULL certificate output");
  if (!cert->workspace || (reinterpret_cast<uintptr_t>(cert->workspace) & 255u) != 0 ||
      cert->workspace_bytes < fbme::cert_scratch_bytes(k.s))
    return fail(FBME_ERR_WORKSPACE,
                "certificate workspace smaller than fbme_plan_certificate_workspace_bytes() or not 256-byte aligned");
  k.cert = *cert;
  k.certify = true;
  k.dc.repairs = cert->support_repairs;
  return FBME_OK;
}

int fbme_plan_state(FbmePlan* plan, FbmeState* st) {
  int rc = single_bucket(plan);
  if (rc != FBME_OK) return rc;
  if (!st) return fail(FBME_ERR_INVALID, "NULL argument");
  const fbme::UampBuffers& u = plan->bk[0].u;
  st->mean = u.mu;
  st->variance = u.var;
  st->prior_variance = u.gamma;
  st->message = u.msg;
  st->prediction = u.pred;
  st->backprojection = u.bp;
  st->noise_variance = u.sc.noise;
  st->data_variance = u.sc.dvar;
  return FBME_OK;
}

}  // extern "C"
