// C ABI of the FBME B200 library: plan creation over a caller-owned
// workspace, replay, and stage entry points.  See include/fbme_b200.h.
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "kernels.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Bytes of one split-BF16 twiddle table for axis length L.
size_t table_bytes(int L, int terms) {
  const int nt = terms == 6 ? 128 : 256;
  const int parts = terms == 6 ? 3 : 2;
  return static_cast<size_t>(ceil_div(2LL * L, nt)) * ceil_div(2LL * L, 64) * parts * nt * 128;
}

struct Layout {
  size_t tab_f2, tab_f1, tab_a2, tab_a1, dir1, dir2;
  size_t mu, bp, var, gamma, msg, pred, tmp, keys, part, scal;
  size_t active, score, pstate, xval, xidx, status, ckey, cidx;
  size_t total;
};

Layout make_layout(const fbme::BatchShape& s, const FbmeConfig& c) {
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
  L.tab_f2 = take(table_bytes(s.n2, c.dft_terms));
  L.tab_a2 = take(table_bytes(s.n2, c.dft_terms));
  if (s.n1 != s.n2) {
    L.tab_f1 = take(table_bytes(s.n1, c.dft_terms));
    L.tab_a1 = take(table_bytes(s.n1, c.dft_terms));
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
  const size_t tmp1 = static_cast<size_t>(s.m2) * s.n1, tmp2 = static_cast<size_t>(s.n2) * s.m1;
  L.tmp = take(B * (tmp1 > tmp2 ? tmp1 : tmp2) * sizeof(float2));
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
  L.total = off;
  return L;
}

int validate(const FbmeShape* shapes, int n, const FbmeConfig* c, fbme::BatchShape* out) {
  if (!shapes || !c || n < 1) return fail(FBME_ERR_INVALID, "shapes, config and n_scenes >= 1 are required");
  const FbmeShape s0 = shapes[0];
  for (int i = 0; i < n; ++i) {
    const FbmeShape& s = shapes[i];
    if (s.n1 < 1 || s.n2 < 1 || s.m1 < 1 || s.m2 < 1 || s.m1 > s.n1 || s.m2 > s.n2)
      return fail(FBME_ERR_INVALID, "Each sample dimension must satisfy 0 < M <= N.");
    if (s.n1 != s0.n1 || s.n2 != s0.n2 || s.m1 != s0.m1 || s.m2 != s0.m2)
      return fail(FBME_ERR_UNSUPPORTED, "scenes of different shapes need the uneven-batch plan");
  }
  const long long N = 1LL * s0.n1 * s0.n2;
  if (c->dft_terms != 3 && c->dft_terms != 6)
    return fail(FBME_ERR_INVALID, "dft_terms must be 3 or 6");
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
  if (1LL * s0.n1 * s0.n2 * n > (1LL << 40)) return fail(FBME_ERR_INVALID, "batch too large");
  if (N > 524288 || s0.n2 > 512)
    return fail(FBME_ERR_UNSUPPORTED, "grids above 524288 points or N2 > 512 are not built");
  if (static_cast<long long>((s0.n1 + 15) / 16) * c->exchange_size > 2048)
    return fail(FBME_ERR_UNSUPPORTED, "exchange candidate count above 2048");
  out->B = n;
  out->n1 = s0.n1;
  out->n2 = s0.n2;
  out->m1 = s0.m1;
  out->m2 = s0.m2;
  return FBME_OK;
}

fbme::DevConfig dev_config(const FbmeConfig& c) {
  fbme::DevConfig d;
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
size_t dft_table_bytes(int L, int terms) { return table_bytes(L, terms); }
}  // namespace fbme

struct FbmePlan {
  fbme::BatchShape s;
  FbmeConfig cfg;
  fbme::DevConfig dc;
  fbme::DftTables tables;
  fbme::UampBuffers u;
  fbme::PolishBuffers p;
  int* status;
};

extern "C" {

const char* fbme_last_error(void) { return g_last_error.c_str(); }
const char* fbme_version(void) { return "fbme-b200 0.1.0 (sm_100a)"; }

size_t fbme_plan_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg) {
  fbme::BatchShape s;
  if (validate(shapes, n_scenes, cfg, &s) != FBME_OK) return 0;
  return make_layout(s, *cfg).total;
}

int fbme_plan_create(const FbmeShape* shapes, int32_t n_scenes, const FbmeConfig* cfg,
                     void* workspace, size_t workspace_bytes, fbme_stream_t stream,
                     FbmePlan** plan) {
  if (!plan) return fail(FBME_ERR_INVALID, "plan output pointer is NULL");
  *plan = nullptr;
  fbme::BatchShape s;
  int rc = validate(shapes, n_scenes, cfg, &s);
  if (rc != FBME_OK) return rc;
  const Layout L = make_layout(s, *cfg);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return fail(FBME_ERR_WORKSPACE, "workspace must be a 256-byte aligned device pointer");
  if (workspace_bytes < L.total)
    return fail(FBME_ERR_WORKSPACE, "workspace smaller than fbme_plan_workspace_bytes()");
  cudaError_t e = fbme::set_dft_attributes();
  if (e != cudaSuccess) return fail(FBME_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));

  FbmePlan* P = new (std::nothrow) FbmePlan();
  if (!P) return fail(FBME_ERR_INVALID, "out of host memory");
  uint8_t* w = static_cast<uint8_t*>(workspace);
  P->s = s;
  P->cfg = *cfg;
  P->dc = dev_config(*cfg);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

  const int terms = cfg->dft_terms;
  const int nt = terms == 6 ? 128 : 256, parts = terms == 6 ? 3 : 2;
  auto build_table = [&](size_t off, int Lx, int sign) {
    fbme::launch_twiddle_table(w + off, Lx, sign, nt, ceil_div(2LL * Lx, nt), ceil_div(2LL * Lx, 64),
                               parts, st);
  };
  build_table(L.tab_f2, s.n2, -1);
  build_table(L.tab_a2, s.n2, +1);
  if (s.n1 != s.n2) {
    build_table(L.tab_f1, s.n1, -1);
    build_table(L.tab_a1, s.n1, +1);
  }
  P->tables.fwd_n2 = w + L.tab_f2;
  P->tables.adj_n2 = w + L.tab_a2;
  P->tables.fwd_n1 = w + L.tab_f1;
  P->tables.adj_n1 = w + L.tab_a1;
  P->tables.kchunks_n1 = ceil_div(2LL * s.n1, 64);
  P->tables.kchunks_n2 = ceil_div(2LL * s.n2, 64);
  float2* dir1 = reinterpret_cast<float2*>(w + L.dir1);
  float2* dir2 = reinterpret_cast<float2*>(w + L.dir2);
  fbme::launch_dirichlet(dir1, s.m1, s.n1, st);
  fbme::launch_dirichlet(dir2, s.m2, s.n2, st);

  fbme::UampBuffers& u = P->u;
  u.y = nullptr;
  u.mu = reinterpret_cast<float2*>(w + L.mu);
  u.bp = reinterpret_cast<float2*>(w + L.bp);
  u.msg = reinterpret_cast<float2*>(w + L.msg);
  u.pred = reinterpret_cast<float2*>(w + L.pred);
  u.tmp = reinterpret_cast<float2*>(w + L.tmp);
  u.var = reinterpret_cast<float*>(w + L.var);
  u.gamma = reinterpret_cast<float*>(w + L.gamma);
  u.part = reinterpret_cast<double*>(w + L.part);
  u.keys = reinterpret_cast<uint32_t*>(w + L.keys);
  float* sc = reinterpret_cast<float*>(w + L.scal);
  const int B = s.B;
  u.sc = fbme::Scalars{sc, sc + B, sc + 2 * B, sc + 3 * B, sc + 4 * B,
                       sc + 5 * B, sc + 6 * B, sc + 7 * B, sc + 8 * B, sc + 9 * B};
  P->status = reinterpret_cast<int*>(w + L.status);
  u.status = P->status;

  fbme::PolishBuffers& p = P->p;
  p.y = nullptr;
  p.bp = u.bp;
  p.mu = u.mu;
  p.dir1 = dir1;
  p.dir2 = dir2;
  p.var = u.var;
  p.gamma = u.gamma;
  p.sc = u.sc;
  p.active = reinterpret_cast<int*>(w + L.active);
  p.score = reinterpret_cast<float*>(w + L.score);
  p.gamma_init = nullptr;
  p.pstate = w + L.pstate;
  p.xcand_val = reinterpret_cast<float*>(w + L.xval);
  p.xcand_idx = reinterpret_cast<int*>(w + L.xidx);
  p.keys = u.keys;
  p.cand_key = reinterpret_cast<uint32_t*>(w + L.ckey);
  p.cand_idx = reinterpret_cast<int*>(w + L.cidx);
  p.status = P->status;

  e = cudaGetLastError();
  if (e != cudaSuccess) {
    delete P;
    return fail(FBME_ERR_CUDA, std::string("plan tables: ") + cudaGetErrorString(e));
  }
  *plan = P;
  return FBME_OK;
}

size_t fbme_plan_warm_workspace_bytes(const FbmeShape* shapes, int32_t n_scenes) {
  if (!shapes || n_scenes < 1) return 0;
  if (fbme::cnn_check(n_scenes, shapes[0].n1, shapes[0].n2)) return 0;
  return fbme::cnn_workspace_bytes(n_scenes, shapes[0].n1, shapes[0].n2);
}

int fbme_plan_set_warm_start(FbmePlan* plan, const float* params, void* workspace,
                             size_t workspace_bytes) {
  if (!plan) return fail(FBME_ERR_INVALID, "plan is NULL");
  if (!params) {
    plan->u.warm_params = nullptr;
    plan->u.warm_ws = nullptr;
    return FBME_OK;
  }
  if (const char* why = fbme::cnn_check(plan->s.B, plan->s.n1, plan->s.n2))
    return fail(FBME_ERR_UNSUPPORTED, why);
  const size_t need = fbme::cnn_workspace_bytes(plan->s.B, plan->s.n1, plan->s.n2);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0 || workspace_bytes < need)
    return fail(FBME_ERR_WORKSPACE, "warm-start workspace smaller than fbme_plan_warm_workspace_bytes() "
                                    "or not 256-byte aligned");
  plan->u.warm_params = params;
  plan->u.warm_ws = workspace;
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
  if (!plan || !coefficients || !data) return fail(FBME_ERR_INVALID, "NULL argument");
  fbme::dft_forward(plan->s, plan->tables, plan->cfg.dft_terms,
                    static_cast<const float2*>(coefficients), static_cast<float2*>(data),
                    plan->u.tmp, plan->status, reinterpret_cast<cudaStream_t>(stream));
  return check_launch("dft_forward");
}

int fbme_dft_adjoint(FbmePlan* plan, const void* data, void* coefficients, fbme_stream_t stream) {
  if (!plan || !coefficients || !data) return fail(FBME_ERR_INVALID, "NULL argument");
  fbme::dft_adjoint(plan->s, plan->tables, plan->cfg.dft_terms, static_cast<const float2*>(data),
                    static_cast<float2*>(coefficients), plan->u.tmp, plan->status,
                    reinterpret_cast<cudaStream_t>(stream));
  return check_launch("dft_adjoint");
}

int fbme_uamp_run(FbmePlan* plan, const void* y, fbme_stream_t stream) {
  if (!plan || !y) return fail(FBME_ERR_INVALID, "NULL argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaMemsetAsync(plan->status, 0, plan->s.B * sizeof(int), st);
  fbme::UampBuffers u = plan->u;
  u.y = static_cast<const float2*>(y);
  fbme::uamp_run(plan->s, plan->tables, plan->dc, u, st);
  return check_launch("uamp_run");
}

int fbme_polish_run(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream) {
  if (!plan || !y || !out) return fail(FBME_ERR_INVALID, "NULL argument");
  if (!out->x || !out->posterior_variance || !out->precision || !out->noise_variance ||
      !out->effective_dof || !out->negative_log_evidence || !out->evidence_trace || !out->status)
    return fail(FBME_ERR_INVALID, "required output buffer is NULL");
  if (plan->cfg.fixed_budget_diagnostics &&
      (!out->fixed_budget_gamma_residual || !out->fixed_budget_noise_residual ||
       !out->fixed_budget_objective_decrease || !out->fixed_budget_monotone))
    return fail(FBME_ERR_INVALID, "fixed-budget diagnostics need their four output buffers");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  fbme::PolishBuffers p = plan->p;
  p.y = static_cast<const float2*>(y);
  fbme::polish_run(plan->s, plan->dc, p, *out, st);
  cudaMemcpyAsync(out->status, plan->status, plan->s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
  return check_launch("polish_run");
}

int fbme_plan_replay(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream) {
  int rc = fbme_uamp_run(plan, y, stream);
  if (rc != FBME_OK) return rc;
  return fbme_polish_run(plan, y, out, stream);
}

const char* fbme_profile_group_name(int32_t group) {
  static const char* names[FBME_NUM_GROUPS] = {
      "init", "adjoint_message", "adjoint_denoise", "forward_1", "forward_residual", "scalars",
      "sweep1_denoise", "topk", "polish", "exchange_score", "output"};
  return (group >= 0 && group < FBME_NUM_GROUPS) ? names[group] : "";
}

int fbme_plan_profile(FbmePlan* plan, const void* y, const FbmeOutputs* out, fbme_stream_t stream,
                      float* group_ms, int32_t* group_launches, int32_t n_groups) {
  if (!plan || !y || !out || !group_ms || !group_launches)
    return fail(FBME_ERR_INVALID, "NULL argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  fbme::Profiler* prof = new (std::nothrow) fbme::Profiler();
  if (!prof) return fail(FBME_ERR_INVALID, "out of host memory");
  prof->st = st;
  for (int i = 0; i < 2 * fbme::Profiler::kMax; ++i) cudaEventCreate(&prof->ev[i]);
  cudaMemsetAsync(plan->status, 0, plan->s.B * sizeof(int), st);
  fbme::UampBuffers u = plan->u;
  u.y = static_cast<const float2*>(y);
  fbme::uamp_run(plan->s, plan->tables, plan->dc, u, st, prof);
  fbme::PolishBuffers p = plan->p;
  p.y = static_cast<const float2*>(y);
  fbme::polish_run(plan->s, plan->dc, p, *out, st, prof);
  cudaMemcpyAsync(out->status, plan->status, plan->s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
  cudaError_t e = cudaStreamSynchronize(st);
  int rc = FBME_OK;
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

int fbme_plan_state(FbmePlan* plan, FbmeState* st) {
  if (!plan || !st) return fail(FBME_ERR_INVALID, "NULL argument");
  st->mean = plan->u.mu;
  st->variance = plan->u.var;
  st->prior_variance = plan->u.gamma;
  st->message = plan->u.msg;
  st->prediction = plan->u.pred;
  st->backprojection = plan->u.bp;
  st->noise_variance = plan->u.sc.noise;
  st->data_variance = plan->u.sc.dvar;
  return FBME_OK;
}

}  // extern "C"
