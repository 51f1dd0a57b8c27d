// Active-set polish of the FBME plans: top-K support from the UAMP score,
// exact reduced posterior with the Type-II evidence, evidence gate, EM
// updates of the active variances and the noise, the residual support
// exchange, fixed-budget diagnostics and the outputs.
//
// Follows torch_sbl/solver.py:1926-2021 (driver), 3961-4510
// (_uamp_active_em_polish, the branches the plans reach), 3591-3779
// (_active_posterior_with_evidence), 2898-2931 (Cholesky loading),
// 3219-3317 (deletion gain), 3408-3496 (fixed-budget residuals),
// 2081-2126 (effective DOF, support mask).
//
// Everything except the exchange scoring is K-dimensional (K <= 32): one
// warp per scene, lane i owning row i.  Fourier atoms are never
// materialised:
//   Gram      G[k][l] = D1[(n1k-n1l) mod N1] * D2[(n2k-n2l) mod N2]
//             (Dirichlet kernels summed in FP64 once per plan),
//   A_S^H y   = (A^H y)[S], a gather of the backprojection,
//   ||y - A_S mu||^2 = ||y||^2 - 2 Re(c^H mu) + mu^H G mu   (FP64),
//   A^H(y - A_S mu)[n] = (A^H y)[n] - sum_k mu_k D(n - n_k)  (exchange).
// The evidence (log-determinant + quadratic form) is accumulated in FP64.
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "topk.cuh"

namespace fbme {

constexpr float kTinyP = 1.17549435e-38f;
constexpr float kEpsP = 1.1920929e-07f;
constexpr int kMaxEval = 8;

struct PolishScene {
  int active[kMaxPolish];      // base active set (best accepted)
  int work_active[kMaxPolish]; // active set of the next evaluation
  float work_gamma[kMaxPolish];
  float work_noise;
  float2 best_mean[kMaxPolish];
  float best_pv[kMaxPolish];
  float best_dd[kMaxPolish];
  float best_gamma[kMaxPolish];
  float best_noise;
  double best_nle;
  float trace[kMaxEval];
  int evals;        // evaluations done
  int pending;      // exchange proposed at the previous transition
  int exch_acc;     // accepted exchanges
  int has_best;
};

size_t polish_state_bytes() { return sizeof(PolishScene); }

struct PolishArgs {
  BatchShape s;
  DevConfig c;
  PolishBuffers p;
};

FBME_DEV float2 dirichlet2(const float2* d1, const float2* d2, int n1, int n2, int a1, int a2,
                           int b1, int b2) {
  int i1 = a1 - b1, i2 = a2 - b2;
  if (i1 < 0) i1 += n1;
  if (i2 < 0) i2 += n2;
  return cmul(d1[i1], d2[i2]);
}

// Gram entry G[i][j] of atoms (a1, a2) and (b1, b2): the separable
// Dirichlet product for the full prefix block, or the 2-D table of an
// observation mask (global memory, L2-resident).
FBME_DEV float2 gram_at(const PolishArgs& A, const float2* d1, const float2* d2, int a1, int a2, int b1,
                        int b2) {
  if (A.p.gram2d) {
    int i1 = a1 - b1, i2 = a2 - b2;
    if (i1 < 0) i1 += A.s.n1;
    if (i2 < 0) i2 += A.s.n2;
    return __ldg(A.p.gram2d + static_cast<long long>(i1) * A.s.n2 + i2);
  }
  return dirichlet2(d1, d2, A.s.n1, A.s.n2, a1, a2, b1, b2);
}

// Copy the Dirichlet tables of a scene shape into shared memory: 8-byte
// asynchronous copies, all in flight before the one wait (a warp copying
// one element per lane at a time waited on every round trip).
FBME_DEV void load_dirichlet(const PolishArgs& A, float2* d1, float2* d2) {
  for (int i = threadIdx.x; i < A.s.n1; i += blockDim.x)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(d1 + i)), "l"(A.p.dir1 + i) : "memory");
  for (int i = threadIdx.x; i < A.s.n2; i += blockDim.x)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(d2 + i)), "l"(A.p.dir2 + i) : "memory");
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncwarp();
}

// Exact reduced posterior + negative log evidence for the work set.
// Returns in lane k: mean_k, pv_k, dd_k; nle (all lanes); status bits.
struct EvalOut {
  float2 mean;
  float pv, dd;
  double nle;
  int status;
  float dscale;  // equilibration scale sqrt(S_kk) of lane k's row
};

FBME_DEV EvalOut evaluate(const PolishArgs& A, float2 (*M)[33], float2 (*X)[33], const float2* d1,
                          const float2* d2, int K, int my_idx, float my_gamma, float nu, float2 my_c,
                          float data_energy) {
  const int lane = threadIdx.x & 31;
  const BatchShape& s = A.s;
  const bool on = lane < K;
  const int n1i = my_idx / s.n2, n2i = my_idx % s.n2;
  // One reciprocal per scale, reused by multiplication: a division here is
  // a full IEEE sequence with a slow-path branch, on the critical path of
  // a single warp.
  const float inv_nu = 1.0f / nu, inv_g = 1.0f / my_gamma;
  // system S = diag(1/gamma) + G / nu, Hermitian-symmetrised
#pragma unroll
  for (int j = 0; j < kMaxPolish; ++j) {
    const int n1j = __shfl_sync(0xffffffffu, n1i, j), n2j = __shfl_sync(0xffffffffu, n2i, j);
    if (on && j < K) {
      const float2 g = gram_at(A, d1, d2, n1i, n2i, n1j, n2j);
      float2 a = make_float2(g.x * inv_nu, g.y * inv_nu);
      if (j == lane) a.x += inv_g;
      M[lane][j] = a;
    }
  }
  __syncwarp();
  float2 row[kMaxPolish];
#pragma unroll
  for (int j = 0; j < kMaxPolish; ++j)
    if (on && j < K) {
      const float2 a = M[lane][j], b = M[j][lane];
      row[j] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
    }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < kMaxPolish; ++j)
    if (on && j < K) M[lane][j] = row[j];
  __syncwarp();
  const float dscale = on ? sqrtf(fmaxf(M[lane][lane].x, kTinyP)) : 1.0f;
  const float inv_d = 1.0f / dscale;
  // equilibrate: E[i][j] = S[i][j] / (d_i d_j), symmetrise again
  {
#pragma unroll
    for (int j = 0; j < kMaxPolish; ++j) {
      const float idj = __shfl_sync(0xffffffffu, inv_d, j);
      if (on && j < K) {
        const float2 a = M[lane][j];
        const float f = inv_d * idj;
        row[j] = make_float2(a.x * f, a.y * f);
      }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kMaxPolish; ++j)
      if (on && j < K) M[lane][j] = row[j];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kMaxPolish; ++j)
      if (on && j < K) {
        const float2 a = M[lane][j], b = M[j][lane];
        row[j] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
      }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kMaxPolish; ++j)
      if (on && j < K) M[lane][j] = row[j];
    __syncwarp();
  }
  // deterministic diagonal loading: multiplier * eps * mean|Re diag|
  float dsum = on ? fabsf(M[lane][lane].x) : 0.f;
  dsum = warp_sum(dsum);
  const float scale = fmaxf(dsum / static_cast<float>(K), kTinyP);
  const float jitter = A.c.jitter * (kEpsP * scale);
  if (on) M[lane][lane].x += jitter;
  __syncwarp();
  // Cholesky, lower, in place, right-looking: once column q is final,
  // lane i > q subtracts L[i][q] conj(L[k][q]) from its row entries k in
  // (q, i] -- independent updates instead of one dot-product chain per
  // entry.  Every entry receives its terms in the same order q = 0, 1, ...
  // as the dot-product form.
  // Each lane writes only its own row inside the loop.  Every lane computes
  // the pivot from the diagonal entry; the column entries L[k][q] reach
  // the other lanes through shared memory.  A row's diagonal takes its last
  // update before the row updates of the step, so the next pivot's entry
  // is final, and is loaded, before those updates.
  int status = 0;
  __syncwarp();
  float dnext = K > 0 ? M[0][0].x : 1.0f;
  for (int q = 0; q < K; ++q) {
    float sdiag = dnext;
    if (!(sdiag > 0.f)) {
      if (lane == q) status |= isfinite(sdiag) ? FBME_STATUS_CHOLESKY : FBME_STATUS_NONFINITE;
      sdiag = kTinyP;
    }
    const float piv = sqrtf(sdiag);
    const float rq = 1.0f / piv;
    if (lane == q) M[q][q] = make_float2(piv, 0.f);
    float2 a = make_float2(0.f, 0.f);
    if (on && lane > q) {
      const float2 v = M[lane][q];
      a = make_float2(v.x * rq, v.y * rq);
      M[lane][q] = a;
      M[lane][lane].x -= abs2(a);
    }
    // column q reaches the other lanes through shared memory (X is free
    // until the inverse factor); the row updates then go in batches of 8:
    // all loads, then the arithmetic, then the stores, so the batch's
    // shared-memory round trips overlap instead of running one by one
    X[0][lane] = a;
    __syncwarp();
    if (q + 1 < K) dnext = M[q + 1][q + 1].x;
    for (int k0 = q + 1; k0 < K; k0 += 8) {
      float2 b[8], v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (on && k0 + u < lane) {
          b[u] = X[0][k0 + u];
          v[u] = M[lane][k0 + u];
        }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (on && k0 + u < lane) {
          v[u].x -= a.x * b[u].x + a.y * b[u].y;  // a * conj(b)
          v[u].y -= a.y * b[u].x - a.x * b[u].y;
          M[lane][k0 + u] = v[u];
        }
    }
    __syncwarp();
  }
  __syncwarp();
  status = __reduce_or_sync(0xffffffffu, status);
  // mean: L z = c / nu / d, L^H w = z, mu = w / d
  const float rl = on ? 1.0f / M[lane][lane].x : 1.0f;  // 1 / L[lane][lane]
  const float2 rhs = on ? make_float2(my_c.x * inv_nu, my_c.y * inv_nu) : make_float2(0.f, 0.f);
  float2 z = make_float2(rhs.x * inv_d, rhs.y * inv_d);
  for (int q = 0; q < K; ++q) {
    if (lane == q) z = make_float2(z.x * rl, z.y * rl);
    const float2 zq = make_float2(__shfl_sync(0xffffffffu, z.x, q), __shfl_sync(0xffffffffu, z.y, q));
    if (on && lane > q) {
      const float2 l = M[lane][q];
      z.x -= l.x * zq.x - l.y * zq.y;
      z.y -= l.x * zq.y + l.y * zq.x;
    }
  }
  float2 w = z;
  for (int q = K - 1; q >= 0; --q) {
    if (lane == q) w = make_float2(w.x * rl, w.y * rl);
    const float2 wq = make_float2(__shfl_sync(0xffffffffu, w.x, q), __shfl_sync(0xffffffffu, w.y, q));
    if (on && lane < q) {
      const float2 l = M[q][lane];  // conj(L[q][lane]) * wq
      w.x -= l.x * wq.x + l.y * wq.y;
      w.y -= l.x * wq.y - l.y * wq.x;
    }
  }
  EvalOut o;
  o.dscale = dscale;
  o.mean = make_float2(w.x * inv_d, w.y * inv_d);
  // inverse factor column `lane`: X = L^{-1}, eq_var = sum_i |X[i][lane]|^2.
  // Right-looking: when X[q][lane] is final, its contribution L[i][q] X[q]
  // is added to the accumulators of every row i > q (held in X until row
  // i is final) -- the same terms in the same order as the dot-product
  // form, without its dependency chain.
  float eqv = 0.f;
  {
    const float2(*__restrict__ L)[33] = M;
    float2(*__restrict__ Xc)[33] = X;
    if (on)
      for (int i = 0; i < K; ++i) Xc[i][lane] = make_float2(0.f, 0.f);
    float2 carry = make_float2(0.f, 0.f);  // Xc[q][lane], kept from step q-1
    for (int q = 0; q < K; ++q) {
      const float rlq = __shfl_sync(0xffffffffu, rl, q);
      if (on && lane <= q) {
        float2 xq;
        if (lane == q) {
          xq = make_float2(rlq, 0.f);
        } else {
          xq = make_float2(-carry.x * rlq, -carry.y * rlq);
        }
        Xc[q][lane] = xq;
        eqv += abs2(xq);
        // batches of 8 rows: loads, arithmetic, stores (as the Cholesky)
        for (int i0 = q + 1; i0 < K; i0 += 8) {
          float2 l[8], acc[8];
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (i0 + u < K) {
              l[u] = L[i0 + u][q];
              acc[u] = Xc[i0 + u][lane];
            }
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (i0 + u < K) {
              acc[u].x += l[u].x * xq.x - l[u].y * xq.y;
              acc[u].y += l[u].x * xq.y + l[u].y * xq.x;
              Xc[i0 + u][lane] = acc[u];
            }
          if (i0 == q + 1) carry = acc[0];
        }
      }
    }
  }
  __syncwarp();
  o.pv = on ? fmaxf(eqv * (inv_d * inv_d), 0.f) : 0.f;
  o.dd = on ? fmaxf((my_gamma - o.pv) * (inv_g * inv_g), 0.f) : 0.f;
  // evidence (FP64 accumulation)
  double ld = 0.0, lg = 0.0, qd = 0.0;
  if (on) {
    ld = log(static_cast<double>(fmaxf(M[lane][lane].x, kTinyP))) + log(static_cast<double>(dscale));
    lg = log(static_cast<double>(my_gamma));
    qd = static_cast<double>(rhs.x) * o.mean.x + static_cast<double>(rhs.y) * o.mean.y;
  }
  ld = warp_sum(ld);
  lg = warp_sum(lg);
  qd = warp_sum(qd);
  const double logdet = observed_samples(s, A.c) * log(static_cast<double>(nu)) + lg + 2.0 * ld;
  double quad = static_cast<double>(data_energy) / nu - qd;
  if (quad < 0.0) quad = 0.0;
  o.nle = logdet + quad;
  if (!isfinite(o.nle)) status |= FBME_STATUS_NONFINITE;
  o.status = status;
  return o;
}

// ||y - A_S mu||^2 by the Gram identity, FP64.
FBME_DEV double residual_energy(const PolishArgs& A, const float2* d1, const float2* d2, int K,
                                int my_idx, float2 my_mu, float2 my_c, float data_energy) {
  const int lane = threadIdx.x & 31;
  const BatchShape& s = A.s;
  double cross = 0.0, quad = 0.0;
  if (lane < K) {
    cross = static_cast<double>(my_c.x) * my_mu.x + static_cast<double>(my_c.y) * my_mu.y;
    const int n1i = my_idx / s.n2, n2i = my_idx % s.n2;
    double gr = 0.0, gi = 0.0;  // (G mu)_i
    // unrolled: the shuffles and Gram entries of later j issue ahead of the
    // FP64 sums, which still run in the order j = 0, 1, ...
    const unsigned am = __activemask();
#pragma unroll 8
    for (int j = 0; j < K; ++j) {
      const int n1j = __shfl_sync(am, n1i, j), n2j = __shfl_sync(am, n2i, j);
      const float mjx = __shfl_sync(am, my_mu.x, j);
      const float mjy = __shfl_sync(am, my_mu.y, j);
      const float2 g = gram_at(A, d1, d2, n1i, n2i, n1j, n2j);
      gr += static_cast<double>(g.x) * mjx - static_cast<double>(g.y) * mjy;
      gi += static_cast<double>(g.x) * mjy + static_cast<double>(g.y) * mjx;
    }
    quad = my_mu.x * gr + my_mu.y * gi;  // Re(conj(mu_i) (G mu)_i)
  }
  cross = warp_sum(cross);
  quad = warp_sum(quad);
  double e = static_cast<double>(data_energy) - 2.0 * cross + quad;
  return e > 0.0 ? e : 0.0;
}

// Deletion gain of one active atom (solver.py:3247-3276).
FBME_DEV float deletion_gain(float2 mean, float pv, float gamma) {
  const float g = fmaxf(gamma, kTinyP);
  const float2 q = make_float2(mean.x / g, mean.y / g);
  const float down = fminf(fmaxf(pv / g, kTinyP), 1.0f);
  return -logf(down) - g * abs_sq(q) / down;
}

// Warp bitonic sort of (value desc, position asc); returns this lane's
// position after sorting.
FBME_DEV int warp_sort_desc(float val, int pos, float* out_val) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= 32; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, val, stride);
      const int op = __shfl_xor_sync(0xffffffffu, pos, stride);
      const bool other_first = (ov > val) || (ov == val && op < pos);
      const bool lower = (lane & stride) == 0;
      const bool asc = (lane & size) == 0;
      if (lower == asc ? other_first : !other_first) {
        val = ov;
        pos = op;
      }
    }
  *out_val = val;
  return pos;
}

constexpr int kPolishWarps = 1;

// Evaluations p in [state.evals, P) until done or an exchange is needed.
// phase 0: initialise from the top-K; phase 1: apply the exchange whose
// candidates are in p.xcand_*, then continue.
FBME_DEV void polish_body(const PolishArgs& A, int phase, int scene) {
  __shared__ float2 Msm[kPolishWarps][32][33];
  __shared__ float2 Xsm[kPolishWarps][32][33];
  extern __shared__ float2 dtab[];  // D1 (n1) then D2 (n2)
  const int lane = threadIdx.x & 31;
  if (scene >= A.s.B) return;
  const BatchShape& s = A.s;
  const DevConfig& c = A.c;
  const int K = c.polish_size;
  const bool on = lane < K;
  PolishScene* ps = reinterpret_cast<PolishScene*>(A.p.pstate) + scene;
  const float fl = A.p.sc.floor_[scene];
  const float data_energy = A.p.sc.data_energy[scene];
  const float Mf = static_cast<float>(observed_samples(s, c));
  const long long N = s.n();
  const float2* bp = A.p.bp + scene * N;
  float2(*M)[33] = Msm[threadIdx.x >> 5];
  float2(*X)[33] = Xsm[threadIdx.x >> 5];
  float2* d1 = dtab;
  float2* d2 = dtab + s.n1;
  load_dirichlet(A, d1, d2);
  int status = 0;

  if (phase == 0) {
    // prune + reinitialise (solver.py:4087-4106)
    if (on) {
      const int idx = A.p.active[scene * K + lane];
      ps->work_active[lane] = idx;
      const float g0 = A.p.gamma[scene * N + idx];
      ps->work_gamma[lane] = c.reinit ? fmaxf(A.p.score[scene * K + lane], fl) : g0;
    }
    if (lane == 0) {
      ps->work_noise = A.p.sc.noise[scene];
      ps->evals = 0;
      ps->pending = 0;
      ps->exch_acc = 0;
      ps->has_best = 0;
    }
    __syncwarp();
  } else {
    // residual support exchange (solver.py:4397-4494), using the best
    // state after evaluation 0 as the base.
    const int E = c.exchange;
    const float2 mu = on ? ps->best_mean[lane] : make_float2(0.f, 0.f);
    const float pv = on ? ps->best_pv[lane] : 0.f;
    const float g = on ? ps->best_gamma[lane] : 0.f;
    const float base_noise = ps->best_noise;
    const float del = on ? deletion_gain(mu, pv, g) : -INFINITY;
    float sval;
    const int spos = warp_sort_desc(on ? del : -INFINITY, on ? lane : 0x7fffffff, &sval);
    // lane r < E: removal position spos, addition candidate r
    const int rem_pos = spos;
    int repl_idx = -1;
    float repl_gamma = 0.f;
    int xmask = 0;
    if (lane < E) {
      const float add_e = A.p.xcand_val[scene * E + lane];
      const int add_i = A.p.xcand_idx[scene * E + lane];
      const float ce = Mf;
      const float ratio = add_e / fmaxf(base_noise * ce, kTinyP);
      const float add_gain = ratio > 1.0f ? ratio - 1.0f - logf(fmaxf(ratio, kTinyP)) : 0.0f;
      xmask = (add_gain + sval) > 0.0f;
      float ag = fmaxf(add_e - base_noise * ce, 0.0f) / (ce * ce);
      ag = fminf(fmaxf(ag, fl), c.max_prec);
      repl_idx = add_i;
      repl_gamma = ag;
    }
    // apply: position rem_pos takes the addition where exchanged
    for (int r = 0; r < E; ++r) {
      const int pr = __shfl_sync(0xffffffffu, rem_pos, r);
      const int xm = __shfl_sync(0xffffffffu, xmask, r);
      const int ri = __shfl_sync(0xffffffffu, repl_idx, r);
      const float rg = __shfl_sync(0xffffffffu, repl_gamma, r);
      if (xm && lane == pr) {
        ps->work_active[lane] = ri;
        ps->work_gamma[lane] = rg;
      }
    }
    const int any = __any_sync(0xffffffffu, xmask != 0);
    if (lane == 0) ps->pending = any;
    __syncwarp();
  }

  const int P = c.polish_iters;
  for (int p = ps->evals; p < P; ++p) {
    const int idx = on ? ps->work_active[lane] : 0;
    const float gam = on ? ps->work_gamma[lane] : 1.0f;
    const float nu = ps->work_noise;
    const float2 cvec = on ? bp[idx] : make_float2(0.f, 0.f);
    const EvalOut o = evaluate(A, M, X, d1, d2, K, idx, gam, nu, cvec, data_energy);
    status |= o.status;
    // evidence gate (solver.py:4168-4298)
    bool accept = true;
    if (c.gate && ps->has_best) {
      const double best = ps->best_nle;
      const double margin = static_cast<double>(c.margin_factor) * kEpsP *
                            (1.0 + fabs(o.nle) + fabs(best));
      accept = isfinite(o.nle) && (!isfinite(best) || o.nle <= best - margin);
    }
    __syncwarp();
    if (lane == 0) {
      if (c.gate && ps->has_best && ps->pending && accept) ps->exch_acc += 1;
      if (c.gate && ps->has_best) ps->pending = 0;
    }
    if (accept) {
      if (on) {
        ps->active[lane] = idx;
        ps->best_mean[lane] = o.mean;
        ps->best_pv[lane] = o.pv;
        ps->best_dd[lane] = o.dd;
        ps->best_gamma[lane] = gam;
      }
      if (lane == 0) {
        ps->best_noise = nu;
        ps->best_nle = o.nle;
        ps->has_best = 1;
      }
    }
    __syncwarp();
    if (lane == 0) {
      ps->trace[p] = static_cast<float>(ps->best_nle);
      ps->evals = p + 1;
    }
    __syncwarp();
    if (p + 1 == P) break;
    // EM between evaluations (solver.py:4320-4391), from the best state
    const int bidx = on ? ps->active[lane] : 0;
    const float2 bmu = on ? ps->best_mean[lane] : make_float2(0.f, 0.f);
    const float bpv = on ? ps->best_pv[lane] : 0.f;
    const float bg = on ? ps->best_gamma[lane] : 1.0f;
    const float bnoise = ps->best_noise;
    float ng = fminf(fmaxf(abs_sq(bmu) + bpv, fl), c.max_prec);
    const float keep = c.polish_damping;
    const float upd_g = keep * bg + (1.0f - keep) * ng;
    const float2 bc = on ? bp[bidx] : make_float2(0.f, 0.f);
    const double er = residual_energy(A, d1, d2, K, bidx, bmu, bc, data_energy);
    float dof = on ? fminf(fmaxf(1.0f - bpv / fmaxf(bg, kTinyP), 0.f), 1.f) : 0.f;
    dof = warp_sum(dof);
    float un;
    if (c.fixed_noise > 0.f) {
      un = c.fixed_noise;
    } else if (!c.noise_evidence) {
      un = static_cast<float>((er + static_cast<double>(bnoise) * dof + c.noise_rate) /
                              (static_cast<double>(Mf) + c.noise_shape));
    } else {
      un = static_cast<float>((er + c.noise_rate) /
                              fmax(static_cast<double>(Mf) - dof + c.noise_shape, kEpsP));
    }
    un = fmaxf(un, fl);
    const float new_noise = c.fixed_noise > 0.f ? un : keep * bnoise + (1.0f - keep) * un;
    if (on) {
      ps->work_active[lane] = bidx;
      ps->work_gamma[lane] = upd_g;
    }
    if (lane == 0) ps->work_noise = new_noise;
    __syncwarp();
    const int E = c.exchange;
    if (E > 0 && p == 0) break;  // exchange candidates are scored over the grid next
  }
  if (status && lane == 0) atomicOr(&A.p.status[scene], status);
}
__global__ void __launch_bounds__(32 * kPolishWarps) polish_kernel(PolishArgs A, int phase) {
  polish_body(A, phase, blockIdx.x * kPolishWarps + (threadIdx.x >> 5));
}

// Residual exchange scoring (solver.py:4398-4412) without the M-space
// residual: score[n] = |A^H y[n] - sum_k mu_k D1[n1-a_k] D2[n2-b_k]|^2 over
// the grid, active atoms excluded.  A CTA covers TY*RPT grid rows; thread
// (tx, ty) accumulates RPT rows x CPT columns, the columns in pairs
// 2tx + {0, 1} + 2*TX*c.  One paired FP32 FMA then serves two columns: with
// RE, IM the real and imaginary accumulators of the pair,
//   RE += ux*Dx;  IM += ux*Dy;  RE += uy*(-Dy);  IM += uy*Dx
// (per element the rounding sequence of a complex MAC).  D2 sits in shared
// memory split into re, im and -im, unrolled past the wrap, and twice, at
// even and at odd offset, so that the pair at any shift is one aligned
// 8-byte load with no index arithmetic.  Each CTA emits its E best
// (key, index) candidates.
template <int RPT_, int CPT, int TX_, int THREADS, int N2MAX>
struct ExTile {
  static constexpr int RPT = RPT_, TX = TX_, threads = THREADS, n2_max = N2MAX;
  static constexpr int ty = THREADS / TX;
  static constexpr int rows = ty * RPT;     // grid rows per CTA
  static constexpr int span = TX * CPT;     // columns of the thread grid
  static constexpr int pairs = CPT / 2;
  static constexpr int kpt = RPT * CPT;     // scores per thread
  static_assert(span >= N2MAX, "the thread grid spans the widest row");
  // floats per D2 table: index e + 1 <= N2 + span must be in range
  __host__ __device__ static constexpr int table_len(int n2) { return (n2 + span + 2) & ~1; }
  static size_t smem_bytes(int n2) {
    return static_cast<size_t>(rows) * n2 * sizeof(float2) + 6ull * table_len(n2) * sizeof(float);
  }
};

// Two CTAs per SM (128 registers a thread): a persistent single CTA per SM
// with double-buffered rows measured slower, its 8 warps too few to keep
// the FMA pipes fed.
template <typename T>
FBME_DEV void exchange_body(const PolishArgs& A, uint32_t* cand_key, int* cand_idx, int scene, int bx, int nbx) {
  constexpr int RPT = T::RPT, TX = T::TX;
  extern __shared__ float4 ex_shm4[];
  __shared__ TopkPrunedShared S;
  __shared__ float4 u4[kMaxPolish][T::rows];  // {ux, ux, uy, uy}
  __shared__ uint32_t excl[T::rows][16];      // active-atom bitmap per row (N2 <= 512)
  __shared__ int atom_a[kMaxPolish], atom_b[kMaxPolish];
  __shared__ float2 atom_mu[kMaxPolish];
  const BatchShape& s = A.s;
  const int r0 = bx * T::rows;
  const int K = A.c.polish_size, E = A.c.exchange;
  const int N1 = s.n1, N2 = s.n2;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  float2* bps = reinterpret_cast<float2*>(ex_shm4);  // [rows][N2]: this CTA's rows of A^H y
  float* tab = reinterpret_cast<float*>(bps + T::rows * N2);
  const int L = T::table_len(N2);
  const PolishScene* ps = reinterpret_cast<const PolishScene*>(A.p.pstate) + scene;
  {
    // A^H y rows, asynchronous copies in flight during the set-up and the
    // MAC loop: 16-byte chunks when N2 is even (every row then starts on a
    // 16-byte boundary), else one 8-byte element each
    const float2* src = A.p.bp + scene * s.n() + static_cast<long long>(r0) * N2;
    const int rows = min(T::rows, N1 - r0);
    if ((N2 & 1) == 0) {
      for (int c = threadIdx.x; c < rows * N2 / 2; c += blockDim.x)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(bps + 2 * c)), "l"(src + 2 * c)
                     : "memory");
    } else {
      for (int c = threadIdx.x; c < rows * N2; c += blockDim.x)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(bps + c)), "l"(src + c) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  // D2 tables: [parity][re, im, -im][L]; parity p holds D2[(e + p) mod N2] at
  // e.  Unrolled to the widest table, so that every thread's loads are in
  // flight together.
  constexpr int kTabIters = (T::table_len(T::n2_max) + T::threads - 1) / T::threads;
#pragma unroll
  for (int it = 0; it < kTabIters; ++it) {
    const int e = threadIdx.x + it * T::threads;
    if (e < L) {
      const int e0 = e % N2;
      const int e1 = e0 + 1 == N2 ? 0 : e0 + 1;
      const float2 v0 = __ldg(A.p.dir2 + e0), v1 = __ldg(A.p.dir2 + e1);
      tab[e] = v0.x;
      tab[L + e] = v0.y;
      tab[2 * L + e] = -v0.y;
      tab[3 * L + e] = v1.x;
      tab[4 * L + e] = v1.y;
      tab[5 * L + e] = -v1.y;
    }
  }
  for (int i = threadIdx.x; i < T::rows * 16; i += blockDim.x) (&excl[0][0])[i] = 0u;
  if (threadIdx.x < K) {
    const int idx = ps->active[threadIdx.x];
    const int a = idx / N2;
    atom_a[threadIdx.x] = a;
    atom_b[threadIdx.x] = idx - a * N2;
    atom_mu[threadIdx.x] = ps->best_mean[threadIdx.x];
  }
  __syncthreads();
  if (threadIdx.x < K) {
    const int ra = atom_a[threadIdx.x] - r0, b = atom_b[threadIdx.x];
    if (ra >= 0 && ra < T::rows) atomicOr(&excl[ra][b >> 5], 1u << (b & 31));
  }
  constexpr int kUIters = (kMaxPolish * T::rows + T::threads - 1) / T::threads;
#pragma unroll
  for (int it = 0; it < kUIters; ++it) {
    const int i = threadIdx.x + it * T::threads;
    const int k = i / T::rows, ri = i % T::rows;
    if (k < K) {
      float2 uv = make_float2(0.f, 0.f);
      if (r0 + ri < N1) {
        int dd = r0 + ri - atom_a[k];
        dd += dd < 0 ? N1 : 0;
        uv = cmul(atom_mu[k], __ldg(A.p.dir1 + dd));
      }
      u4[k][ri] = make_float4(uv.x, uv.x, uv.y, uv.y);
    }
  }
  __syncthreads();
  float2 re[RPT][T::pairs], im[RPT][T::pairs];
#pragma unroll
  for (int r = 0; r < RPT; ++r)
#pragma unroll
    for (int c = 0; c < T::pairs; ++c) {
      re[r][c] = make_float2(0.f, 0.f);
      im[r][c] = make_float2(0.f, 0.f);
    }
#pragma unroll 1
  for (int k = 0; k < K; ++k) {
    // pair (D2[e], D2[e+1]) at e = n2 - b + N2 >= 1; e's parity is the warp's
    const int e0 = 2 * tx - atom_b[k] + N2;
    const int odd = e0 & 1;
    const float* base = tab + odd * 3 * L + (e0 - odd);
    float2 dx[T::pairs], dy[T::pairs], ny[T::pairs];
#pragma unroll
    for (int c = 0; c < T::pairs; ++c) {
      dx[c] = *reinterpret_cast<const float2*>(base + 2 * TX * c);
      dy[c] = *reinterpret_cast<const float2*>(base + L + 2 * TX * c);
      ny[c] = *reinterpret_cast<const float2*>(base + 2 * L + 2 * TX * c);
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const float4 uu = u4[k][ty * RPT + r];
      const float2 ux = make_float2(uu.x, uu.y), uy = make_float2(uu.z, uu.w);
#pragma unroll
      for (int c = 0; c < T::pairs; ++c) {
        re[r][c] = __ffma2_rn(ux, dx[c], re[r][c]);
        im[r][c] = __ffma2_rn(ux, dy[c], im[r][c]);
        re[r][c] = __ffma2_rn(uy, ny[c], re[r][c]);
        im[r][c] = __ffma2_rn(uy, dx[c], im[r][c]);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  uint32_t key[T::kpt];
  uint32_t valid = 0u;
#pragma unroll
  for (int r = 0; r < RPT; ++r)
#pragma unroll
    for (int c = 0; c < T::pairs; ++c)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int i = (r * T::pairs + c) * 2 + j;
        const int lr = ty * RPT + r;
        const int n2 = 2 * tx + 2 * TX * c + j;
        key[i] = 0u;
        if (r0 + lr < N1 && n2 < N2) {
          valid |= 1u << i;
          const float2 bv = bps[lr * N2 + n2];
          const float2 acc = j ? make_float2(re[r][c].y, im[r][c].y) : make_float2(re[r][c].x, im[r][c].x);
          const float2 d = make_float2(bv.x - acc.x, bv.y - acc.y);
          const bool act = (excl[lr][n2 >> 5] >> (n2 & 31)) & 1u;
          key[i] = act ? 0u : float_key_t(abs_sq(d));
        }
      }
  const size_t off = (static_cast<size_t>(scene) * nbx + bx) * E;
  auto gidx = [&](int i) {
    const int r = i / (2 * T::pairs), c = (i / 2) % T::pairs, j = i & 1;
    return (r0 + ty * RPT + r) * N2 + 2 * tx + 2 * TX * c + j;
  };
  // residual scores of one CTA crowd into few top-byte bins (radix fallback)
  block_topk_pruned<T::kpt, true>(key, valid, gidx, E, S, cand_key + off, cand_idx + off);
}

template <typename T>
__global__ void __launch_bounds__(T::threads, 2)
exchange_kernel(PolishArgs A, uint32_t* cand_key, int* cand_idx) {
  exchange_body<T>(A, cand_key, cand_idx, blockIdx.y, blockIdx.x, gridDim.x);
}

using ExSmall = ExTile<8, 2, 32, 256, 64>;
using ExMid = ExTile<8, 2, 64, 256, 128>;
using ExWide = ExTile<8, 4, 64, 256, 256>;
using ExWidest = ExTile<4, 8, 64, 256, 512>;

// Final K-space outputs, fixed-budget diagnostics, effective DOF
// (solver.py:1989-2021, 2081-2092, 3408-3496, 2108-2126).
FBME_DEV void polish_finish_body(const PolishArgs& A, const FbmeOutputs& out, int scene) {
  extern __shared__ float2 dtab[];
  const int lane = threadIdx.x & 31;
  if (scene >= A.s.B) return;
  const BatchShape& s = A.s;
  const DevConfig& c = A.c;
  const int K = c.polish_size, P = c.polish_iters;
  const int R = c.repairs;
  const bool on = lane < K;
  const PolishScene* ps = reinterpret_cast<const PolishScene*>(A.p.pstate) + scene;
  const float fl = A.p.sc.floor_[scene];
  const float Mf = static_cast<float>(observed_samples(s, c));
  const long long N = s.n();
  float2* d1 = dtab;
  float2* d2 = dtab + s.n1;
  load_dirichlet(A, d1, d2);
  const int idx = on ? ps->active[lane] : 0;
  const float2 mu = on ? ps->best_mean[lane] : make_float2(0.f, 0.f);
  const float pv = on ? ps->best_pv[lane] : 0.f;
  const float dd = on ? ps->best_dd[lane] : 0.f;
  const float g = on ? ps->best_gamma[lane] : 1.0f;
  const float nu = ps->best_noise;
  // effective DOF with relevance projection
  float rel = on ? fminf(fmaxf(g * dd, 0.f), 1.f) : 0.f;
  const float raw = warp_sum(rel);
  const float max_dof = static_cast<float>(observed_samples(s, c) * (1.0 - 10.0 * kEpsP));
  const float sc = fminf(1.0f, max_dof / fmaxf(raw, kEpsP));
  const float dof = warp_sum(rel * sc);
  if (lane == 0) {
    out.noise_variance[scene] = nu;
    out.effective_dof[scene] = dof;
    out.negative_log_evidence[scene] = static_cast<float>(ps->best_nle);
    for (int p = 0; p < P; ++p) out.evidence_trace[scene * (P + R) + p] = ps->trace[p];
    if (out.support_exchanges_accepted) out.support_exchanges_accepted[scene] = ps->exch_acc;
    // the support repairs append their evidence after the polish's
    for (int r = 0; r < R; ++r) out.evidence_trace[scene * (P + R) + P + r] = ps->trace[P + r];
    if (out.support_score_threshold && c.false_alarm > 0.f)
      out.support_score_threshold[scene] =
          static_cast<float>(log(static_cast<double>(N) / static_cast<double>(c.false_alarm)));
  }
  if (on && out.active_indices) out.active_indices[scene * K + lane] = idx;
  if (c.fixed_budget && out.fixed_budget_gamma_residual) {
    const float ag = fmaxf(g, kTinyP);
    const float gt = fminf(fmaxf(abs_sq(mu) + pv, fl), c.max_prec);
    const float gs = fmaxf(fmaxf(fabsf(ag), fabsf(gt)), kTinyP);
    const float gr = warp_max(on ? fabsf(ag - gt) / gs : 0.f);
    float dofd = on ? fminf(fmaxf(1.0f - pv / ag, 0.f), 1.f) : 0.f;
    dofd = warp_sum(dofd);
    const float2 cv = on ? A.p.bp[scene * N + idx] : make_float2(0.f, 0.f);
    const double er = residual_energy(A, d1, d2, K, idx, mu, cv, A.p.sc.data_energy[scene]);
    float nt;
    if (c.fixed_noise > 0.f) {
      nt = nu;
    } else if (!c.noise_evidence) {
      nt = static_cast<float>((er + static_cast<double>(nu) * dofd + c.noise_rate) /
                              (static_cast<double>(Mf) + c.noise_shape));
    } else {
      nt = static_cast<float>((er + c.noise_rate) /
                              fmax(static_cast<double>(Mf) - dofd + c.noise_shape, kEpsP));
    }
    nt = fminf(fmaxf(nt, fl), c.max_prec);
    const float ns = fmaxf(fmaxf(fabsf(nu), fabsf(nt)), kTinyP);
    if (lane == 0) {
      out.fixed_budget_gamma_residual[scene] = gr;
      out.fixed_budget_noise_residual[scene] = c.fixed_noise > 0.f ? 0.f : fabsf(nu - nt) / ns;
      bool fin = true, mono = true;
      for (int p = 0; p < P; ++p) fin &= isfinite(ps->trace[p]) != 0;
      for (int p = 1; p < P; ++p) mono &= ps->trace[p] <= ps->trace[p - 1];
      out.fixed_budget_monotone[scene] = fin && mono;
      out.fixed_budget_objective_decrease[scene] = fmaxf(ps->trace[0] - ps->trace[P - 1], 0.f);
    }
  }
}
__global__ void __launch_bounds__(32) polish_finish_kernel(PolishArgs A, FbmeOutputs out) {
  polish_finish_body(A, out, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Global certificate and support repairs (solver.py:3522-3588 inactive
// certificate, 3219-3317 active certificate, 4511-4628 repairs, 4851-4870
// and 5388-5460 final diagnostics).  One CTA per scene: warp 0 runs the
// K-dimensional algebra (evaluate(), as in the polish), every thread scores
// grid atoms.  For atom j, with g_i = a_j^H a_i from the Dirichlet tables,
//   q_j   = (A^H y)[j] - sum_i g_i mu_i             (nu a_j^H C^-1 y)
//   v     = L^-1 D^-1 conj(g)                       (forward substitution)
//   s_j   = M / nu - ||v||^2 / nu^2                 (a_j^H C^-1 a_j)
//   rho_j = |q_j / nu|^2 / s_j, and 0 on the active set,
// where L is the Cholesky factor of the equilibrated reduced system
// D^-1 (Gamma^-1 + A_S^H A_S / nu) D^-1: the reference obtains the same
// quantities from K adjoint transforms of the active columns and a
// K-right-hand-side triangular solve over the grid.
constexpr int kCertThreads = 256;

struct CertBest {
  float ratio, prec;
  int index;
};

FBME_DEV void cert_pick(CertBest& b, float ratio, float prec, int index) {
  if (ratio > b.ratio || (ratio == b.ratio && index < b.index)) b = CertBest{ratio, prec, index};
}

FBME_DEV CertBest cert_warp_best(CertBest b) {
  for (int off = 16; off > 0; off >>= 1) {
    const float r = __shfl_xor_sync(0xffffffffu, b.ratio, off);
    const float p = __shfl_xor_sync(0xffffffffu, b.prec, off);
    const int i = __shfl_xor_sync(0xffffffffu, b.index, off);
    cert_pick(b, r, p, i);
  }
  return b;
}

// The active set of one evaluation, staged for the grid scan.
struct CertModel {
  int a1[kMaxPolish], a2[kMaxPolish], idx[kMaxPolish];
  float2 mu[kMaxPolish];
  float inv_d[kMaxPolish], inv_l[kMaxPolish];
};

// Largest one-coordinate ratio over the atoms [j0, j1) of the grid (first
// index on ties, as torch's max), with its atom precision s_j; the block's
// best, in every thread.
FBME_DEV CertBest cert_scan(const PolishArgs& A, const float2 (*L)[34], const CertModel& m, int K, float nu,
                            const float2* bp, const float2* d1, const float2* d2, long long j0, long long j1,
                            CertBest* red) {
  const BatchShape& s = A.s;
  const float Mf = static_cast<float>(observed_samples(s, A.c));
  const float nu2 = nu * nu;
  CertBest b{-1.f, 1.f, 0x7fffffff};
  for (long long j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const int j1i = static_cast<int>(j / s.n2);
    const int j2i = static_cast<int>(j - static_cast<long long>(j1i) * s.n2);
    float2 q = __ldg(bp + j);
    bool act = false;
    float2 v[kMaxPolish];
    float red2 = 0.f;
#pragma unroll
    for (int i = 0; i < kMaxPolish; ++i) {
      if (i < K) {
        act |= m.idx[i] == j;
        const float2 g = gram_at(A, d1, d2, j1i, j2i, m.a1[i], m.a2[i]);
        const float2 mu = m.mu[i];
        q.x -= g.x * mu.x - g.y * mu.y;
        q.y -= g.x * mu.y + g.y * mu.x;
        float2 c = make_float2(g.x * m.inv_d[i], -g.y * m.inv_d[i]);
        // Row i of L in 16-byte pairs (rows start 16-byte aligned), same
        // order of the multiply-adds as one entry at a time.
#pragma unroll
        for (int k = 0; k + 1 < i; k += 2) {
          const float4 l2 = *reinterpret_cast<const float4*>(&L[i][k]);
          c.x -= l2.x * v[k].x - l2.y * v[k].y;
          c.y -= l2.x * v[k].y + l2.y * v[k].x;
          c.x -= l2.z * v[k + 1].x - l2.w * v[k + 1].y;
          c.y -= l2.z * v[k + 1].y + l2.w * v[k + 1].x;
        }
        if (i & 1) {
          const float2 l = L[i][i - 1];
          c.x -= l.x * v[i - 1].x - l.y * v[i - 1].y;
          c.y -= l.x * v[i - 1].y + l.y * v[i - 1].x;
        }
        v[i] = make_float2(c.x * m.inv_l[i], c.y * m.inv_l[i]);
        red2 += abs_sq(v[i]);
      }
    }
    const float prec = fmaxf(Mf / nu - red2 / nu2, kTinyP);
    const float2 qn = make_float2(q.x / nu, q.y / nu);
    cert_pick(b, act ? 0.f : abs_sq(qn) / prec, prec, static_cast<int>(j));
  }
  b = cert_warp_best(b);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = b;
  __syncthreads();
  if (w == 0) {
    b = lane < static_cast<int>(blockDim.x >> 5) ? red[lane] : CertBest{-1.f, 1.f, 0x7fffffff};
    b = cert_warp_best(b);
    __syncwarp();
    if (lane == 0) red[0] = b;
  }
  __syncthreads();
  b = red[0];
  __syncthreads();
  return b;
}

// Inactive certificate of the best atom (solver.py:3568-3588).
struct CertState {
  float ratio, gain, optvar;
  int index;
};

FBME_DEV CertState cert_state(const CertBest& b) {
  const bool up = b.ratio > 1.0f;
  return CertState{b.ratio, up ? b.ratio - 1.0f - logf(fmaxf(b.ratio, kTinyP)) : 0.f,
                   up ? (b.ratio - 1.0f) / b.prec : 0.f, b.index};
}

// Lane k's exact one-coordinate terms (solver.py:3244-3290): the current
// deletion delta, the gain of the optimal variance and that variance.
struct ActiveTerms {
  float current, gain, optvar;
};

FBME_DEV ActiveTerms active_terms(float2 mean, float pv, float gamma) {
  const float g = fmaxf(gamma, kTinyP);
  const float2 q = make_float2(mean.x / g, mean.y / g);
  const float sc = fmaxf((g - pv) / (g * g), kTinyP);
  const float down = fminf(fmaxf(pv / g, kTinyP), 1.0f);
  const float loo = fmaxf(sc / down, kTinyP);
  const float ratio = abs_sq(q) / fmaxf(sc * down, kTinyP);
  ActiveTerms t;
  t.optvar = ratio > 1.0f ? (ratio - 1.0f) / loo : 0.f;
  t.current = -logf(down) - g * abs_sq(q) / down;
  const float opt = ratio > 1.0f ? logf(fmaxf(ratio, kTinyP)) - ratio + 1.0f : 0.f;
  t.gain = fmaxf(t.current - opt, 0.f);
  return t;
}

// Warp argmax of (value, lane), the first lane on ties.
FBME_DEV int warp_argmax(float v, float* best) {
  int pos = threadIdx.x & 31;
  for (int off = 16; off > 0; off >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int op = __shfl_xor_sync(0xffffffffu, pos, off);
    if (ov > v || (ov == v && op < pos)) {
      v = ov;
      pos = op;
    }
  }
  *best = v;
  return pos;
}

// Per-scene scratch of the certificate steps (caller workspace): the
// factor and staged active set of the model whose certificate the next
// scan computes, the pending repair, the current inactive certificate and
// the scan's per-block partial results.
struct CertScratch {
  float2 L[kMaxPolish][kMaxPolish];
  CertModel m;
  int nu_bits;  // the model's noise variance
  int pending;  // the scanned model is a repair proposal
  int p_idx[kMaxPolish];
  float p_gam[kMaxPolish];
  float2 p_mean[kMaxPolish];
  float p_pv[kMaxPolish], p_dd[kMaxPolish];
  double p_nle;
  CertState cur;
};

// Scan blocks per scene: enough CTAs to cover the SMs a few times, at least
// 1024 atoms per block, at most kCertMaxBlocks.  Within that range the
// count is raised (up to 4x) until the B * nblk CTAs fill their last wave of
// `resident` CTAs per SM to 97 %, or to the best fill seen: a last wave that
// is mostly empty leaves the scan's slowest blocks running alone.  The
// result does not depend on the count (first index on ties).
constexpr int kCertMaxBlocks = 256;
int cert_blocks(const BatchShape& s, int resident) {
  static const int sms = [] {
    int dev = 0, v = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
  }();
  const long long most = std::min(std::max(1LL, (s.n() + 1023) / 1024), static_cast<long long>(kCertMaxBlocks));
  const long long lo = std::max(1LL, std::min((4LL * sms + s.B - 1) / s.B, most));
  const long long slots = static_cast<long long>(sms) * std::max(1, resident);
  long long best = lo;
  double best_fill = 0.0;
  for (long long n = lo; n <= std::min(most, 4 * lo); ++n) {
    const long long ctas = n * s.B;
    const double fill = static_cast<double>(ctas) / static_cast<double>(((ctas + slots - 1) / slots) * slots);
    if (fill > best_fill + 1e-9) {
      best_fill = fill;
      best = n;
    }
    if (fill >= 0.97) break;
  }
  return static_cast<int>(best);
}

size_t cert_scratch_bytes(const BatchShape& s) {
  return static_cast<size_t>(s.B) * (sizeof(CertScratch) + sizeof(CertBest) * kCertMaxBlocks);
}

FBME_DEV CertScratch* cert_scene(void* ws, int scene) {
  return reinterpret_cast<CertScratch*>(ws) + scene;
}
FBME_DEV CertBest* cert_parts(void* ws, int B, int scene) {
  return reinterpret_cast<CertBest*>(reinterpret_cast<CertScratch*>(ws) + B) + static_cast<long long>(scene) *
         kCertMaxBlocks;
}

// Warp 0 of a step: evaluate the work set (idx, gam) and stage its factor
// and active set for the scan.
FBME_DEV EvalOut cert_model(const PolishArgs& A, CertScratch* cs, float2 (*M)[33], float2 (*X)[33],
                            const float2* d1, const float2* d2, int idx, float gam, float nu, const float2* bp,
                            float data_energy) {
  const int lane = threadIdx.x & 31;
  const int K = A.c.polish_size;
  const bool on = lane < K;
  const EvalOut o = evaluate(A, M, X, d1, d2, K, idx, gam, nu, on ? bp[idx] : make_float2(0.f, 0.f), data_energy);
  if (on) {
    for (int k = 0; k < lane; ++k) cs->L[lane][k] = M[lane][k];
    cs->m.idx[lane] = idx;
    cs->m.a1[lane] = idx / A.s.n2;
    cs->m.a2[lane] = idx % A.s.n2;
    cs->m.mu[lane] = o.mean;
    cs->m.inv_d[lane] = 1.0f / o.dscale;
    cs->m.inv_l[lane] = 1.0f / M[lane][lane].x;
  }
  if (lane == 0) cs->nu_bits = __float_as_int(nu);
  return o;
}

// The scan's result: the block partials merged (first index on ties).
FBME_DEV CertBest cert_merge(void* ws, int B, int scene, int nblk) {
  const int lane = threadIdx.x & 31;
  const CertBest* part = cert_parts(ws, B, scene);
  CertBest b{-1.f, 1.f, 0x7fffffff};
  for (int i = lane; i < nblk; i += 32) cert_pick(b, part[i].ratio, part[i].prec, part[i].index);
  return cert_warp_best(b);
}

// One certificate step of one scene (one warp).  Step 0 stages the model
// the polish kept.  Step t in [1, R] merges the previous scan (the kept
// model's certificate at t = 1; otherwise repair t-1's certificate and its
// decision: kept when the inactive ratio that proposed it exceeds 1 and
// the exact evidence does not rise) and stages repair t: the best inactive
// atom replaces the active atom of largest deletion delta, with variance
// max(optimal, floor).  Step R + 1 merges the last scan and writes the
// final certificate (solver.py:4851-4870, 5388-5460).
__global__ void __launch_bounds__(32) cert_step_kernel(PolishArgs A, FbmeCertificate C, void* ws, int nblk,
                                                       int t) {
  __shared__ float2 M[32][33];
  __shared__ float2 X[32][33];
  extern __shared__ float2 dtab[];
  const int scene = blockIdx.x;
  if (scene >= A.s.B) return;
  const BatchShape& s = A.s;
  const DevConfig& c = A.c;
  const int K = c.polish_size, P = c.polish_iters, R = c.repairs;
  const int lane = threadIdx.x & 31;
  const bool on = lane < K;
  PolishScene* ps = reinterpret_cast<PolishScene*>(A.p.pstate) + scene;
  CertScratch* cs = cert_scene(ws, scene);
  const long long N = s.n();
  const float2* bp = A.p.bp + scene * N;
  const float fl = A.p.sc.floor_[scene];
  const float data_energy = A.p.sc.data_energy[scene];
  const float nu = ps->best_noise;
  int status = 0;
  if (t > 0) {
    const CertState next = cert_state(cert_merge(ws, s.B, scene, nblk));
    bool keep = true;
    if (cs->pending) {  // decide the repair the scan certified
      const CertState prop = cs->cur;
      const double nle = cs->p_nle;
      keep = prop.ratio > 1.0f && isfinite(nle) && static_cast<float>(nle) <= static_cast<float>(ps->best_nle);
      __syncwarp();
      if (keep) {
        if (on) {
          ps->active[lane] = cs->p_idx[lane];
          ps->best_mean[lane] = cs->p_mean[lane];
          ps->best_pv[lane] = cs->p_pv[lane];
          ps->best_dd[lane] = cs->p_dd[lane];
          ps->best_gamma[lane] = cs->p_gam[lane];
        }
        if (lane == 0) {
          ps->best_nle = nle;
          ps->exch_acc += 1;
        }
      }
      __syncwarp();
      if (lane == 0) ps->trace[P + t - 2] = static_cast<float>(ps->best_nle);
    }
    __syncwarp();
    if (lane == 0 && keep) cs->cur = next;
    __syncwarp();
  }
  if (t <= R) {
    float2* d1 = dtab;
    float2* d2 = dtab + s.n1;
    load_dirichlet(A, d1, d2);
    int idx = on ? ps->active[lane] : 0;
    float gam = on ? ps->best_gamma[lane] : 1.0f;
    if (t > 0) {
      const float2 mu = on ? ps->best_mean[lane] : make_float2(0.f, 0.f);
      const float pv = on ? ps->best_pv[lane] : 0.f;
      float dmax;
      const int pos = warp_argmax(on ? deletion_gain(mu, pv, gam) : -INFINITY, &dmax);
      const CertState cur = cs->cur;
      if (lane == pos) {
        idx = cur.index;
        gam = fmaxf(cur.optvar, fl);
      }
    }
    const EvalOut o = cert_model(A, cs, M, X, d1, d2, idx, gam, nu, bp, data_energy);
    status |= o.status;
    if (on) {
      cs->p_idx[lane] = idx;
      cs->p_gam[lane] = gam;
      cs->p_mean[lane] = o.mean;
      cs->p_pv[lane] = o.pv;
      cs->p_dd[lane] = o.dd;
    }
    if (lane == 0) {
      cs->p_nle = o.nle;
      cs->pending = t > 0;
    }
  } else {
    // final certificate of the kept model
    const float2 mu = on ? ps->best_mean[lane] : make_float2(0.f, 0.f);
    const float pv = on ? ps->best_pv[lane] : 0.f;
    const float g = on ? ps->best_gamma[lane] : 1.0f;
    const int idx = on ? ps->active[lane] : 0;
    const ActiveTerms at = active_terms(mu, pv, g);
    float max_gain, max_nondel, max_del;
    const int gp = warp_argmax(on ? at.gain : -INFINITY, &max_gain);
    warp_argmax(on ? (at.optvar > 0.f ? at.gain : 0.f) : -INFINITY, &max_nondel);
    warp_argmax(on ? at.current : -INFINITY, &max_del);
    const int best_idx = __shfl_sync(0xffffffffu, idx, gp);
    const float best_var = __shfl_sync(0xffffffffu, at.optvar, gp);
    if (lane == 0) {
      const CertState cur = cs->cur;
      const float tol = C.coordinate_tolerance;
      const float pen = fmaxf(max_nondel, fmaxf(max_del, 0.f));
      C.inactive_max_evidence_ratio[scene] = cur.ratio;
      C.inactive_best_index[scene] = cur.index;
      C.inactive_evidence_gain[scene] = cur.gain;
      C.inactive_optimal_variance[scene] = cur.optvar;
      C.support_repairs_accepted[scene] = ps->exch_acc;
      C.active_max_evidence_gain[scene] = max_gain;
      C.active_best_index[scene] = best_idx;
      C.active_optimal_variance[scene] = best_var;
      C.active_max_deletion_gain[scene] = max_del;
      C.active_penalized_evidence_gain[scene] = pen;
      C.coordinate_stationary[scene] = cur.gain <= tol && max_gain <= tol;
      C.type2_map_coordinate_stationary[scene] = fmaxf(cur.gain, 0.f) <= tol && pen <= tol;
      if (C.familywise_ratio_threshold > 0.f)
        C.familywise_no_discovery[scene] = cur.ratio <= C.familywise_ratio_threshold;
    }
  }
  status = __reduce_or_sync(0xffffffffu, status);
  if (status && lane == 0) atomicOr(&A.p.status[scene], status);
}

// Block (bx, scene) scores atoms [bx chunk, (bx + 1) chunk) against the
// staged model and writes its best to the scene's partials.
__global__ void __launch_bounds__(kCertThreads, 3) cert_scan_kernel(PolishArgs A, void* ws) {
  __shared__ __align__(16) float2 M[32][34];
  __shared__ CertModel model;
  __shared__ CertBest red[kCertThreads / 32];
  extern __shared__ float2 dtab[];
  const int scene = blockIdx.y;
  if (scene >= A.s.B) return;
  const BatchShape& s = A.s;
  const int K = A.c.polish_size;
  const CertScratch* cs = cert_scene(ws, scene);
  float2* d1 = dtab;
  float2* d2 = dtab + s.n1;
  load_dirichlet(A, d1, d2);
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) {
    const int i = e / K, k = e - i * K;
    if (k < i) M[i][k] = cs->L[i][k];
  }
  if (threadIdx.x < K) {
    const int i = threadIdx.x;
    model.idx[i] = cs->m.idx[i];
    model.a1[i] = cs->m.a1[i];
    model.a2[i] = cs->m.a2[i];
    model.mu[i] = cs->m.mu[i];
    model.inv_d[i] = cs->m.inv_d[i];
    model.inv_l[i] = cs->m.inv_l[i];
  }
  __syncthreads();
  const float nu = __int_as_float(cs->nu_bits);
  const long long N = s.n();
  const long long chunk = (N + gridDim.x - 1) / gridDim.x;
  const long long j0 = blockIdx.x * chunk, j1 = min(N, j0 + chunk);
  const CertBest b = cert_scan(A, M, model, K, nu, A.p.bp + scene * N, d1, d2, j0, j1, red);
  if (threadIdx.x == 0) cert_parts(ws, s.B, scene)[blockIdx.x] = b;
}

// N-space outputs in one pass: zero mean, floor variance and 1/floor
// precision off the active set, and the active entries.  Block b of a scene
// owns the contiguous pixel range [e0, e1): it fills the range, then its
// threads k < K write active atom k where it falls inside the range, so no
// other block touches those pixels and one launch replaces fill + scatter.
FBME_DEV void output_body(const PolishArgs& A, const FbmeOutputs& out, int scene, int bx, int nbx) {
  const BatchShape& s = A.s;
  const long long N = s.n();
  const int K = A.c.polish_size;
  const float fl = A.p.sc.floor_[scene];
  const float inv = 1.0f / fl;
  const long long chunk = (N + nbx - 1) / nbx;
  const long long e0 = bx * chunk, e1 = min(N, e0 + chunk);
  float2* x = reinterpret_cast<float2*>(out.x) + scene * N;
  float* pv = out.posterior_variance + scene * N;
  float* pr = out.precision + scene * N;
  uint8_t* mk = out.support_mask ? out.support_mask + scene * N : nullptr;
  for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    x[e] = make_float2(0.f, 0.f);
    pv[e] = fl;
    pr[e] = inv;
    if (mk) mk[e] = 0;
  }
  __syncthreads();
  const int k = threadIdx.x;
  if (k >= K) return;
  const PolishScene* ps = reinterpret_cast<const PolishScene*>(A.p.pstate) + scene;
  const int idx = ps->active[k];
  const float2 mu = ps->best_mean[k];
  if (bx == 0 && out.active_values) reinterpret_cast<float2*>(out.active_values)[scene * K + k] = mu;
  if (idx < e0 || idx >= e1) return;
  const float apv = ps->best_pv[k];
  x[idx] = mu;
  pv[idx] = apv;
  pr[idx] = 1.0f / ps->best_gamma[k];
  if (mk && A.c.false_alarm > 0.f) {
    const float thr = static_cast<float>(log(static_cast<double>(N) / A.c.false_alarm));
    mk[idx] = (abs_sq(mu) / fmaxf(apv, kTinyP)) > thr;
  }
}
__global__ void __launch_bounds__(256) output_kernel(PolishArgs A, FbmeOutputs out) {
  output_body(A, out, blockIdx.y, blockIdx.x, gridDim.x);
}

void launch_topk_blocks(const uint32_t* keys, long long n, int k, int B, uint32_t* cand_key, int* cand_idx,
                        cudaStream_t st);
void launch_topk_merge(const uint32_t* cand_key, const int* cand_idx, int ncand, int k, int B,
                       int* out_idx, float* out_val, cudaStream_t st);

// The polish steps of several shape buckets (an uneven plan's), one launch
// each: bucket i is blockIdx.z = i with its own arguments; blocks past its
// scenes or blocks return, and every scene runs the single-bucket code.
struct PolishSet {
  int n;
  PolishArgs a[kBucketSetMax];
  FbmeOutputs out[kBucketSetMax];
  int ex_blocks[kBucketSetMax];   // exchange row blocks per scene
  int out_blocks[kBucketSetMax];  // output blocks per scene
};
static_assert(sizeof(PolishSet) <= 32764, "kernel parameter limit");

FBME_DEV bool has_exchange(const DevConfig& c) { return c.exchange > 0 && c.polish_iters > 1; }

__global__ void __launch_bounds__(32 * kPolishWarps) polish_set_kernel(const PolishSet S, int phase) {
  const PolishArgs& A = S.a[blockIdx.z];
  if (phase == 1 && !has_exchange(A.c)) return;
  polish_body(A, phase, blockIdx.x * kPolishWarps + (threadIdx.x >> 5));
}

template <typename T>
__global__ void __launch_bounds__(T::threads, 2) exchange_set_kernel(const PolishSet S) {
  const PolishArgs& A = S.a[blockIdx.z];
  const int nbx = S.ex_blocks[blockIdx.z];
  if (static_cast<int>(blockIdx.x) >= nbx || static_cast<int>(blockIdx.y) >= A.s.B) return;
  exchange_body<T>(A, A.p.cand_key, A.p.cand_idx, blockIdx.y, blockIdx.x, nbx);
}

__global__ void __launch_bounds__(32) polish_finish_set_kernel(const PolishSet S) {
  polish_finish_body(S.a[blockIdx.z], S.out[blockIdx.z], blockIdx.x);
}

__global__ void __launch_bounds__(256) output_set_kernel(const PolishSet S) {
  const int nbx = S.out_blocks[blockIdx.z];
  if (static_cast<int>(blockIdx.x) >= nbx || static_cast<int>(blockIdx.y) >= S.a[blockIdx.z].s.B) return;
  output_body(S.a[blockIdx.z], S.out[blockIdx.z], blockIdx.y, blockIdx.x, nbx);
}

static int exchange_rows(int n2) {
  return n2 <= 64 ? ExSmall::rows : n2 <= 128 ? ExMid::rows : n2 <= 256 ? ExWide::rows : ExWidest::rows;
}

int exchange_blocks(const BatchShape& s) {
  const int rows = exchange_rows(s.n2);
  return (s.n1 + rows - 1) / rows;
}

template <typename T>
static cudaError_t set_exchange_smem() {
  cudaError_t e = cudaFuncSetAttribute(exchange_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(T::smem_bytes(T::n2_max)));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(exchange_set_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(T::smem_bytes(T::n2_max)));
  return e;
}

cudaError_t set_polish_attributes() {
  cudaError_t e = set_exchange_smem<ExSmall>();
  if (e == cudaSuccess) e = set_exchange_smem<ExMid>();
  if (e == cudaSuccess) e = set_exchange_smem<ExWide>();
  if (e == cudaSuccess) e = set_exchange_smem<ExWidest>();
  return e;
}

// Residual exchange scoring under an observation mask (solver.py:4398-4412
// with the masked operator): score[n] = |A^H y[n] - sum_k mu_k G(n - a_k)|^2
// with the mask's 2-D Gram table G, written as order-preserving keys for a
// top-E selection; active atoms get key 0 (the reference's -inf).  One
// thread per grid point; the table lookups hit L2.
__global__ void __launch_bounds__(256) exchange_masked_kernel(PolishArgs A) {
  __shared__ int atom1[kMaxPolish], atom2[kMaxPolish], atom[kMaxPolish];
  __shared__ float2 amu[kMaxPolish];
  const int scene = blockIdx.y;
  const BatchShape& s = A.s;
  const int K = A.c.polish_size;
  const PolishScene* ps = reinterpret_cast<const PolishScene*>(A.p.pstate) + scene;
  if (threadIdx.x < K) {
    const int a = ps->active[threadIdx.x];
    atom[threadIdx.x] = a;
    atom1[threadIdx.x] = a / s.n2;
    atom2[threadIdx.x] = a % s.n2;
    amu[threadIdx.x] = ps->best_mean[threadIdx.x];
  }
  __syncthreads();
  const long long N = s.n();
  const float2* bp = A.p.bp + scene * N;
  uint32_t* keys = A.p.keys + scene * N;
  for (long long n = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int n1 = static_cast<int>(n / s.n2), n2 = static_cast<int>(n % s.n2);
    float2 r = __ldg(bp + n);
    bool act = false;
    for (int k = 0; k < K; ++k) {
      act |= atom[k] == n;
      const float2 t = cmul(amu[k], gram_at(A, nullptr, nullptr, n1, n2, atom1[k], atom2[k]));
      r = make_float2(r.x - t.x, r.y - t.y);
    }
    keys[n] = act ? 0u : float_key_t(abs_sq(r));
  }
}

template <typename T>
static void launch_exchange(const PolishArgs& A, const PolishBuffers& p, cudaStream_t st) {
  const dim3 grid(exchange_blocks(A.s), A.s.B);
  exchange_kernel<T><<<grid, T::threads, T::smem_bytes(A.s.n2), st>>>(A, p.cand_key, p.cand_idx);
}

void polish_run(const BatchShape& s, const DevConfig& c, const PolishBuffers& p,
                const FbmeOutputs& out, cudaStream_t st, Profiler* prof, const FbmeCertificate* cert) {
  PolishArgs A{s, c, p};
  const int K = c.polish_size;
  // each launch timed on its own, so the profile counts launches
  FBME_TIMED(prof, FBME_GROUP_TOPK, launch_topk_blocks(p.keys, s.n(), K, s.B, p.cand_key, p.cand_idx, st));
  FBME_TIMED(prof, FBME_GROUP_TOPK,
             launch_topk_merge(p.cand_key, p.cand_idx, topk_slices(s.n()) * K, K, s.B, p.active, p.score, st));
  const size_t dsm = (s.n1 + s.n2) * sizeof(float2);
  FBME_TIMED(prof, FBME_GROUP_POLISH, (polish_kernel<<<s.B, 32, dsm, st>>>(A, 0)));
  if (c.exchange > 0 && c.polish_iters > 1 && p.gram2d) {
    const long long nblk = (s.n() + 255) / 256;
    FBME_TIMED(prof, FBME_GROUP_EXCHANGE,
               (exchange_masked_kernel<<<dim3(static_cast<unsigned>(nblk < 1024 ? nblk : 1024), s.B), 256, 0, st>>>(A)));
    FBME_TIMED(prof, FBME_GROUP_TOPK,
               launch_topk_blocks(p.keys, s.n(), c.exchange, s.B, p.cand_key, p.cand_idx, st));
    FBME_TIMED(prof, FBME_GROUP_TOPK,
               launch_topk_merge(p.cand_key, p.cand_idx, topk_slices(s.n()) * c.exchange, c.exchange, s.B,
                                 p.xcand_idx, p.xcand_val, st));
    FBME_TIMED(prof, FBME_GROUP_POLISH, (polish_kernel<<<s.B, 32, dsm, st>>>(A, 1)));
  } else if (c.exchange > 0 && c.polish_iters > 1) {
    const int nb = exchange_blocks(s);
    if (s.n2 <= 64)
      FBME_TIMED(prof, FBME_GROUP_EXCHANGE, (launch_exchange<ExSmall>(A, p, st)));
    else if (s.n2 <= 128)
      FBME_TIMED(prof, FBME_GROUP_EXCHANGE, (launch_exchange<ExMid>(A, p, st)));
    else if (s.n2 <= 256)
      FBME_TIMED(prof, FBME_GROUP_EXCHANGE, (launch_exchange<ExWide>(A, p, st)));
    else
      FBME_TIMED(prof, FBME_GROUP_EXCHANGE, (launch_exchange<ExWidest>(A, p, st)));
    FBME_TIMED(prof, FBME_GROUP_TOPK,
               launch_topk_merge(p.cand_key, p.cand_idx, nb * c.exchange, c.exchange, s.B,
                                 p.xcand_idx, p.xcand_val, st));
    FBME_TIMED(prof, FBME_GROUP_POLISH, (polish_kernel<<<s.B, 32, dsm, st>>>(A, 1)));
  }
  if (cert) {  // model, scan, (decide + model, scan) per repair, final
    int resident = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, cert_scan_kernel, kCertThreads, dsm) !=
        cudaSuccess)
      resident = 1;
    const int nblk = cert_blocks(s, resident);
    for (int t = 0; t <= c.repairs + 1; ++t) {
      FBME_TIMED(prof, FBME_GROUP_CERTIFICATE,
                 (cert_step_kernel<<<s.B, 32, dsm, st>>>(A, *cert, cert->workspace, nblk, t)));
      if (t <= c.repairs)
        FBME_TIMED(prof, FBME_GROUP_CERTIFICATE,
                   (cert_scan_kernel<<<dim3(nblk, s.B), kCertThreads, dsm, st>>>(A, cert->workspace)));
    }
  }
  FBME_TIMED(prof, FBME_GROUP_POLISH, (polish_finish_kernel<<<s.B, 32, dsm, st>>>(A, out)));
  const int fb = static_cast<int>((s.n() + 2047) / 2048);
  FBME_TIMED(prof, FBME_GROUP_OUTPUT, (output_kernel<<<dim3(fb < 64 ? fb : 64, s.B), 256, 0, st>>>(A, out)));
}

// The polish of an uneven plan's buckets, one launch per step over all of
// them (at most kBucketSetMax per launch), in polish_run's order.  Buckets
// under an observation mask take polish_run.
static int exchange_class(int n2) { return n2 <= 64 ? 0 : n2 <= 128 ? 1 : n2 <= 256 ? 2 : 3; }

template <typename T>
static void launch_exchange_set(const PolishSet& S, int max_blocks, int max_b, int max_n2, cudaStream_t st) {
  exchange_set_kernel<T><<<dim3(max_blocks, max_b, S.n), T::threads, T::smem_bytes(max_n2), st>>>(S);
}

void polish_run_multi(const PolishBucket* b, int n, cudaStream_t st) {
  for (int c0 = 0; c0 < n; c0 += kBucketSetMax) {
    const int cnt = n - c0 < kBucketSetMax ? n - c0 : kBucketSetMax;
    std::vector<int> plain;  // set members (masked buckets run on their own)
    for (int i = 0; i < cnt; ++i) {
      const PolishBucket& k = b[c0 + i];
      if (k.p.gram2d) {
        polish_run(k.s, k.c, k.p, k.out, st);
        if (k.out.status && k.out.status != k.p.status)
          cudaMemcpyAsync(k.out.status, k.p.status, k.s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
      } else {
        plain.push_back(c0 + i);
      }
    }
    if (plain.empty()) continue;
    const int m = static_cast<int>(plain.size());
    auto* S = new PolishSet();  // ~31 KB: not on the stack
    TopkJobs tj{};
    TopkMergeJobs tm{}, tx{};
    S->n = m;
    tj.n = tm.n = m;
    int max_b = 1, max_slices = 1, max_out = 1;
    size_t dsm = 0;
    for (int i = 0; i < m; ++i) {
      const PolishBucket& k = b[plain[i]];
      const int K = k.c.polish_size, sl = topk_slices(k.s.n());
      S->a[i] = PolishArgs{k.s, k.c, k.p};
      S->out[i] = k.out;
      S->ex_blocks[i] = exchange_blocks(k.s);
      const int fb = static_cast<int>((k.s.n() + 2047) / 2048);
      S->out_blocks[i] = fb < 64 ? fb : 64;
      tj.j[i] = TopkJob{k.p.keys, k.s.n(), K, k.s.B, k.p.cand_key, k.p.cand_idx};
      tm.j[i] = TopkMergeJob{k.p.cand_key, k.p.cand_idx, sl * K, K, k.s.B, k.p.active, k.p.score};
      max_b = std::max(max_b, k.s.B);
      max_slices = std::max(max_slices, sl);
      max_out = std::max(max_out, S->out_blocks[i]);
      dsm = std::max(dsm, static_cast<size_t>(k.s.n1 + k.s.n2) * sizeof(float2));
    }
    launch_topk_blocks_multi(tj, max_slices, max_b, st);
    launch_topk_merge_multi(tm, max_b, st);
    const int pb = (max_b + kPolishWarps - 1) / kPolishWarps;
    polish_set_kernel<<<dim3(pb, 1, m), 32 * kPolishWarps, dsm, st>>>(*S, 0);
    // the exchange, one launch per row-tile class, then its candidates' merge
    bool any = false;
    for (int cls = 0; cls < 4; ++cls) {
      auto* X = new PolishSet();
      int xb = 1, xbl = 1, xn2 = 1;
      X->n = 0;
      for (int i = 0; i < m; ++i) {
        const PolishArgs& A = S->a[i];
        if (!(A.c.exchange > 0 && A.c.polish_iters > 1) || exchange_class(A.s.n2) != cls) continue;
        X->a[X->n] = A;
        X->ex_blocks[X->n] = S->ex_blocks[i];
        xb = std::max(xb, A.s.B);
        xbl = std::max(xbl, S->ex_blocks[i]);
        xn2 = std::max(xn2, A.s.n2);
        ++X->n;
      }
      if (X->n > 0) {
        any = true;
        if (cls == 0) launch_exchange_set<ExSmall>(*X, xbl, xb, xn2, st);
        else if (cls == 1) launch_exchange_set<ExMid>(*X, xbl, xb, xn2, st);
        else if (cls == 2) launch_exchange_set<ExWide>(*X, xbl, xb, xn2, st);
        else launch_exchange_set<ExWidest>(*X, xbl, xb, xn2, st);
      }
      delete X;
    }
    if (any) {
      tx.n = 0;
      for (int i = 0; i < m; ++i) {
        const PolishArgs& A = S->a[i];
        if (!(A.c.exchange > 0 && A.c.polish_iters > 1)) continue;
        const int E = A.c.exchange;
        tx.j[tx.n++] = TopkMergeJob{A.p.cand_key, A.p.cand_idx, S->ex_blocks[i] * E, E, A.s.B, A.p.xcand_idx,
                                    A.p.xcand_val};
      }
      launch_topk_merge_multi(tx, max_b, st);
      polish_set_kernel<<<dim3(pb, 1, m), 32 * kPolishWarps, dsm, st>>>(*S, 1);
    }
    polish_finish_set_kernel<<<dim3(max_b, 1, m), 32, dsm, st>>>(*S);
    output_set_kernel<<<dim3(max_out, max_b, m), 256, 0, st>>>(*S);
    for (int i = 0; i < m; ++i) {
      const PolishBucket& k = b[plain[i]];
      if (k.out.status && k.out.status != k.p.status)
        cudaMemcpyAsync(k.out.status, k.p.status, k.s.B * sizeof(int), cudaMemcpyDeviceToDevice, st);
    }
    delete S;
  }
}

}  // namespace fbme
