// UAMP stage of the FBME plan: initialisation, T_u message-passing sweeps
// and the final E-step, for a batch of equally shaped scenes.
//
// Per sweep (solver.py:2726-2870 with the fused Triton updates of
// triton_kernels.py:37-192, 267-417):
//   adjoint stage 1  prologue: message update  m' = d m + (1-d) (y - (p - dv m)) / (dv + nv)
//   adjoint stage 2  epilogue: Gaussian denoiser, damping, ARD prior update,
//                              per-tile sums of relevance (DOF) and variance
//   forward stage 1
//   forward stage 2  epilogue: prediction p = A mu and per-tile sum |y - p|^2
//   scalars          noise update (EM / evidence), data variance, pseudo variance
// The first sweep reuses A^H y from the initialisation (solver.py:2775-2783).
//
// Layouts: coefficient arrays [B][N1][N2], data arrays [B][M1][M2] (the
// caller's prefix block layout), forward intermediate [B][M2][N1], adjoint
// intermediate [B][N2][M1].  All reductions are per-tile sums written to
// fixed slots and added in a fixed order, so results are reproducible run
// to run.
#include <math.h>

#include <map>
#include <vector>

#include "denoise.cuh"
#include "dft_umma.cuh"
#include "kernels.cuh"
#include "stage.cuh"

namespace fbme {

// ---------------------------------------------------------------------------
// prologues
// ---------------------------------------------------------------------------

// Plain load; also sums |y|^2 (for the data power) over the column-tile-0 tiles.
struct ProYPower {
  static constexpr int kBatch = 16;
  static constexpr bool kPipelined = true;
  using Frag = float4;
  const float2* in;
  double* part;
  float acc;
  FBME_DEV void fetch(const TileCtx& t, long long e, int avail, Frag& f) const {
    f = load_pair(in, e, avail, t.g->vec4 != 0);
  }
  FBME_DEV float4 make(const TileCtx& t, long long, int, const Frag& v) {
    if (t.col_tile == 0) {
      acc += abs_sq(make_float2(v.x, v.y));
      acc += abs_sq(make_float2(v.z, v.w));
    }
    return v;
  }
  FBME_DEV void tile_done(const TileCtx& t, int w, int lane) {
    warp_partial(acc, part, t, 3, w, lane);
    acc = 0.f;
  }
};

// ---------------------------------------------------------------------------
// epilogues
// ---------------------------------------------------------------------------

// Forward stage 2: store the prediction and sum |y - p|^2.
struct EpiPredict {
  struct Pre {
    float2 y[8];
  };
  float2* pred;
  const float2* y;
  double* part;
  float acc;
  const uint8_t* mask;  // observation mask: the residual sums observed samples only
  FBME_DEV void prefetch(const TileCtx& t, int row, int c0, Pre& p) const {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    const float2* ys = y + t.scene * g.out_stride;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      p.y[i] = (r < g.rows && jb + i < g.cols) ? __ldg(ys + (jb + i) * g.out_ld + r)
                                               : make_float2(0.f, 0.f);
  }
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre& pre) {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    float2* ps = pred + t.scene * g.out_stride;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const float2 p = make_float2(v[2 * i], v[2 * i + 1]);
        ps[(jb + i) * g.out_ld + r] = p;
        const float dr = pre.y[i].x - p.x, di = pre.y[i].y - p.y;
        if (!mask || mask[(jb + i) * g.out_ld + r]) acc += dr * dr + di * di;
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx& t, int w, int lane) {
    warp_partial(acc, part, t, 2, w, lane);
    acc = 0.f;
  }
};

// Adjoint stage 2 during initialisation: store A^H y and sum |A^H y|^2.
struct EpiBackprojection {
  using Pre = NoPre;
  float2* bp;
  double* part;
  float acc;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    float2* bs = bp + t.scene * g.out_stride + r;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const float2 b = make_float2(v[2 * i], v[2 * i + 1]);
        bs[(jb + i) * g.out_ld] = b;
        acc += abs_sq(b);
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx& t, int w, int lane) {
    warp_partial(acc, part, t, 1, w, lane);
    acc = 0.f;
  }
};

// ---------------------------------------------------------------------------
// elementwise kernels
// ---------------------------------------------------------------------------
// Block coordinates of an elementwise body: block x of gx along a scene's
// range, scene y.  A plain launch passes blockIdx / gridDim; a launch merged
// over shape buckets passes each bucket's own block count, so every block
// covers the same elements (and sums them in the same order) as in the
// bucket's own launch.
struct Blk {
  int x, gx, y;
};
FBME_DEV Blk blk_here() {
  return Blk{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x), static_cast<int>(blockIdx.y)};
}
// ---------------------------------------------------------------------------
// Initial prior variances (solver.py:1063-1099): backprojection blend or
// uniform, floored; per-block sums of the result.
FBME_DEV void gamma0_body(Blk k, BatchShape s, DevConfig c, Scalars sc, const float2* bp, float* gamma,
                          double* part) {
  __shared__ double red[32];
  const int scene = k.y;
  const long long n = s.n();
  const float dp = sc.data_power[scene], fl = sc.floor_[scene];
  const float ebp = fmaxf(sc.ebp[scene], kEps);
  const float uniform = dp / static_cast<float>(n);
  float acc = 0.f;
  auto prior = [&](float2 b) {
    float g = uniform;
    if (c.blend >= 0.f) {
      const float structured = abs_sq(b) / ebp * dp;
      g = c.blend * structured + (1.0f - c.blend) * uniform;
    }
    g = fmaxf(g, fl);
    acc += g;
    return g;
  };
  const long long first = k.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long stride = static_cast<long long>(k.gx) * blockDim.x;
  if ((n & 1) == 0) {  // two coefficients per step, 16- and 8-byte accesses
    for (long long j = first; j < n / 2; j += stride) {
      const long long e = scene * n + 2 * j;
      const float4 b = __ldg(reinterpret_cast<const float4*>(bp + e));
      const float g0 = prior(make_float2(b.x, b.y));
      const float g1 = prior(make_float2(b.z, b.w));
      *reinterpret_cast<float2*>(gamma + e) = make_float2(g0, g1);
    }
  } else {
    for (long long i = first; i < n; i += stride) gamma[scene * n + i] = prior(bp[scene * n + i]);
  }
  write_block_partial(acc, red, part, scene, k.x, 0 * kPartWarps);
}
__global__ void __launch_bounds__(kEwThreads) gamma0_kernel(BatchShape s, DevConfig c, Scalars sc,
                                                            const float2* bp, float* gamma,
                                                            double* part) {
  gamma0_body(blk_here(), s, c, sc, bp, gamma, part);
}

// Denoiser of sweeps 2..T_u and of the final E-step, on the adjoint output
// A^H m that adjoint stage 2 stored (`lift`): the epilogue of that stage
// runs one CTA per SM, too few warps to keep the denoiser's loads in
// flight, while this kernel runs at full occupancy.  Per-block DOF and
// variance sums go to partial slots 0 and 1, as sweep1_kernel's.
FBME_DEV void denoise_body(Blk k, BatchShape s, DenoiseArgs a, const float2* lift) {
  __shared__ double red[32];
  const int scene = k.y;
  const long long n = s.n();
  const float pv = a.pv[scene], fl = a.floor_[scene];
  float dof = 0.f, sv = 0.f;
  auto one = [&](long long e, float g, float2 m, float v, float2 l) {
    const DenoiseOut o = denoise_math(a, g, m, v, l, pv, fl);
    dof += o.rel;
    sv += o.variance;
    return o;
  };
  const long long stride = static_cast<long long>(k.gx) * blockDim.x;
  const long long first = k.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if ((n & 1) == 0) {
    // two coefficients per step: 16-byte accesses to mu and the lift, 8-byte
    // to the variances (scene offsets are even, so every access is aligned)
    const long long base = scene * n;
    for (long long j = first; j < n / 2; j += stride) {
      const long long e = base + 2 * j;
      const float4 m = *reinterpret_cast<const float4*>(a.mu + e);
      const float4 l = __ldg(reinterpret_cast<const float4*>(lift + e));
      const float2 v = *reinterpret_cast<const float2*>(a.var + e);
      const float2 g = *reinterpret_cast<const float2*>(a.gamma + e);
      const DenoiseOut o0 = one(e, g.x, make_float2(m.x, m.y), v.x, make_float2(l.x, l.y));
      const DenoiseOut o1 = one(e + 1, g.y, make_float2(m.z, m.w), v.y, make_float2(l.z, l.w));
      *reinterpret_cast<float4*>(a.mu + e) = make_float4(o0.mean.x, o0.mean.y, o1.mean.x, o1.mean.y);
      *reinterpret_cast<float2*>(a.var + e) = make_float2(o0.variance, o1.variance);
      if (a.update_prior) *reinterpret_cast<float2*>(a.gamma + e) = make_float2(o0.gamma, o1.gamma);
      if (a.keys)
        *reinterpret_cast<uint2*>(a.keys + e) = make_uint2(float_key(abs_sq(o0.mean) + o0.variance),
                                                           float_key(abs_sq(o1.mean) + o1.variance));
    }
  } else {
    for (long long i = first; i < n; i += stride) {
      const long long e = scene * n + i;
      const DenoiseOut o = one(e, a.gamma[e], a.mu[e], a.var[e], lift[e]);
      a.mu[e] = o.mean;
      a.var[e] = o.variance;
      if (a.update_prior) a.gamma[e] = o.gamma;
      if (a.keys) a.keys[e] = float_key(abs_sq(o.mean) + o.variance);
    }
  }
  write_block_partial(dof, red, a.part, scene, k.x, 0 * kPartWarps);
  write_block_partial(sv, red, a.part, scene, k.x, 1 * kPartWarps);
}
__global__ void __launch_bounds__(kEwThreads) denoise_kernel(BatchShape s, DenoiseArgs a, const float2* lift) {
  denoise_body(blk_here(), s, a, lift);
}

// UAMP message update (triton_kernels.py:72-84) for sweeps 2..T_u and the
// final E-step: m' = d m + (1-d) prec (y - (p - dvar m)), into `msg_out`,
// which adjoint stage 1 then reads.  Full occupancy, two samples per step
// where y is 16-byte aligned and M even.
// Under an observation mask the message of an unobserved sample is zero: the
// masked operator's rows stop at the observed samples, and A^H of the
// zero-filled message is the masked adjoint (operators.py:255-280, 484-496).
FBME_DEV void message_body(Blk k, BatchShape s, const float2* y, const float2* pred, const float2* msg_in,
                           float2* msg_out, const float* prec, const float* dvar, float damping,
                           const uint8_t* mask = nullptr) {
  const int scene = k.y;
  const long long m = s.m();
  const float pr = prec[scene], dv = dvar[scene];
  const float keep = damping, upd = 1.0f - damping;
  auto step = [&](float2 yy, float2 pp, float2 mm) {
    const float2 pseudo = make_float2(pp.x - dv * mm.x, pp.y - dv * mm.y);
    const float2 cand = make_float2(pr * (yy.x - pseudo.x), pr * (yy.y - pseudo.y));
    return make_float2(keep * mm.x + upd * cand.x, keep * mm.y + upd * cand.y);
  };
  const long long first = k.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long stride = static_cast<long long>(k.gx) * blockDim.x;
  if ((m & 1) == 0 && (reinterpret_cast<uintptr_t>(y) & 15u) == 0) {
    for (long long j = first; j < m / 2; j += stride) {
      const long long e = scene * m + 2 * j;
      const float4 a = __ldg(reinterpret_cast<const float4*>(y + e));
      const float4 p = __ldg(reinterpret_cast<const float4*>(pred + e));
      const float4 q = __ldg(reinterpret_cast<const float4*>(msg_in + e));
      float2 o0 = step(make_float2(a.x, a.y), make_float2(p.x, p.y), make_float2(q.x, q.y));
      float2 o1 = step(make_float2(a.z, a.w), make_float2(p.z, p.w), make_float2(q.z, q.w));
      if (mask) {
        if (!mask[2 * j]) o0 = make_float2(0.f, 0.f);
        if (!mask[2 * j + 1]) o1 = make_float2(0.f, 0.f);
      }
      *reinterpret_cast<float4*>(msg_out + e) = make_float4(o0.x, o0.y, o1.x, o1.y);
    }
  } else {
    for (long long i = first; i < m; i += stride) {
      const long long e = scene * m + i;
      msg_out[e] = (mask && !mask[i]) ? make_float2(0.f, 0.f) : step(y[e], pred[e], msg_in[e]);
    }
  }
}
__global__ void __launch_bounds__(kEwThreads)
message_kernel(BatchShape s, const float2* y, const float2* pred, const float2* msg_in, float2* msg_out,
               const float* prec, const float* dvar, float damping, const uint8_t* mask) {
  message_body(blk_here(), s, y, pred, msg_in, msg_out, prec, dvar, damping, mask);
}

// First sweep: the lifted message is (1-d)/(dv+nv) * A^H y, the previous
// mean is zero and the previous variance equals the initial prior
// (solver.py:1160-1182, 2775-2783).  Blocks past `nblk_n` write the first
// message m1 = (1-d) * (y / (dv+nv)) instead.
FBME_DEV void sweep1_body(Blk k, BatchShape s, DevConfig c, Scalars sc, DenoiseArgs a, const float2* bp,
                          const float2* y, float2* msg, int nblk_n) {
  __shared__ double red[32];
  const int scene = k.y;
  if (static_cast<int>(k.x) >= nblk_n) {
    const long long m = s.m();
    const float pr = sc.prec[scene];
    const float keep = c.uamp_damping, upd = 1.0f - c.uamp_damping;
    for (long long i = (k.x - nblk_n) * static_cast<long long>(blockDim.x) + threadIdx.x;
         i < m; i += static_cast<long long>(k.gx - nblk_n) * blockDim.x) {
      const long long e = scene * m + i;
      const float2 yy = y[e];
      msg[e] = make_float2(keep * 0.0f + upd * (pr * yy.x), keep * 0.0f + upd * (pr * yy.y));
    }
    return;
  }
  const long long n = s.n();
  const float pv = sc.pv[scene], fl = sc.floor_[scene];
  const float scale = (1.0f - c.uamp_damping) / (fmaxf(sc.dvar[scene], kTiny) + sc.noise[scene]);
  float dof = 0.f, sv = 0.f;
  auto one = [&](float g0, float2 b) {
    const DenoiseOut o =
        denoise_math(a, g0, make_float2(0.f, 0.f), g0, make_float2(scale * b.x, scale * b.y), pv, fl);
    dof += o.rel;
    sv += o.variance;
    return o;
  };
  const long long first = k.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long stride = static_cast<long long>(nblk_n) * blockDim.x;
  if ((n & 1) == 0) {  // two coefficients per step, 16- and 8-byte accesses
    for (long long j = first; j < n / 2; j += stride) {
      const long long e = scene * n + 2 * j;
      const float2 g = *reinterpret_cast<const float2*>(a.gamma + e);
      const float4 b = __ldg(reinterpret_cast<const float4*>(bp + e));
      const DenoiseOut o0 = one(g.x, make_float2(b.x, b.y));
      const DenoiseOut o1 = one(g.y, make_float2(b.z, b.w));
      *reinterpret_cast<float4*>(a.mu + e) = make_float4(o0.mean.x, o0.mean.y, o1.mean.x, o1.mean.y);
      *reinterpret_cast<float2*>(a.var + e) = make_float2(o0.variance, o1.variance);
      if (a.update_prior) *reinterpret_cast<float2*>(a.gamma + e) = make_float2(o0.gamma, o1.gamma);
    }
  } else {
    for (long long i = first; i < n; i += stride) {
      const long long e = scene * n + i;
      const DenoiseOut o = one(a.gamma[e], bp[e]);
      a.mu[e] = o.mean;
      a.var[e] = o.variance;
      if (a.update_prior) a.gamma[e] = o.gamma;
    }
  }
  write_block_partial(dof, red, a.part, scene, k.x, 0 * kPartWarps);
  write_block_partial(sv, red, a.part, scene, k.x, 1 * kPartWarps);
}
__global__ void __launch_bounds__(kEwThreads) sweep1_kernel(BatchShape s, DevConfig c, Scalars sc,
                                                            DenoiseArgs a, const float2* bp,
                                                            const float2* y, float2* msg,
                                                            int nblk_n) {
  sweep1_body(blk_here(), s, c, sc, a, bp, y, msg, nblk_n);
}

// Per-scene scalar updates from the per-tile sums (fixed summation order).
enum ScalarMode { kScalarInit1 = 0, kScalarInit2 = 1, kScalarSweep = 2 };

// One warp per scene: lanes stride the partial slots, a fixed shuffle tree
// adds them, lane 0 applies the update.
constexpr int kScalarScenesPerBlock = 4;

FBME_DEV void scalars_body(Blk k, int mode, BatchShape s, DevConfig c, Scalars sc, const double* part,
                           PartSrc p0, PartSrc p1, PartSrc p2) {
  const int lane = threadIdx.x & 31;
  const int scene = k.x * kScalarScenesPerBlock + (threadIdx.x >> 5);
  if (scene >= s.B) return;
  auto sum = [&](int id, PartSrc src) {
    double v = 0.0;
    const int n = src.tiles * src.warps;
    for (int i = lane; i < n; i += 32) {
      const int t = i / src.warps, w = i % src.warps;
      v += part[(static_cast<long long>(scene) * kMaxTilesPerScene + t) * kPartSlots +
                id * kPartWarps + w];
    }
    return warp_sum(v);
  };
  const double Md = observed_samples(s, c);
  const float M = static_cast<float>(Md);
  // all reductions first (collective over the warp), then lane 0 alone
  const double r0 = mode == kScalarInit1 ? sum(3, p0) : sum(0, p0);
  const double r1 = mode == kScalarInit2 ? 0.0 : sum(1, p1);
  const double r2 = mode == kScalarSweep ? sum(2, p2) : 0.0;
  if (lane != 0) return;
  if (mode == kScalarInit1) {
    const double ysum = r0;
    const float dp = fmaxf(static_cast<float>(ysum / Md), kEps);
    const float fl = fmaxf(dp * c.min_var, kTiny);
    sc.data_power[scene] = dp;
    sc.floor_[scene] = fl;
    sc.data_energy[scene] = static_cast<float>(ysum);
    sc.ebp[scene] = static_cast<float>(r1);
    sc.noise[scene] = c.fixed_noise > 0.f ? c.fixed_noise : fmaxf(c.init_noise * dp, fl);
  } else if (mode == kScalarInit2) {
    const float dv = fmaxf(static_cast<float>(r0), kTiny);
    const float nv = sc.noise[scene];
    sc.dvar[scene] = dv;
    sc.pv[scene] = fmaxf((dv + nv) / M, kTiny);
    sc.prec[scene] = 1.0f / (dv + nv);
  } else {
    const float max_dof = static_cast<float>(Md * (1.0 - 10.0 * kEps));
    const float dof = fminf(static_cast<float>(r0), max_dof);
    const float sv = static_cast<float>(r1);
    const float energy = static_cast<float>(r2);
    const float fl = sc.floor_[scene];
    float nv = sc.noise[scene];
    if (!(c.fixed_noise > 0.f)) {
      float cand;
      if (c.noise_evidence)
        cand = (energy + c.noise_rate) / fmaxf(M - dof + c.noise_shape, kEps);
      else
        cand = (energy + nv * dof + c.noise_rate) / (M + c.noise_shape);
      cand = fmaxf(cand, fl);
      nv = c.damping * nv + (1.0f - c.damping) * cand;
      nv = fmaxf(nv, fl);
    }
    const float dv = fmaxf(sv, kTiny);
    sc.dof[scene] = dof;
    sc.energy[scene] = energy;
    sc.noise[scene] = nv;
    sc.dvar[scene] = dv;
    sc.pv[scene] = fmaxf((dv + nv) / M, kTiny);
    sc.prec[scene] = 1.0f / (dv + nv);
  }
}
__global__ void __launch_bounds__(32 * kScalarScenesPerBlock)
scalars_kernel(int mode, BatchShape s, DevConfig c, Scalars sc, const double* part, PartSrc p0, PartSrc p1,
               PartSrc p2) {
  scalars_body(blk_here(), mode, s, c, sc, part, p0, p1, p2);
}

// ---------------------------------------------------------------------------
// elementwise launches merged over shape buckets: blockIdx.z is the bucket;
// blocks past a bucket's own grid return at once
// ---------------------------------------------------------------------------
constexpr int kEwMulti = 64;
template <class J>
struct EwJobs {
  int n;
  J j[kEwMulti];
};
FBME_DEV bool ew_block(int gx, int scenes, Blk& k) {
  k = Blk{static_cast<int>(blockIdx.x), gx, static_cast<int>(blockIdx.y)};
  return k.x < gx && k.y < scenes;
}

struct Gamma0Job {
  int gx;
  BatchShape s;
  DevConfig c;
  Scalars sc;
  const float2* bp;
  float* gamma;
  double* part;
};
__global__ void __launch_bounds__(kEwThreads) gamma0_multi_kernel(const __grid_constant__ EwJobs<Gamma0Job> m) {
  const Gamma0Job& j = m.j[blockIdx.z];
  Blk k;
  if (ew_block(j.gx, j.s.B, k)) gamma0_body(k, j.s, j.c, j.sc, j.bp, j.gamma, j.part);
}

struct DenoiseJob {
  int gx;
  BatchShape s;
  DenoiseArgs a;
  const float2* lift;
};
__global__ void __launch_bounds__(kEwThreads) denoise_multi_kernel(const __grid_constant__ EwJobs<DenoiseJob> m) {
  const DenoiseJob& j = m.j[blockIdx.z];
  Blk k;
  if (ew_block(j.gx, j.s.B, k)) denoise_body(k, j.s, j.a, j.lift);
}

struct MessageJob {
  int gx;
  BatchShape s;
  const float2 *y, *pred, *msg_in;
  float2* msg_out;
  const float *prec, *dvar;
  float damping;
};
__global__ void __launch_bounds__(kEwThreads) message_multi_kernel(const __grid_constant__ EwJobs<MessageJob> m) {
  const MessageJob& j = m.j[blockIdx.z];
  Blk k;
  if (ew_block(j.gx, j.s.B, k)) message_body(k, j.s, j.y, j.pred, j.msg_in, j.msg_out, j.prec, j.dvar, j.damping);
}

struct Sweep1Job {
  int gx, nblk_n;
  BatchShape s;
  DevConfig c;
  Scalars sc;
  DenoiseArgs a;
  const float2 *bp, *y;
  float2* msg;
};
__global__ void __launch_bounds__(kEwThreads) sweep1_multi_kernel(const __grid_constant__ EwJobs<Sweep1Job> m) {
  const Sweep1Job& j = m.j[blockIdx.z];
  Blk k;
  if (ew_block(j.gx, j.s.B, k)) sweep1_body(k, j.s, j.c, j.sc, j.a, j.bp, j.y, j.msg, j.nblk_n);
}

// Scalar updates: blockIdx.x strides the bucket's scene blocks.
struct ScalarsJob {
  int gx;
  BatchShape s;
  DevConfig c;
  Scalars sc;
  const double* part;
  PartSrc p0, p1, p2;
};
__global__ void __launch_bounds__(32 * kScalarScenesPerBlock)
scalars_multi_kernel(int mode, const __grid_constant__ EwJobs<ScalarsJob> m) {
  const ScalarsJob& j = m.j[blockIdx.z];
  if (static_cast<int>(blockIdx.x) < j.gx)
    scalars_body(Blk{static_cast<int>(blockIdx.x), j.gx, 0}, mode, j.s, j.c, j.sc, j.part, j.p0, j.p1, j.p2);
}

// ---------------------------------------------------------------------------
// stage geometry and launch
// ---------------------------------------------------------------------------
cudaError_t set_dft_attributes() {
  cudaError_t e;
  if ((e = set_attr_both<ProPlain, EpiStoreT, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProYPower, EpiStoreT, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiPredict, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiBackprojection, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiSplitT, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProYPower, EpiSplitT, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProSplit, EpiStoreT, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProSplit, EpiPredict, true>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProSplit, EpiBackprojection, true>()) != cudaSuccess) return e;
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// the intermediate of a two-stage transform
// ---------------------------------------------------------------------------
// Stage 1 stores it in `tmp` and stage 2 reads it.  With `split` (plans of
// 3-term products) it is stage 2's A operand already split into BF16 parts
// and swizzled (EpiSplitT), which stage 2 bulk-copies (ProSplit); otherwise
// FP32 complex (EpiStoreT / ProPlain) that stage 2's producer splits.  The
// same FP32 values are split the same way in both, so results are identical.
static EpiSplitT split_epi(float2* tmp, const DftGeom& g2) {
  return EpiSplitT{reinterpret_cast<uint8_t*>(tmp), split_unit_bytes(g2.rows, g2.kcplx), g2.kchunks};
}
static ProSplit split_pro(const float2* tmp, const DftGeom& g2) {
  return ProSplit{reinterpret_cast<const uint8_t*>(tmp), split_unit_bytes(g2.rows, g2.kcplx)};
}
template <class Pro1>
static void stage1(int terms, bool split, const DftGeom& g1, const DftGeom& g2, const Pro1& p1, float2* tmp,
                   int* status, cudaStream_t st) {
  if (split)
    run_stage(terms, g1, p1, split_epi(tmp, g2), status, st);
  else
    run_stage(terms, g1, p1, EpiStoreT{tmp}, status, st);
}
template <class Epi2>
static void stage2(int terms, bool split, const DftGeom& g2, const float2* tmp, const Epi2& e2, int* status,
                   cudaStream_t st) {
  if (split)
    run_stage(terms, g2, split_pro(tmp, g2), e2, status, st);
  else
    run_stage(terms, g2, ProPlain{tmp}, e2, status, st);
}

// FP32 FFT form of stage `which` (dft_terms = 0), fft.cu: stages 1 contract
// the N2 axis, stages 2 the N1 axis; forward stages take the minus sign.
static void fft_of(Stage which, const BatchShape& s, const DftTables& t, const DftGeom& g, const float2* in,
                   float2* out, const float2* y, const uint8_t* mask, double* part, int mode, int ysum,
                   cudaStream_t st, const DenoiseArgs* dn = nullptr) {
  const bool ax2 = which == kFwd1 || which == kAdj1;
  fft_stage(g, ax2 ? s.n2 : s.n1, (which == kFwd1 || which == kFwd2) ? -1 : 1, ax2 ? t.fft_n2 : t.fft_n1, in,
            out, y, mask, part, mode, ysum, st, dn);
}
// Partial-sum source of an FFT stage: its row tiles x 8 warps.
static PartSrc fft_src(Stage which, const BatchShape& s, const DftGeom& g) {
  const bool ax2 = which == kFwd1 || which == kAdj1;
  return PartSrc{fft_stage_tiles(g.rows, ax2 ? s.n2 : s.n1), kPartWarps};
}

void dft_forward(const BatchShape& s, const DftTables& t, int terms, const float2* coeff,
                 float2* data, float2* tmp, int* status, cudaStream_t st) {
  const int nt = t.n_tile;
  const DftGeom g1 = stage_geom(kFwd1, s, t, nt), g2 = stage_geom(kFwd2, s, t, nt);
  if (terms == 0) {
    fft_of(kFwd1, s, t, g1, coeff, tmp, nullptr, nullptr, nullptr, 0, 0, st);
    fft_of(kFwd2, s, t, g2, tmp, data, nullptr, nullptr, nullptr, 0, 0, st);
    return;
  }
  stage1(terms, terms == 3, g1, g2, ProPlain{coeff}, tmp, status, st);
  stage2(terms, terms == 3, g2, tmp, EpiStoreT{data}, status, st);
}

void dft_adjoint(const BatchShape& s, const DftTables& t, int terms, const float2* data,
                 float2* coeff, float2* tmp, int* status, cudaStream_t st) {
  const int nt = t.n_tile;
  const DftGeom g1 = stage_geom(kAdj1, s, t, nt), g2 = stage_geom(kAdj2, s, t, nt);
  if (terms == 0) {
    fft_of(kAdj1, s, t, g1, data, tmp, nullptr, nullptr, nullptr, 0, 0, st);
    fft_of(kAdj2, s, t, g2, tmp, coeff, nullptr, nullptr, nullptr, 0, 0, st);
    return;
  }
  stage1(terms, terms == 3, g1, g2, ProPlain{data}, tmp, status, st);
  stage2(terms, terms == 3, g2, tmp, EpiStoreT{coeff}, status, st);
}

// Initialisation shared by the UAMP and PCG paths (solver.py:1063-1159):
// A^H y, data power, variance floor, initial noise and the initial prior
// variances (backprojection blend or uniform).
// Geometry of a stage whose prologue reads the caller's observations y:
// vector (16-byte) accesses need y itself 16-byte aligned, which a caller's
// pointer need not be (complex64 is 8-byte aligned).
// Denoiser arguments of a sweep (prior update on, no score keys).
static DenoiseArgs denoise_args(const DevConfig& c, const UampBuffers& u) {
  DenoiseArgs da;
  da.mu = u.mu;
  da.var = u.var;
  da.gamma = u.gamma;
  da.pv = u.sc.pv;
  da.floor_ = u.sc.floor_;
  da.part = u.part;
  da.keys = nullptr;
  da.damping = c.uamp_damping;
  da.prior_damping = c.damping;
  da.prior_max = c.max_prec;
  da.hyper_shape = c.hyper_shape;
  da.hyper_rate = c.hyper_rate;
  da.inv_hyper = 1.0f / (1.0f + c.hyper_shape);
  da.update_prior = 1;
  return da;
}

static DftGeom with_y(DftGeom g, const float2* y) {
  if (reinterpret_cast<uintptr_t>(y) & 15u) g.vec4 = 0;
  return g;
}

void sbl_init(const BatchShape& s, const DftTables& t, const DevConfig& c, const UampBuffers& u,
              cudaStream_t st, Profiler* prof, bool plain_prior) {
  const int nt = t.n_tile;
  const DftGeom a1 = with_y(stage_geom(kAdj1, s, t, nt), u.y), a2 = stage_geom(kAdj2, s, t, nt);
  const int sc_blocks = ceil_div(s.B, kScalarScenesPerBlock);
  const bool split = u.split && c.terms == 3;
  PartSrc src_y{a1.row_tiles * a1.col_tiles, kProWarps}, src_bp{a2.row_tiles * a2.col_tiles, kPartWarps};
  if (c.terms == 0) {  // FP32 FFT mode
    FBME_TIMED(prof, FBME_GROUP_INIT, fft_of(kAdj1, s, t, a1, u.y, u.tmp, nullptr, nullptr, u.part, 0, 1, st));
    FBME_TIMED(prof, FBME_GROUP_INIT, fft_of(kAdj2, s, t, a2, u.tmp, u.bp, nullptr, nullptr, u.part, 1, 0, st));
    src_y = fft_src(kAdj1, s, a1);
    src_bp = fft_src(kAdj2, s, a2);
  } else {
    FBME_TIMED(prof, FBME_GROUP_INIT,
               stage1(c.terms, split, a1, a2, ProYPower{u.y, u.part, 0.f}, u.tmp, u.status, st));
    FBME_TIMED(prof, FBME_GROUP_INIT,
               stage2(c.terms, split, a2, u.tmp, EpiBackprojection{u.bp, u.part, 0.f}, u.status, st));
  }
  FBME_TIMED(prof, FBME_GROUP_INIT,
             (scalars_kernel<<<sc_blocks, 32 * kScalarScenesPerBlock, 0, st>>>(
                 kScalarInit1, s, c, u.sc, u.part, src_y, src_bp, PartSrc{0, 0})));
  if (!plain_prior) return;
  const int bn = ew_blocks_host(s.n());
  FBME_TIMED(prof, FBME_GROUP_INIT,
             (gamma0_kernel<<<dim3(bn, s.B), kEwThreads, 0, st>>>(s, c, u.sc, u.bp, u.gamma,
                                                                  u.part)));
  FBME_TIMED(prof, FBME_GROUP_INIT,
             (scalars_kernel<<<sc_blocks, 32 * kScalarScenesPerBlock, 0, st>>>(kScalarInit2, s, c, u.sc, u.part,
                                                        PartSrc{bn, 1}, PartSrc{0, 0},
                                                        PartSrc{0, 0})));
}

// Message buffers ping-pong between sweeps: msg[0] / msg[1] are both
// M-sized regions starting at u.msg and u.msg + B*M.
void uamp_run(const BatchShape& s, const DftTables& t, const DevConfig& c, const UampBuffers& u,
              cudaStream_t st, Profiler* prof) {
  const int nt = t.n_tile;
  const DftGeom f1 = stage_geom(kFwd1, s, t, nt), f2 = stage_geom(kFwd2, s, t, nt);
  const DftGeom a1 = stage_geom(kAdj1, s, t, nt), a2 = stage_geom(kAdj2, s, t, nt);
  const int sc_blocks = ceil_div(s.B, kScalarScenesPerBlock);
  const long long BM = static_cast<long long>(s.B) * s.m();
  const bool split = u.split && c.terms == 3;
  float2* msg[2] = {u.msg, u.msg + BM};

  // A warm start replaces the initial prior, its partial sums and the
  // scalars computed from them, so the plain prior is not formed.
  const bool warm = u.warm_params != nullptr || u.warm_map != nullptr;
  sbl_init(s, t, c, u, st, prof, !warm);
  const int bn = ew_blocks_host(s.n()), bm = ew_blocks_host(s.m());
  if (warm) {
    // learned warm start: the network's prior (or a caller's map) replaces
    // the initial prior, then the scalar initialisation is redone from its sums
    if (u.warm_params)
      FBME_TIMED(prof, FBME_GROUP_INIT,
                 cnn_warm_prior(u.warm_params, u.bp, s.B, s.n1, s.n2, u.warm_ws, u.sc.data_power,
                                u.sc.floor_, u.gamma, u.part, bn, st, u.sc.ebp));
    else
      FBME_TIMED(prof, FBME_GROUP_INIT,
                 warm_prior_from_map(u.warm_map, s.B, s.n1, s.n2, u.sc.data_power, u.sc.floor_, u.gamma, u.part, bn,
                                     st));
    FBME_TIMED(prof, FBME_GROUP_INIT,
               (scalars_kernel<<<sc_blocks, 32 * kScalarScenesPerBlock, 0, st>>>(
                   kScalarInit2, s, c, u.sc, u.part, PartSrc{bn, 1}, PartSrc{0, 0}, PartSrc{0, 0})));
  }
  DenoiseArgs da = denoise_args(c, u);

  // the four stages: tensor-core split-BF16 products, or FP32 FFTs (dft_terms = 0)
  const bool fft = c.terms == 0;
  auto adj1 = [&](const float2* m) {
    if (fft) fft_of(kAdj1, s, t, a1, m, u.tmp, nullptr, nullptr, nullptr, 0, 0, st);
    else stage1(c.terms, split, a1, a2, ProPlain{m}, u.tmp, u.status, st);
  };
  auto adj2 = [&]() {
    if (fft) fft_of(kAdj2, s, t, a2, u.tmp, u.lift, nullptr, nullptr, nullptr, 0, 0, st);
    else stage2(c.terms, split, a2, u.tmp, EpiStoreT{u.lift}, u.status, st);
  };
  // FP32 FFT mode: adjoint stage 2 runs the denoiser in its epilogue, so
  // A^H m never goes to memory
  const bool fused_denoise = fft && fft_denoise_fused(s.n1);
  auto adj2_denoise = [&]() { fft_of(kAdj2, s, t, a2, u.tmp, nullptr, nullptr, nullptr, u.part, 3, 0, st, &da); };
  auto fwd1 = [&]() {
    if (fft) fft_of(kFwd1, s, t, f1, u.mu, u.tmp, nullptr, nullptr, nullptr, 0, 0, st);
    else stage1(c.terms, split, f1, f2, ProPlain{u.mu}, u.tmp, u.status, st);
  };
  auto fwd2 = [&]() {
    if (fft) fft_of(kFwd2, s, t, f2, u.tmp, u.pred, u.y, u.mask, u.part, 2, 0, st);
    else stage2(c.terms, split, f2, u.tmp, EpiPredict{u.pred, u.y, u.part, 0.f, u.mask}, u.status, st);
  };
  const PartSrc src_res = fft ? fft_src(kFwd2, s, f2) : PartSrc{f2.row_tiles * f2.col_tiles, kPartWarps};

  // --- sweeps ---
  int cur = 0;  // msg[cur] holds the latest message
  for (int it = 1; it <= c.uamp_iters; ++it) {
    PartSrc src_dof;
    if (it == 1) {
      FBME_TIMED(prof, FBME_GROUP_SWEEP1,
                 (sweep1_kernel<<<dim3(bn + bm, s.B), kEwThreads, 0, st>>>(s, c, u.sc, da, u.bp,
                                                                           u.y, msg[cur], bn)));
      src_dof = PartSrc{bn, 1};
    } else {
      FBME_TIMED(prof, FBME_GROUP_MESSAGE,
                 (message_kernel<<<dim3(bm, s.B), kEwThreads, 0, st>>>(s, u.y, u.pred, msg[cur], msg[cur ^ 1],
                                                                      u.sc.prec, u.sc.dvar, c.uamp_damping, u.mask)));
      FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE, adj1(msg[cur ^ 1]));
      cur ^= 1;
      if (fused_denoise) {
        FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, adj2_denoise());
        src_dof = fft_src(kAdj2, s, a2);
      } else {
        FBME_TIMED(prof, FBME_GROUP_ADJ_2, adj2());
        FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE,
                   (denoise_kernel<<<dim3(bn, s.B), kEwThreads, 0, st>>>(s, da, u.lift)));
        src_dof = PartSrc{bn, 1};
      }
    }
    FBME_TIMED(prof, FBME_GROUP_FWD_1, fwd1());
    FBME_TIMED(prof, FBME_GROUP_FWD_RESIDUAL, fwd2());
    FBME_TIMED(prof, FBME_GROUP_SCALARS,
               (scalars_kernel<<<sc_blocks, 32 * kScalarScenesPerBlock, 0, st>>>(
                   kScalarSweep, s, c, u.sc, u.part, src_dof, src_dof, src_res)));
  }

  // --- final E-step (no prior update, no prediction), score keys ---
  FBME_TIMED(prof, FBME_GROUP_MESSAGE,
             (message_kernel<<<dim3(bm, s.B), kEwThreads, 0, st>>>(s, u.y, u.pred, msg[cur], msg[cur ^ 1],
                                                                  u.sc.prec, u.sc.dvar, c.uamp_damping, u.mask)));
  FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE, adj1(msg[cur ^ 1]));
  da.update_prior = 0;
  da.keys = reinterpret_cast<uint32_t*>(u.keys);
  if (fused_denoise) {
    FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, adj2_denoise());
  } else {
    FBME_TIMED(prof, FBME_GROUP_ADJ_2, adj2());
    FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE,
               (denoise_kernel<<<dim3(bn, s.B), kEwThreads, 0, st>>>(s, da, u.lift)));
  }
}

// ---------------------------------------------------------------------------
// several shape buckets at once
// ---------------------------------------------------------------------------
static_assert(sizeof(EwJobs<Sweep1Job>) < 32000, "merged launch parameters exceed the 32 KB limit");
static_assert(sizeof(StageSet<ProYPower, EpiPredict, kStageSetMax>) < 32000,
              "merged stage parameters exceed the 32 KB limit");

// Merged elementwise launches of `jobs` in groups of kEwMulti; the grid is
// the largest bucket's block count x scene count x buckets.
template <class J, class F>
static void ew_launch(const std::vector<J>& jobs, F&& launch) {
  EwJobs<J> m;
  for (size_t i0 = 0; i0 < jobs.size(); i0 += kEwMulti) {
    m.n = 0;
    int gx = 1, gy = 1;
    for (size_t i = i0; i < jobs.size() && m.n < kEwMulti; ++i) {
      m.j[m.n++] = jobs[i];
      gx = jobs[i].gx > gx ? jobs[i].gx : gx;
      gy = jobs[i].s.B > gy ? jobs[i].s.B : gy;
    }
    launch(m, dim3(gx, gy, m.n));
  }
}

static void scalars_multi(int mode, const std::vector<ScalarsJob>& jobs, cudaStream_t st) {
  ew_launch(jobs, [&](const EwJobs<ScalarsJob>& m, dim3 g) {
    scalars_multi_kernel<<<dim3(g.x, 1, g.z), 32 * kScalarScenesPerBlock, 0, st>>>(mode, m);
  });
}

// uamp_run for several shape buckets (no warm start): each stage and
// elementwise step is one launch over all buckets, and bucket b takes part
// in sweeps 1..T_u(b) only.  A bucket's blocks, tiles and summation orders
// are those of its own uamp_run, so the results are identical.
void uamp_run_multi(const UampJob* J, int nb, cudaStream_t st, Profiler* prof, const cudaStream_t* aux,
                    const cudaEvent_t* ev, int naux) {
  std::vector<DftGeom> f1(nb), f2(nb), a1(nb), a2(nb);
  std::vector<int> bn(nb), bm(nb), cur(nb, 0);
  int iters = 0;
  for (int b = 0; b < nb; ++b) {
    const BatchShape& s = J[b].s;
    const int nt = J[b].t.n_tile;
    f1[b] = stage_geom(kFwd1, s, J[b].t, nt);
    f2[b] = stage_geom(kFwd2, s, J[b].t, nt);
    a1[b] = stage_geom(kAdj1, s, J[b].t, nt);
    a2[b] = stage_geom(kAdj2, s, J[b].t, nt);
    bn[b] = ew_blocks_host(s.n());
    bm[b] = ew_blocks_host(s.m());
    iters = J[b].c.uamp_iters > iters ? J[b].c.uamp_iters : iters;
  }
  auto msg = [&](int b, int which) { return J[b].u.msg + which * static_cast<long long>(J[b].s.B) * J[b].s.m(); };
  auto sgx = [&](int b) { return ceil_div(J[b].s.B, kScalarScenesPerBlock); };
  // Stage 1 / stage 2 of the buckets `bs` through their intermediates (the
  // pre-split form for 3-term buckets, FP32 for the others: two launches
  // when a step holds both kinds).
  auto split_of = [&](int b) { return J[b].u.split && J[b].c.terms == 3; };
  auto stage1_m = [&](const std::vector<int>& bs, const std::vector<DftGeom>& g1, const std::vector<DftGeom>& g2,
                      auto pro) {
    using P = decltype(pro(0));
    std::vector<StageJob<P, EpiSplitT>> js;
    std::vector<StageJob<P, EpiStoreT>> jp;
    for (int b : bs) {
      if (split_of(b))
        js.push_back({J[b].c.terms, {g1[b], pro(b), split_epi(J[b].u.tmp, g2[b]), J[b].u.status}});
      else
        jp.push_back({J[b].c.terms, {g1[b], pro(b), EpiStoreT{J[b].u.tmp}, J[b].u.status}});
    }
    if (!js.empty()) run_stage_multi(js.data(), static_cast<int>(js.size()), st);
    if (!jp.empty()) run_stage_multi(jp.data(), static_cast<int>(jp.size()), st);
  };
  auto stage2_m = [&](const std::vector<int>& bs, const std::vector<DftGeom>& g2, auto epi) {
    using E = decltype(epi(0));
    std::vector<StageJob<ProSplit, E>> js;
    std::vector<StageJob<ProPlain, E>> jp;
    for (int b : bs) {
      if (split_of(b))
        js.push_back({J[b].c.terms, {g2[b], split_pro(J[b].u.tmp, g2[b]), epi(b), J[b].u.status}});
      else
        jp.push_back({J[b].c.terms, {g2[b], ProPlain{J[b].u.tmp}, epi(b), J[b].u.status}});
    }
    if (!js.empty()) run_stage_multi(js.data(), static_cast<int>(js.size()), st);
    if (!jp.empty()) run_stage_multi(jp.data(), static_cast<int>(jp.size()), st);
  };
  // FP32 FFT buckets (dft_terms 0): each stage step is one two-pass kernel
  // launch per transform length, over the buckets of that length
  auto is_fft = [&](int b) { return J[b].c.terms == 0; };
  auto tens_of = [&](const std::vector<int>& bs) {
    std::vector<int> r;
    for (int b : bs)
      if (!is_fft(b)) r.push_back(b);
    return r;
  };
  auto fft_m = [&](Stage which, const std::vector<int>& bs, const std::vector<DftGeom>& g, int mode,
                   auto make) {
    const bool ax2 = which == kFwd1 || which == kAdj1;
    const int sign = (which == kFwd1 || which == kFwd2) ? -1 : 1;
    std::map<int, std::vector<FftSetJob>> by_len;
    for (int b : bs) {
      if (!is_fft(b)) continue;
      FftSetJob j = make(b);
      j.g = g[b];
      j.tw = ax2 ? J[b].t.fft_n2 : J[b].t.fft_n1;
      by_len[ax2 ? J[b].s.n2 : J[b].s.n1].push_back(j);
    }
    // lengths 1.. on side streams, forked from and joined back to `st`, so
    // the launches of one step overlap instead of queueing
    const int nl = static_cast<int>(by_len.size());
    const bool fork = !prof && nl > 1 && aux && ev && naux >= nl - 1;
    if (fork) {
      cudaEventRecord(ev[0], st);
      for (int k = 1; k < nl; ++k) cudaStreamWaitEvent(aux[k - 1], ev[0], 0);
    }
    int k = 0;
    for (auto& kv : by_len) {
      const cudaStream_t sk = fork && k > 0 ? aux[k - 1] : st;
      fft_stage_set(kv.second.data(), static_cast<int>(kv.second.size()), kv.first, sign, mode, sk);
      ++k;
    }
    if (fork)
      for (int j = 1; j < nl; ++j) {
        cudaEventRecord(ev[j], aux[j - 1]);
        cudaStreamWaitEvent(st, ev[j], 0);
      }
  };
  auto job = [](const float2* in, float2* out, double* part = nullptr) {
    FftSetJob j{};
    j.in = in;
    j.out = out;
    j.part = part;
    return j;
  };
  auto fft_part = [&](Stage which, int b, const DftGeom& g) {
    const bool ax2 = which == kFwd1 || which == kAdj1;
    return PartSrc{fft_stage_tiles(g.rows, ax2 ? J[b].s.n2 : J[b].s.n1), kPartWarps};
  };
  // FFT buckets whose adjoint stage 2 runs the denoiser in its epilogue
  auto fused = [&](int b) { return is_fft(b) && fft_denoise_fused(J[b].s.n1); };
  std::vector<DenoiseArgs> das(nb);
  std::vector<int> all(nb);
  for (int b = 0; b < nb; ++b) all[b] = b;

  // --- initialisation (sbl_init) ---
  {
    std::vector<DftGeom> a1ys(nb);
    std::vector<ScalarsJob> s1, s2;
    std::vector<Gamma0Job> g0;
    for (int b = 0; b < nb; ++b) {
      const UampBuffers& u = J[b].u;
      const DftGeom a1y = with_y(a1[b], u.y);
      a1ys[b] = a1y;
      if (is_fft(b))
        s1.push_back({sgx(b), J[b].s, J[b].c, u.sc, u.part, fft_part(kAdj1, b, a1y), fft_part(kAdj2, b, a2[b]),
                      PartSrc{0, 0}});
      else
        s1.push_back({sgx(b), J[b].s, J[b].c, u.sc, u.part, PartSrc{a1y.row_tiles * a1y.col_tiles, kProWarps},
                      PartSrc{a2[b].row_tiles * a2[b].col_tiles, kPartWarps}, PartSrc{0, 0}});
      g0.push_back({bn[b], J[b].s, J[b].c, u.sc, u.bp, u.gamma, u.part});
      s2.push_back({sgx(b), J[b].s, J[b].c, u.sc, u.part, PartSrc{bn[b], 1}, PartSrc{0, 0}, PartSrc{0, 0}});
    }
    const std::vector<int> tens = tens_of(all);
    FBME_TIMED(prof, FBME_GROUP_INIT, stage1_m(tens, a1ys, a2, [&](int b) {
                 return ProYPower{J[b].u.y, J[b].u.part, 0.f};
               }));
    FBME_TIMED(prof, FBME_GROUP_INIT, fft_m(kAdj1, all, a1ys, 0, [&](int b) {
                 FftSetJob j = job(J[b].u.y, J[b].u.tmp, J[b].u.part);
                 j.ysum = 1;
                 return j;
               }));
    FBME_TIMED(prof, FBME_GROUP_INIT, stage2_m(tens, a2, [&](int b) {
                 return EpiBackprojection{J[b].u.bp, J[b].u.part, 0.f};
               }));
    FBME_TIMED(prof, FBME_GROUP_INIT, fft_m(kAdj2, all, a2, 1, [&](int b) {
                 return job(J[b].u.tmp, J[b].u.bp, J[b].u.part);
               }));
    FBME_TIMED(prof, FBME_GROUP_INIT, scalars_multi(kScalarInit1, s1, st));
    FBME_TIMED(prof, FBME_GROUP_INIT, ew_launch(g0, [&](const EwJobs<Gamma0Job>& m, dim3 g) {
                 gamma0_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
               }));
    FBME_TIMED(prof, FBME_GROUP_INIT, scalars_multi(kScalarInit2, s2, st));
  }

  // --- sweeps ---
  for (int it = 1; it <= iters; ++it) {
    std::vector<int> act;
    for (int b = 0; b < nb; ++b)
      if (J[b].c.uamp_iters >= it) act.push_back(b);
    if (it == 1) {
      std::vector<Sweep1Job> j;
      for (int b : act) {
        const UampBuffers& u = J[b].u;
        j.push_back({bn[b] + bm[b], bn[b], J[b].s, J[b].c, u.sc, denoise_args(J[b].c, u), u.bp, u.y, msg(b, cur[b])});
      }
      FBME_TIMED(prof, FBME_GROUP_SWEEP1, ew_launch(j, [&](const EwJobs<Sweep1Job>& m, dim3 g) {
                   sweep1_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
                 }));
    } else {
      std::vector<MessageJob> jm;
      std::vector<DenoiseJob> jd;
      std::vector<int> lifted, fusing;
      for (int b : act) {
        const UampBuffers& u = J[b].u;
        jm.push_back({bm[b], J[b].s, u.y, u.pred, msg(b, cur[b]), msg(b, cur[b] ^ 1), u.sc.prec, u.sc.dvar,
                      J[b].c.uamp_damping});
        das[b] = denoise_args(J[b].c, u);
        if (fused(b)) {
          fusing.push_back(b);
        } else {
          lifted.push_back(b);
          jd.push_back({bn[b], J[b].s, das[b], u.lift});
        }
      }
      FBME_TIMED(prof, FBME_GROUP_MESSAGE, ew_launch(jm, [&](const EwJobs<MessageJob>& m, dim3 g) {
                   message_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
                 }));
      FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE,
                 stage1_m(tens_of(act), a1, a2, [&](int b) { return ProPlain{msg(b, cur[b] ^ 1)}; }));
      FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE,
                 fft_m(kAdj1, act, a1, 0, [&](int b) { return job(msg(b, cur[b] ^ 1), J[b].u.tmp); }));
      for (int b : act) cur[b] ^= 1;
      FBME_TIMED(prof, FBME_GROUP_ADJ_2,
                 stage2_m(tens_of(lifted), a2, [&](int b) { return EpiStoreT{J[b].u.lift}; }));
      FBME_TIMED(prof, FBME_GROUP_ADJ_2,
                 fft_m(kAdj2, lifted, a2, 0, [&](int b) { return job(J[b].u.tmp, J[b].u.lift); }));
      FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, fft_m(kAdj2, fusing, a2, 3, [&](int b) {
                   FftSetJob j = job(J[b].u.tmp, nullptr, J[b].u.part);
                   j.dn = &das[b];
                   return j;
                 }));
      if (!jd.empty())
        FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, ew_launch(jd, [&](const EwJobs<DenoiseJob>& m, dim3 g) {
                     denoise_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
                   }));
    }
    FBME_TIMED(prof, FBME_GROUP_FWD_1,
               stage1_m(tens_of(act), f1, f2, [&](int b) { return ProPlain{J[b].u.mu}; }));
    FBME_TIMED(prof, FBME_GROUP_FWD_1, fft_m(kFwd1, act, f1, 0, [&](int b) { return job(J[b].u.mu, J[b].u.tmp); }));
    {
      std::vector<ScalarsJob> sj;
      for (int b : act) {
        const UampBuffers& u = J[b].u;
        const PartSrc dof = it > 1 && fused(b) ? fft_part(kAdj2, b, a2[b]) : PartSrc{bn[b], 1};
        const PartSrc res =
            is_fft(b) ? fft_part(kFwd2, b, f2[b]) : PartSrc{f2[b].row_tiles * f2[b].col_tiles, kPartWarps};
        sj.push_back({sgx(b), J[b].s, J[b].c, u.sc, u.part, dof, dof, res});
      }
      FBME_TIMED(prof, FBME_GROUP_FWD_RESIDUAL, stage2_m(tens_of(act), f2, [&](int b) {
                   return EpiPredict{J[b].u.pred, J[b].u.y, J[b].u.part, 0.f};
                 }));
      FBME_TIMED(prof, FBME_GROUP_FWD_RESIDUAL, fft_m(kFwd2, act, f2, 2, [&](int b) {
                   FftSetJob j = job(J[b].u.tmp, J[b].u.pred, J[b].u.part);
                   j.y = J[b].u.y;
                   j.mask = J[b].u.mask;
                   return j;
                 }));
      FBME_TIMED(prof, FBME_GROUP_SCALARS, scalars_multi(kScalarSweep, sj, st));
    }
  }

  // --- final E-step (no prior update, no prediction), score keys ---
  std::vector<MessageJob> jm;
  std::vector<DenoiseJob> jd;
  std::vector<int> lifted, fusing;
  for (int b = 0; b < nb; ++b) {
    const UampBuffers& u = J[b].u;
    jm.push_back({bm[b], J[b].s, u.y, u.pred, msg(b, cur[b]), msg(b, cur[b] ^ 1), u.sc.prec, u.sc.dvar,
                  J[b].c.uamp_damping});
    das[b] = denoise_args(J[b].c, u);
    das[b].update_prior = 0;
    das[b].keys = reinterpret_cast<uint32_t*>(u.keys);
    if (fused(b)) {
      fusing.push_back(b);
    } else {
      lifted.push_back(b);
      jd.push_back({bn[b], J[b].s, das[b], u.lift});
    }
  }
  FBME_TIMED(prof, FBME_GROUP_MESSAGE, ew_launch(jm, [&](const EwJobs<MessageJob>& m, dim3 g) {
               message_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
             }));
  FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE,
             stage1_m(tens_of(all), a1, a2, [&](int b) { return ProPlain{msg(b, cur[b] ^ 1)}; }));
  FBME_TIMED(prof, FBME_GROUP_ADJ_MESSAGE,
             fft_m(kAdj1, all, a1, 0, [&](int b) { return job(msg(b, cur[b] ^ 1), J[b].u.tmp); }));
  FBME_TIMED(prof, FBME_GROUP_ADJ_2, stage2_m(tens_of(lifted), a2, [&](int b) { return EpiStoreT{J[b].u.lift}; }));
  FBME_TIMED(prof, FBME_GROUP_ADJ_2, fft_m(kAdj2, lifted, a2, 0, [&](int b) { return job(J[b].u.tmp, J[b].u.lift); }));
  FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, fft_m(kAdj2, fusing, a2, 3, [&](int b) {
               FftSetJob j = job(J[b].u.tmp, nullptr, J[b].u.part);
               j.dn = &das[b];
               return j;
             }));
  if (!jd.empty())
    FBME_TIMED(prof, FBME_GROUP_ADJ_DENOISE, ew_launch(jd, [&](const EwJobs<DenoiseJob>& m, dim3 g) {
                 denoise_multi_kernel<<<g, kEwThreads, 0, st>>>(m);
               }));
}

}  // namespace fbme


// ---------------------------------------------------------------------------
// failure-detection self-test of the stage kernel's bounded waits
// ---------------------------------------------------------------------------
namespace fbme {

// One 128 x 128 output tile over one 64-wide K chunk: input 128 x 32
// complex, output 128 x 128 complex, one 256-column twiddle block of two
// parts (nothing of it is read: the producer is held).
size_t stage_selftest_bytes() { return 128 * 32 * 8 + 128 * 128 * 8 + 2 * 256 * 128; }

// Launch that stage with its producer held back and `wait_cycles` as the
// wait limit: the issuer's wait for a full stage and the epilogue's wait
// for the accumulator run out, record FBME_STATUS_TIMEOUT in *status, and
// the kernel returns.
cudaError_t stage_selftest(void* ws, int* status, long long wait_cycles, cudaStream_t st) {
  uint8_t* p = static_cast<uint8_t*>(ws);
  float2* in = reinterpret_cast<float2*>(p);
  float2* out = reinterpret_cast<float2*>(p + 128 * 32 * 8);
  const uint8_t* table = p + 128 * 32 * 8 + 128 * 128 * 8;
  const DftGeom g = make_geom(1, 128, 32, 128, 32, 128 * 32, 128, 128 * 128, table, 1, 256);
  StageSet<ProPlain, EpiStoreT, 1> set;
  set.n = 1;
  set.tile0[0] = 0;
  set.tile0[1] = tiles(g);
  set.it[0] = StageItem<ProPlain, EpiStoreT>{g, ProPlain{in}, EpiStoreT{out}, status};
  set.wait_cycles = wait_cycles;
  set.hold = 1;
  cudaError_t e = set_attr<2, 256, ProPlain, EpiStoreT, 1>();
  if (e != cudaSuccess) return e;
  launch_set<2, 256>(set, st);
  return cudaGetLastError();
}

}  // namespace fbme
