// PCG + Hutchinson sparse Bayesian learning (mode="cg") for a batch of
// equally shaped scenes.
//
// Follows torch_sbl/solver.py (FBME-SBL v1.1):
//   fast_sbl mode="cg"        1063-1159 (initialisation, shared with UAMP),
//                             1191-1221 (probe count, lifted probes),
//                             1315-1904 (EM loop), 2023-2080 (final posterior)
//   _posterior (cg branch)    2991-3036
//   _pcg                      5582-5723
//   low-rank preconditioner   5786-5848 (+ Cholesky loading 2898-2931)
//   _project_relevance        3156-3181
//   _cg_schedule              6086-6118 (host side)
//
// Layout.  A "unit" is one right-hand side of one scene: unit = b*R + j,
// j = 0 the data y, j >= 1 the Hutchinson probes.  PCG vectors are
// [B][R][M1][M2] complex64; lifted vectors [B][R][N1][N2].
//
// Matvec.  Q v = noise v + A diag(prior) A^H v runs on the tcgen05 DFT
// stage kernel over all units at once (the reference's "fourier" matvec;
// its default "tbt" form applies the same matrix through a BTTB embedding,
// operators.py:299-371):
//   adjoint 1  prologue forms the direction d = z + beta d_prev (masked)
//   adjoint 2  epilogue multiplies by the prior variances
//   forward 1
//   forward 2  epilogue adds noise * d, stores Q d and the per-tile
//              partial sums of Re(d^H Q d) (FP64)
//
// Preconditioner.  Q ~ b I + F F^H with F the K strongest Fourier atoms
// scaled by sqrt(prior); applied by the Woodbury identity
//   z = r/b - F (S^-1 (F^H r / b)) / b,   S = I + F^H F / b.
// F is never stored: each vector kernel evaluates its slice of atoms from
// exact integer phases; F^H F comes from the Dirichlet tables.
//
// Every inner product that steers the iteration (alpha, beta, residual
// norms) and the Hutchinson average are accumulated in FP64, per block or
// per tile, and summed in a fixed order: results are reproducible run to
// run.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <map>
#include <vector>

#include "dft_umma.cuh"
#include "kernels.cuh"
#include "stage.cuh"

namespace fbme {

constexpr int kCgRankMax = 32;
constexpr int kCgSlice = 256;   // samples per block in the PCG vector kernels
constexpr int kCgThreads = 256;
constexpr int kCgChunk = 16;    // right-hand sides staged together in shared memory
constexpr int kDSlots = 4;      // FP64 partials per (block, unit): rho', |r|^2, |b|^2
constexpr int kFsLd = 33;       // padded row of the staged atom slice

enum CgFinish { kFinishInit = 0, kFinishStep = 1, kFinishRestart = 2 };

struct CgArgs {
  BatchShape s;
  int R;       // right-hand sides per scene
  int K;       // preconditioner rank
  int nblk;    // vector-kernel blocks per scene
  const float2* rhs;
  float2 *x, *r, *z, *q;
  const float2* d;  // current direction
  const float* gamma;
  const float* noise;
  const long long* pidx;  // [B][K] top-K prior indices
  const float* pval;      // [B][K] their prior variances
  const float* bg;        // [B] preconditioner background
  const float2* F;        // [B][M][kCgRankMax] preconditioner atoms
  const float2* sinv;     // [B][K][K]
  float2* w;              // [B][R][K] Woodbury weights
  float2* ppart;          // [B][nblk][R][K] projection partials
  double* dpart;          // [B][nblk][R][kDSlots]
  const double* cpart;    // curvature partials per unit (stage layout)
  int ctiles;             // tiles per unit of the forward-2 stage
  double* rho;
  float* beta;
  int* dmask;
  int* active;
  int* valid;
  int* improved;
  float* init_norm;
  float* rel;
  float* best_rel;
  int* any_active;
  float tol;
  const float* tol_dev;  // the tolerance in device memory (graph-resident loops), else nullptr
  int fixed;
};

// ---------------------------------------------------------------------------
// Fourier atoms of the preconditioner
// ---------------------------------------------------------------------------

// sqrt(v) * exp(-2 pi i (m1 n1 / N1 + m2 n2 / N2)) with the phase reduced
// exactly in integers (operators.py:444-466 forms the same atom).
FBME_DEV float2 atom_value(const BatchShape& s, int m1, int m2, long long idx, float sv) {
  const unsigned long long n1 = static_cast<unsigned long long>(idx / s.n2);
  const unsigned long long n2 = static_cast<unsigned long long>(idx % s.n2);
  const unsigned long long N1 = s.n1, N2 = s.n2, NN = N1 * N2;
  const unsigned long long a = (static_cast<unsigned long long>(m1) * n1) % N1;
  const unsigned long long b = (static_cast<unsigned long long>(m2) * n2) % N2;
  long long num = static_cast<long long>((a * N2 + b * N1) % NN);
  if (2 * num >= static_cast<long long>(NN)) num -= static_cast<long long>(NN);
  const float turns = static_cast<float>(2.0 * static_cast<double>(num) / static_cast<double>(NN));
  float sn, cs;
  sincospif(turns, &sn, &cs);
  return make_float2(sv * cs, -sv * sn);
}

// ---------------------------------------------------------------------------
// DFT-stage policies of the matvec
// ---------------------------------------------------------------------------

// Adjoint-1 prologue: direction d = dmask ? (beta != 0 ? z + beta d_prev : z)
// : 0 (solver.py:5712-5719 and the restarts of 5697-5705), written to
// d_out by the column-tile-0 tiles and fed to the tensor core.
struct ProDirection {
  static constexpr int kBatch = 8;
  static constexpr bool kPipelined = false;
  struct Frag {
    float2 z0, z1, d0, d1;
  };
  const float2* z;
  const float2* d_in;
  float2* d_out;
  const float* beta;
  const int* dmask;
  FBME_DEV void fetch(const TileCtx& t, long long e, int avail, Frag& f) const {
    if (avail <= 0) {
      f.z0 = f.z1 = f.d0 = f.d1 = make_float2(0.f, 0.f);
      return;
    }
    const bool vec = vec_ok(*t.g);
    load2c(z, e, avail, vec, f.z0, f.z1);
    load2c(d_in, e, avail, vec, f.d0, f.d1);
  }
  FBME_DEV float4 make(const TileCtx& t, long long e, int avail, const Frag& f) const {
    if (avail <= 0) return make_float4(0.f, 0.f, 0.f, 0.f);
    const int mk = dmask[t.scene];
    const float bt = beta[t.scene];
    auto dir = [&](float2 zz, float2 dd) {
      if (!mk) return make_float2(0.f, 0.f);
      if (bt == 0.f) return zz;
      return make_float2(zz.x + bt * dd.x, zz.y + bt * dd.y);
    };
    const float2 o0 = dir(f.z0, f.d0);
    const float2 o1 = avail >= 2 ? dir(f.z1, f.d1) : make_float2(0.f, 0.f);
    if (t.col_tile == 0) {
      if (avail >= 2 && vec_ok(*t.g)) {
        *reinterpret_cast<float4*>(d_out + e) = make_float4(o0.x, o0.y, o1.x, o1.y);
      } else {
        d_out[e] = o0;
        if (avail >= 2) d_out[e + 1] = o1;
      }
    }
    return make_float4(o0.x, o0.y, o1.x, o1.y);
  }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Adjoint-2 epilogue: prior[b] * (A^H v) into [unit][N1][N2].
struct EpiGamma {
  using Pre = NoPre;
  float2* out;
  const float* gamma;
  int R;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) const {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    const int b = t.scene / R;
    float2* o = out + t.scene * g.out_stride + r;
    const float* gm = gamma + b * g.out_stride + r;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const float gg = gm[(jb + i) * g.out_ld];
        o[(jb + i) * g.out_ld] = make_float2(gg * v[2 * i], gg * v[2 * i + 1]);
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Forward-2 epilogue of Q d: q = acc + noise * d, partial Re(d^H q).
struct EpiCurv {
  using Pre = NoPre;
  float2* q;
  const float2* d;
  const float* noise;
  double* part;
  int R;
  double acc;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    const float nv = noise[t.scene / R];
    const long long base = t.scene * g.out_stride + r;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const long long e = base + static_cast<long long>(jb + i) * g.out_ld;
        const float2 dv = d[e];
        const float2 qq = make_float2(v[2 * i] + nv * dv.x, v[2 * i + 1] + nv * dv.y);
        q[e] = qq;
        acc += static_cast<double>(dv.x) * qq.x + static_cast<double>(dv.y) * qq.y;
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx& t, int w, int lane) {
    warp_partial(acc, part, t, 0, w, lane);
    acc = 0.0;
  }
};

// Forward-2 epilogue of the true residual r = rhs - (acc + noise * x).
struct EpiResid {
  using Pre = NoPre;
  float2* r;
  const float2* rhs;
  const float2* x;
  const float* noise;
  int R;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) const {
    const DftGeom& g = *t.g;
    const int rr = t.row0() + row;
    if (rr >= g.rows) return;
    const float nv = noise[t.scene / R];
    const long long base = t.scene * g.out_stride + rr;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const long long e = base + static_cast<long long>(jb + i) * g.out_ld;
        const float2 xv = x[e], bv = rhs[e];
        const float qx = v[2 * i] + nv * xv.x, qy = v[2 * i + 1] + nv * xv.y;
        r[e] = make_float2(bv.x - qx, bv.y - qy);
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Forward-2 epilogue of the noise update: partial |y - A mean|^2.
struct EpiEnergy {
  using Pre = NoPre;
  const float2* y;
  double* part;
  double acc;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    const long long base = t.scene * g.out_stride + r;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) {
        const float2 yy = __ldg(y + base + static_cast<long long>(jb + i) * g.out_ld);
        const float dr = yy.x - v[2 * i], di = yy.y - v[2 * i + 1];
        const float h = hypotf(dr, di);
        acc += static_cast<double>(h * h);
      }
    }
  }
  FBME_DEV void tile_done(const TileCtx& t, int w, int lane) {
    warp_partial(acc, part, t, 2, w, lane);
    acc = 0.0;
  }
};

// ---------------------------------------------------------------------------
// PCG vector kernels (grid: blocks x scenes, one sample per thread)
// ---------------------------------------------------------------------------

// alpha of unit u from the forward-2 curvature partials (solver.py:5652-5662).
FBME_DEV float unit_alpha(const CgArgs& A, int unit, int* valid_out) {
  const double curv = unit_sum(A.cpart, unit, 0, A.ctiles, kPartWarps);
  const double rho = A.rho[unit];
  const double tiny = static_cast<double>(kTiny);
  const bool ok = A.active[unit] && isfinite(curv) && isfinite(rho) && curv > tiny && rho > tiny;
  *valid_out = ok ? 1 : 0;
  return ok ? static_cast<float>(rho / fmax(curv, tiny)) : 0.f;
}

// Atom matrix of the preconditioner, F[b][m][k] (rows of kCgRankMax, zero
// past K), rebuilt once per preconditioner from the top-K prior indices.
__global__ void __launch_bounds__(256) cg_atoms_kernel(BatchShape s, int K, const long long* pidx,
                                                       const float* pval, float2* F) {
  const int b = blockIdx.y;
  const long long M = s.m();
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= M * kCgRankMax) return;
  const long long m = i / kCgRankMax;
  const int k = static_cast<int>(i % kCgRankMax);
  float2 f = make_float2(0.f, 0.f);
  if (k < K)
    f = atom_value(s, static_cast<int>(m / s.m2), static_cast<int>(m % s.m2), pidx[b * K + k],
                   sqrtf(pval[b * K + k]));
  F[static_cast<long long>(b) * M * kCgRankMax + i] = f;
}

// Vector kernels: grid (sample blocks, scenes, groups of kCgChunk units).
// STEP: x += alpha d (and r -= alpha q when PROJ) with alpha of this
// iteration; PROJ: per-block partials of F^H r; NORMS: partials of |r|^2
// and |rhs|^2.  Block 0 of each scene and group records valid
// (solver.py:5656-5663).
template <bool STEP, bool PROJ, bool NORMS>
__global__ void __launch_bounds__(kCgThreads) cg_vector_kernel(const __grid_constant__ CgArgs A) {
  extern __shared__ float2 cg_smem[];
  float2* Fs = cg_smem;                      // [kCgSlice][kFsLd]
  float2* Rs = cg_smem + kCgSlice * kFsLd;   // [kCgChunk][kCgSlice]
  __shared__ float s_alpha[kCgChunk];
  __shared__ double s_red[kCgThreads / 32][kCgChunk][2];
  const int b = blockIdx.y, blk = blockIdx.x, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.z * kCgChunk;
  const int nc = min(kCgChunk, A.R - c0);
  const long long M = A.s.m();
  const long long m0 = static_cast<long long>(blk) * kCgSlice;
  const long long m = m0 + tid;
  const bool inb = m < M;
  if (STEP && tid < nc) {
    int ok = 0;
    s_alpha[tid] = unit_alpha(A, b * A.R + c0 + tid, &ok);
    if (blk == 0) A.valid[b * A.R + c0 + tid] = ok;
  }
  if (PROJ && A.K > 0) {
    const float2* Fb = A.F + (static_cast<long long>(b) * M + m0) * kCgRankMax;
    const long long rows = min(static_cast<long long>(kCgSlice), M - m0);
    for (int e = tid; e < kCgSlice * kCgRankMax; e += kCgThreads) {
      const int row = e / kCgRankMax, k = e % kCgRankMax;
      Fs[row * kFsLd + k] = row < rows ? Fb[e] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  for (int j = 0; j < nc; ++j) {
    const long long unit = static_cast<long long>(b) * A.R + c0 + j;
    const long long e = unit * M + m;
    float2 rv = make_float2(0.f, 0.f);
    if (inb) {
      if (STEP) {
        const float al = s_alpha[j];
        const float2 dv = A.d[e];
        float2 xv = A.x[e];
        xv.x += al * dv.x;
        xv.y += al * dv.y;
        A.x[e] = xv;
        if (PROJ) {
          const float2 qv = A.q[e];
          rv = A.r[e];
          rv.x -= al * qv.x;
          rv.y -= al * qv.y;
          A.r[e] = rv;
        }
      } else if (PROJ || NORMS) {
        rv = A.r[e];
      }
    }
    if (PROJ) Rs[j * kCgSlice + tid] = rv;
    if (NORMS) {
      double rr = static_cast<double>(rv.x) * rv.x + static_cast<double>(rv.y) * rv.y;
      double bb = 0.0;
      if (inb) {
        const float2 bv = A.rhs[e];
        bb = static_cast<double>(bv.x) * bv.x + static_cast<double>(bv.y) * bv.y;
      }
      rr = warp_sum(rr);
      bb = warp_sum(bb);
      if (lane == 0) {
        s_red[warp][j][0] = rr;
        s_red[warp][j][1] = bb;
      }
    }
  }
  __syncthreads();
  if (NORMS && tid < nc) {
    double rr = 0.0, bb = 0.0;
    for (int w = 0; w < kCgThreads / 32; ++w) {
      rr += s_red[w][tid][0];
      bb += s_red[w][tid][1];
    }
    double* dp = A.dpart + ((static_cast<long long>(b) * A.nblk + blk) * A.R + c0 + tid) * kDSlots;
    dp[1] = rr;
    dp[2] = bb;
  }
  if (PROJ && lane < A.K) {
    // thread (k = lane, warp): units warp, warp + 8 of the group
    for (int j = warp; j < nc; j += kCgThreads / 32) {
      float ax = 0.f, ay = 0.f;
      const float2* rs = Rs + j * kCgSlice;
#pragma unroll 8
      for (int tt = 0; tt < kCgSlice; ++tt) {
        const float2 f = Fs[tt * kFsLd + lane];
        const float2 rv = rs[tt];
        ax += f.x * rv.x + f.y * rv.y;  // conj(f) * r
        ay += f.x * rv.y - f.y * rv.x;
      }
      A.ppart[((static_cast<long long>(b) * A.nblk + blk) * A.R + c0 + j) * A.K + lane] =
          make_float2(ax, ay);
    }
  }
}

// Woodbury weights w = S^-1 (F^H r / b): one block per unit; thread
// (k, group) sums every eighth block partial, then warp 0 applies S^-1.
__global__ void __launch_bounds__(256) cg_weights_kernel(const __grid_constant__ CgArgs A) {
  __shared__ double s_u[8][kCgRankMax][2];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const long long unit = blockIdx.x;
  const int b = static_cast<int>(unit / A.R), j = static_cast<int>(unit % A.R);
  double ux = 0.0, uy = 0.0;
  if (lane < A.K) {
    for (int blk = grp; blk < A.nblk; blk += 8) {
      const float2 p = A.ppart[((static_cast<long long>(b) * A.nblk + blk) * A.R + j) * A.K + lane];
      ux += p.x;
      uy += p.y;
    }
  }
  s_u[grp][lane][0] = ux;
  s_u[grp][lane][1] = uy;
  __syncthreads();
  if (grp != 0) return;
  ux = 0.0;
  uy = 0.0;
  for (int g = 0; g < 8; ++g) {
    ux += s_u[g][lane][0];
    uy += s_u[g][lane][1];
  }
  const float inv_b = 1.0f / A.bg[b];
  const float2 ut = make_float2(static_cast<float>(ux) * inv_b, static_cast<float>(uy) * inv_b);
  float2 acc = make_float2(0.f, 0.f);
  const float2* S = A.sinv + static_cast<long long>(b) * A.K * A.K;
  for (int l = 0; l < A.K; ++l) {
    const float2 ul = make_float2(__shfl_sync(0xffffffffu, ut.x, l), __shfl_sync(0xffffffffu, ut.y, l));
    if (lane < A.K) {
      const float2 sv = S[lane * A.K + l];
      acc.x += sv.x * ul.x - sv.y * ul.y;
      acc.y += sv.x * ul.y + sv.y * ul.x;
    }
  }
  if (lane < A.K) A.w[unit * A.K + lane] = acc;
}

// z = r / b - F w / b and partials of Re(r^H z) (solver.py:5836-5848);
// grid as the vector kernels.
__global__ void __launch_bounds__(kCgThreads) cg_precond_kernel(const __grid_constant__ CgArgs A) {
  __shared__ float2 Ws[kCgChunk][kCgRankMax];
  __shared__ double s_red[kCgThreads / 32][kCgChunk];
  const int b = blockIdx.y, blk = blockIdx.x, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.z * kCgChunk;
  const int nc = min(kCgChunk, A.R - c0);
  const long long M = A.s.m();
  const long long m = static_cast<long long>(blk) * kCgSlice + tid;
  const bool inb = m < M;
  for (int i = tid; i < nc * A.K; i += blockDim.x)
    Ws[i / A.K][i % A.K] = A.w[(static_cast<long long>(b) * A.R + c0) * A.K + i];
  float2 f[kCgRankMax];
  if (A.K > 0 && inb) {
    const float4* fr = reinterpret_cast<const float4*>(A.F + (static_cast<long long>(b) * M + m) * kCgRankMax);
#pragma unroll
    for (int k2 = 0; k2 < kCgRankMax / 2; ++k2) {
      const float4 v = __ldg(fr + k2);
      f[2 * k2] = make_float2(v.x, v.y);
      f[2 * k2 + 1] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll
    for (int k = 0; k < kCgRankMax; ++k) f[k] = make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float bgv = A.bg[b];
  for (int j = 0; j < nc; ++j) {
    const long long unit = static_cast<long long>(b) * A.R + c0 + j;
    const long long e = unit * M + m;
    double rz = 0.0;
    if (inb) {
      const float2 rv = A.r[e];
      float cx = 0.f, cy = 0.f;
#pragma unroll
      for (int k = 0; k < kCgRankMax; ++k) {
        if (k < A.K) {
          const float2 ww = Ws[j][k];
          cx += f[k].x * ww.x - f[k].y * ww.y;
          cy += f[k].x * ww.y + f[k].y * ww.x;
        }
      }
      const float2 zv = make_float2(rv.x / bgv - cx / bgv, rv.y / bgv - cy / bgv);
      A.z[e] = zv;
      rz = static_cast<double>(rv.x) * zv.x + static_cast<double>(rv.y) * zv.y;
    }
    rz = warp_sum(rz);
    if (lane == 0) s_red[warp][j] = rz;
  }
  __syncthreads();
  if (tid < nc) {
    double v = 0.0;
    for (int w = 0; w < kCgThreads / 32; ++w) v += s_red[w][tid];
    A.dpart[((static_cast<long long>(b) * A.nblk + blk) * A.R + c0 + tid) * kDSlots + 0] = v;
  }
}

// Per-unit PCG scalars after the preconditioner: one warp per unit sums the
// block partials (lanes stride the blocks, fixed shuffle tree).
__global__ void __launch_bounds__(256) cg_finish_kernel(const __grid_constant__ CgArgs A, int mode) {
  const int lane = threadIdx.x & 31;
  const long long unit = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (unit >= static_cast<long long>(A.s.B) * A.R) return;
  const int b = static_cast<int>(unit / A.R), j = static_cast<int>(unit % A.R);
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for (int blk = lane; blk < A.nblk; blk += 32) {
    const double* dp = A.dpart + ((static_cast<long long>(b) * A.nblk + blk) * A.R + j) * kDSlots;
    rz += dp[0];
    if (mode != kFinishStep) {
      rr += dp[1];
      bb += dp[2];
    }
  }
  rz = warp_sum(rz);
  rr = warp_sum(rr);
  bb = warp_sum(bb);
  if (lane != 0) return;
  const double tiny = static_cast<double>(kTiny);
  const float tol = A.tol_dev ? *A.tol_dev : A.tol;
  if (mode == kFinishInit) {
    // solver.py:5620-5639
    const float inorm = fmaxf(static_cast<float>(sqrt(bb)), kEps);
    A.init_norm[unit] = inorm;
    const float rn = static_cast<float>(sqrt(rr));
    const int act = rn > tol * inorm ? 1 : 0;
    A.active[unit] = act;
    A.dmask[unit] = act;
    A.beta[unit] = 0.f;
    A.rho[unit] = rz;
    A.best_rel[unit] = rn / inorm;
    A.improved[unit] = 1;
  } else if (mode == kFinishStep) {
    // solver.py:5709-5721
    const double rho = A.rho[unit];
    const int upd = A.valid[unit] && isfinite(rz) && rz > tiny;
    A.beta[unit] = upd ? static_cast<float>(rz / fmax(rho, tiny)) : 0.f;
    A.rho[unit] = upd ? rz : rho;
    A.dmask[unit] = upd;
    A.active[unit] = upd;
  } else {
    // solver.py:5667-5707
    const float rl = static_cast<float>(sqrt(rr)) / A.init_norm[unit];
    A.rel[unit] = rl;
    int act = (isfinite(rl) && rl > tol) ? 1 : 0;
    if (A.fixed) {
      act = act && A.valid[unit];
      const int imp = rl < A.best_rel[unit];
      A.improved[unit] = imp;
      if (imp) A.best_rel[unit] = rl;
    }
    act = act && isfinite(rz) && rz > tiny;
    A.active[unit] = act;
    A.dmask[unit] = act;
    A.beta[unit] = 0.f;
    if (act) {
      A.rho[unit] = rz;
      atomicOr(A.any_active, 1);
    }
  }
}

// Fixed-iteration mode: keep the best checkpoint (solver.py:5677-5687).
__global__ void cg_best_kernel(BatchShape s, int R, const int* improved, const float2* x,
                               float2* best) {
  const long long M = s.m();
  const long long units = static_cast<long long>(s.B) * R;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < units * M;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (improved[i / M]) best[i] = x[i];
  }
}

// ---------------------------------------------------------------------------
// Preconditioner factorisation: one warp per scene (solver.py:5786-5833)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) cg_precond_build_kernel(BatchShape s, int K, float jitter_mult,
                                                              const long long* pidx,
                                                              const float* pval, const float* gsum,
                                                              const float* noise, const float2* d1,
                                                              const float2* d2, float* bg,
                                                              float2* sinv, int* status) {
  __shared__ float2 Mx[kCgRankMax][kCgRankMax + 1];
  __shared__ float2 X[kCgRankMax][kCgRankMax + 1];
  const int b = blockIdx.x, lane = threadIdx.x;
  const bool on = lane < K;
  const long long my_idx = on ? pidx[b * K + lane] : 0;
  const float my_v = on ? pval[b * K + lane] : 0.f;
  const float my_sv = sqrtf(my_v);
  const double vsum = warp_sum(static_cast<double>(my_v));
  const float total = gsum[b];
  const float omitted = fmaxf(total - static_cast<float>(vsum), 0.f);
  const float bgv = fmaxf(noise[b] + omitted, kEps * total);
  const int n1i = static_cast<int>(my_idx / s.n2), n2i = static_cast<int>(my_idx % s.n2);
  // S = I + F^H F / b with (F^H F)[k][l] = sqrt(v_k v_l) D1(n1_k - n1_l) D2(n2_k - n2_l)
  for (int l = 0; l < K; ++l) {
    const long long il = __shfl_sync(0xffffffffu, my_idx, l);
    const float svl = __shfl_sync(0xffffffffu, my_sv, l);
    if (on) {
      int a1 = n1i - static_cast<int>(il / s.n2), a2 = n2i - static_cast<int>(il % s.n2);
      if (a1 < 0) a1 += s.n1;
      if (a2 < 0) a2 += s.n2;
      const float2 g = cmul(d1[a1], d2[a2]);
      const float sc = my_sv * svl / bgv;
      float2 a = make_float2(sc * g.x, sc * g.y);
      if (l == lane) a.x += 1.0f;
      Mx[lane][l] = a;
    }
  }
  __syncwarp();
  float2 row[kCgRankMax];
#pragma unroll
  for (int j = 0; j < kCgRankMax; ++j)
    if (on && j < K) {
      const float2 a = Mx[lane][j], c = Mx[j][lane];
      row[j] = make_float2(0.5f * (a.x + c.x), 0.5f * (a.y - c.y));
    }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < kCgRankMax; ++j)
    if (on && j < K) Mx[lane][j] = row[j];
  __syncwarp();
  // deterministic loading max(10, m) * eps * mean|Re diag| (solver.py:2907-2920)
  float dsum = on ? fabsf(Mx[lane][lane].x) : 0.f;
  dsum = warp_sum(dsum);
  const float scale = fmaxf(dsum / static_cast<float>(K), kTiny);
  if (on) Mx[lane][lane].x += fmaxf(10.0f, jitter_mult) * (kEps * scale);
  __syncwarp();
  int bad = 0;
  for (int j = 0; j < K; ++j) {
    if (lane == j) {
      float sd = Mx[j][j].x;
      for (int q = 0; q < j; ++q) sd -= abs2(Mx[j][q]);
      if (!(sd > 0.f) || !isfinite(sd)) {
        bad = 1;
        sd = 1.0f;
      }
      Mx[j][j] = make_float2(sqrtf(sd), 0.f);
    }
    __syncwarp();
    const float ljj = Mx[j][j].x;
    if (on && lane > j) {
      float2 v = Mx[lane][j];
      for (int q = 0; q < j; ++q) {
        const float2 a = Mx[lane][q], c = Mx[j][q];
        v.x -= a.x * c.x + a.y * c.y;
        v.y -= a.y * c.x - a.x * c.y;
      }
      Mx[lane][j] = make_float2(v.x / ljj, v.y / ljj);
    }
    __syncwarp();
  }
  bad = __reduce_or_sync(0xffffffffu, bad);
  // X = L^-1, column `lane`
  if (on) {
    for (int i = 0; i < K; ++i) X[i][lane] = make_float2(0.f, 0.f);
    X[lane][lane] = make_float2(1.0f / Mx[lane][lane].x, 0.f);
    for (int i = lane + 1; i < K; ++i) {
      float2 acc = make_float2(0.f, 0.f);
      for (int q = lane; q < i; ++q) {
        const float2 l = Mx[i][q], x = X[q][lane];
        acc.x += l.x * x.x - l.y * x.y;
        acc.y += l.x * x.y + l.y * x.x;
      }
      const float lii = Mx[i][i].x;
      X[i][lane] = make_float2(-acc.x / lii, -acc.y / lii);
    }
  }
  __syncwarp();
  // S^-1 = X^H X: column `lane`
  float2* Sb = sinv + static_cast<long long>(b) * K * K;
  if (on) {
    for (int i = 0; i < K; ++i) {
      float2 acc = make_float2(0.f, 0.f);
      const int k0 = i > lane ? i : lane;
      for (int k = k0; k < K; ++k) {
        const float2 a = X[k][i], c = X[k][lane];  // conj(a) * c
        acc.x += a.x * c.x + a.y * c.y;
        acc.y += a.x * c.y - a.y * c.x;
      }
      Sb[i * K + lane] = bad ? make_float2(0.f, 0.f) : acc;
    }
  }
  if (lane == 0) {
    // a failed factorisation falls back to the scalar preconditioner
    // (solver.py:5825-5830)
    bg[b] = bad ? noise[b] + total : bgv;
    if (bad && status) atomicOr(status + b, FBME_STATUS_CHOLESKY);
  }
}

// ---------------------------------------------------------------------------
// EM step kernels (grid: blocks x scenes over the N coefficients)
// ---------------------------------------------------------------------------

// Hutchinson diagonal, posterior mean / variance and clipped relevance
// (solver.py:3017-3036, 3156-3163).  Partial sums of the relevance go to
// sum 0 of `part`.
__global__ void __launch_bounds__(kEwThreads)
cg_hutch_kernel(BatchShape s, int R, int count, int P, const float2* ls, const float2* lp,
                const float* gamma, float2* mean, float* relc, float* pv_out, double* part) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const long long N = s.n();
  double acc_rel = 0.0;
  const double inv_count = count > 0 ? 1.0 / count : 0.0;
  for (long long n = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (int p = 1; p <= count; ++p) {
      const float2 a = ls[(static_cast<long long>(b) * R + p) * N + n];
      const float2 c = lp[(static_cast<long long>(b) * P + p - 1) * N + n];
      acc += static_cast<double>(a.x) * c.x + static_cast<double>(a.y) * c.y;  // Re(a conj(c))
    }
    const float dd = fmaxf(static_cast<float>(acc * inv_count), 0.f);
    const float g = gamma[b * N + n];
    const float2 l0 = ls[static_cast<long long>(b) * R * N + n];
    mean[b * N + n] = make_float2(g * l0.x, g * l0.y);
    const float rc = fminf(fmaxf(g * dd, 0.f), 1.f);
    relc[b * N + n] = rc;
    if (pv_out) pv_out[b * N + n] = fmaxf(g - g * g * dd, 0.f);
    acc_rel += rc;
  }
  write_block_partial(acc_rel, red, part, b, blockIdx.x, 0 * kPartWarps);
}

struct CgEmArgs {
  BatchShape s;
  int nb;  // blocks per scene of the hutch / EM kernels
  const double* part;
  double* part2;
  const float2* mean;
  float2* prev;
  const float* relc;
  float* gamma;
  const float* floor_;
  float keep, hyper_shape, hyper_rate, max_prec;
  // after an active-set switch: 1 on the active set; the prior variances
  // elsewhere keep their value (ARD deletion is permanent, solver.py:1684-1693)
  const uint8_t* amask;
};

FBME_DEV float relevance_scale(const double* part, int b, int nb, long long M) {
  double raw = 0.0;
  for (int t = 0; t < nb; ++t)
    raw += part[(static_cast<long long>(b) * kMaxTilesPerScene + t) * kPartSlots + 0];
  const float max_dof = static_cast<float>(static_cast<double>(M) * (1.0 - 10.0 * kEps));
  return fminf(1.0f, max_dof / fmaxf(static_cast<float>(raw), kEps));
}

// MacKay prior update with damping and floor (solver.py:1669-1677,
// 1768-1778) and the relative-change sums (1820-1824).
__global__ void __launch_bounds__(kEwThreads) cg_em_kernel(const __grid_constant__ CgEmArgs A) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const long long N = A.s.n();
  const float scale = relevance_scale(A.part, b, A.nb, A.s.m());
  const float fl = A.floor_[b];
  const float lo = 1.0f / A.max_prec;
  double gs = 0.0, dn = 0.0, mn = 0.0;
  for (long long n = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long e = b * N + n;
    const float rel = fminf(fmaxf(A.relc[e], 0.f), 1.f) * scale;
    const float2 mu = A.mean[e];
    const float am = abs_sq(mu);
    float prec = (rel + A.hyper_shape) / (am + A.hyper_rate);
    prec = fminf(fmaxf(prec, lo), A.max_prec);
    const float gold = A.gamma[e];
    const float gnew = (A.amask && !A.amask[e]) ? gold : 1.0f / prec;
    const float g = fmaxf(A.keep * gold + (1.0f - A.keep) * gnew, fl);
    A.gamma[e] = g;
    gs += g;
    const float2 pm = A.prev[e];
    const float dx = mu.x - pm.x, dy = mu.y - pm.y;
    dn += static_cast<double>(dx) * dx + static_cast<double>(dy) * dy;
    mn += static_cast<double>(mu.x) * mu.x + static_cast<double>(mu.y) * mu.y;
    A.prev[e] = mu;
  }
  write_block_partial(gs, red, A.part2, b, blockIdx.x, 0 * kPartWarps);
  write_block_partial(dn, red, A.part2, b, blockIdx.x, 1 * kPartWarps);
  write_block_partial(mn, red, A.part2, b, blockIdx.x, 2 * kPartWarps);
}

struct CgScalarArgs {
  BatchShape s;
  int nb;            // hutch / EM blocks per scene
  int etiles;        // forward-2 tiles per scene (energy partials)
  const double* part;
  const double* part2;
  float* noise;
  const float* floor_;
  float* gsum;
  float* dof;
  float* change;
  float* hist;       // row of 6 floats for this iteration, or nullptr
  float keep, fixed_noise, noise_shape, noise_rate;
  int evidence;
  int cg_iters, probes;
  const int* cg_iters_dev;  // PCG iterations counted on the device (graph-resident loop), else nullptr
  float cg_tol;
  int update;        // 0: final pass (DOF only)
};

// Per-scene DOF, noise update (solver.py:1737-1791) and relative change;
// one block, history row from block reductions.
__global__ void __launch_bounds__(256) cg_scalars_kernel(const __grid_constant__ CgScalarArgs A) {
  __shared__ double red[32];
  const float M = static_cast<float>(A.s.m());
  double cmax = 0.0, nsum = 0.0, dsum = 0.0;
  for (int b = threadIdx.x; b < A.s.B; b += blockDim.x) {
    double raw = 0.0;
    for (int t = 0; t < A.nb; ++t)
      raw += A.part[(static_cast<long long>(b) * kMaxTilesPerScene + t) * kPartSlots + 0];
    const float max_dof = static_cast<float>(static_cast<double>(A.s.m()) * (1.0 - 10.0 * kEps));
    const float sc = fminf(1.0f, max_dof / fmaxf(static_cast<float>(raw), kEps));
    const float dofv = static_cast<float>(raw * sc);
    A.dof[b] = dofv;
    if (A.update) {
      double energy = 0.0, gs = 0.0, dn = 0.0, mn = 0.0;
      for (int t = 0; t < A.etiles; ++t)
        for (int w = 0; w < kPartWarps; ++w)
          energy += A.part[(static_cast<long long>(b) * kMaxTilesPerScene + t) * kPartSlots +
                           2 * kPartWarps + w];
      for (int t = 0; t < A.nb; ++t) {
        const double* p2 = A.part2 + (static_cast<long long>(b) * kMaxTilesPerScene + t) * kPartSlots;
        gs += p2[0];
        dn += p2[1 * kPartWarps];
        mn += p2[2 * kPartWarps];
      }
      const float fl = A.floor_[b];
      float nv = A.noise[b];
      if (A.fixed_noise > 0.f) {
        nv = A.fixed_noise;
      } else {
        const float en = static_cast<float>(energy);
        float cand = A.evidence ? (en + A.noise_rate) / fmaxf(M - dofv + A.noise_shape, kEps)
                                : (en + nv * dofv + A.noise_rate) / (M + A.noise_shape);
        cand = fmaxf(cand, fl);
        nv = A.keep * nv + (1.0f - A.keep) * cand;
      }
      A.noise[b] = nv;
      A.gsum[b] = static_cast<float>(gs);
      const float den = fmaxf(static_cast<float>(sqrt(mn)), kEps);
      const float ch = static_cast<float>(sqrt(dn)) / den;
      A.change[b] = ch;
      cmax = fmax(cmax, static_cast<double>(ch));
    }
    nsum += A.noise[b];
    dsum += dofv;
  }
  if (!A.hist) return;
  // block max / sums (fixed order)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
  if (lane == 0) red[warp] = cmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (blockDim.x >> 5); ++w) cmax = fmax(cmax, red[w]);
  }
  __syncthreads();
  const double ns = block_sum(nsum, red);
  const double ds = block_sum(dsum, red);
  if (threadIdx.x == 0) {
    A.hist[0] = static_cast<float>(cmax);
    A.hist[1] = static_cast<float>(ns / A.s.B);
    A.hist[2] = static_cast<float>(ds / A.s.B);
    A.hist[3] = static_cast<float>(A.cg_iters_dev ? *A.cg_iters_dev : A.cg_iters);
    A.hist[4] = static_cast<float>(A.probes);
    A.hist[5] = A.cg_tol;
  }
}

// ---------------------------------------------------------------------------
// small layout kernels
// ---------------------------------------------------------------------------

// probes (+-1 floats [B][P][M]) -> complex64
__global__ void cg_probe_kernel(long long total, const float* probes, float2* pz) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    pz[i] = make_float2(probes[i], 0.f);
}

// rhs[b][0] = y[b], rhs[b][j] = probe j-1 of scene b (j < R)
__global__ void cg_rhs_kernel(BatchShape s, int R, int P, const float2* y, const float2* pz,
                              float2* rhs) {
  const long long M = s.m();
  const long long total = static_cast<long long>(s.B) * R * M;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long unit = i / M, m = i % M;
    const int b = static_cast<int>(unit / R), j = static_cast<int>(unit % R);
    rhs[i] = j == 0 ? y[b * M + m] : pz[(static_cast<long long>(b) * P + j - 1) * M + m];
  }
}

// warm start resized from R_old to R_new right-hand sides (solver.py:6121-6138)
__global__ void cg_resize_kernel(BatchShape s, int r_old, int r_new, const float2* src, float2* dst) {
  const long long M = s.m();
  const long long total = static_cast<long long>(s.B) * r_new * M;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long unit = i / M, m = i % M;
    const int b = static_cast<int>(unit / r_new), j = static_cast<int>(unit % r_new);
    dst[i] = j < r_old ? src[(static_cast<long long>(b) * r_old + j) * M + m] : make_float2(0.f, 0.f);
  }
}

// precision = 1 / prior, x = mean, support mask |x|^2 / max(v, tiny) > thr
// (solver.py:2081-2126)
__global__ void cg_output_kernel(long long total, const float* gamma, const float2* mean, float* prec,
                                 float2* x, const float* pv, uint8_t* mask, float thr) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 mu = mean[i];
    if (prec) prec[i] = 1.0f / gamma[i];
    if (x) x[i] = mu;
    if (mask) mask[i] = (abs_sq(mu) / fmaxf(pv[i], kTiny)) > thr ? 1 : 0;
  }
}

static int grid_for(long long total, int threads = 256) {
  const long long b = (total + threads - 1) / threads;
  const long long cap = static_cast<long long>(sm_count()) * 16;
  return static_cast<int>(b < 1 ? 1 : (b > cap ? cap : b));
}

cudaError_t set_cg_attributes() {
  cudaError_t e;
  if ((e = set_attr_both<ProPlain, EpiStoreT>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProDirection, EpiStoreT>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiGamma>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiCurv>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiResid>()) != cudaSuccess) return e;
  if ((e = set_attr_both<ProPlain, EpiEnergy>()) != cudaSuccess) return e;
  const int vec_smem = (kCgSlice * kFsLd + kCgChunk * kCgSlice) * static_cast<int>(sizeof(float2));
  if ((e = cudaFuncSetAttribute(cg_vector_kernel<true, true, false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, vec_smem)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(cg_vector_kernel<false, true, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, vec_smem)) != cudaSuccess)
    return e;
  return cudaSuccess;
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct CgSettings {
  int terms;            // split-BF16 products of the DFT stages (3 or 6)
  int rank;             // preconditioner rank K
  int fixed_iterations; // > 0: static PCG schedule with best-checkpoint tracking
  int max_cg_iter;
  int check_interval;
  float jitter;         // Cholesky loading multiplier
};

// Device buffers of a cg plan, carved from the caller's workspace.
struct CgBuffers {
  static constexpr int kSlots = 38;
  float2* bp;
  float* gamma;
  Scalars scal;
  double *part, *part2;
  int* status;
  float2 *pz, *lp;
  float2 *rhs, *x, *r, *z, *q, *d[2], *best;
  float2 *t1, *wide, *t2;
  float2 *mean, *prev;
  float* relc;
  double* cpart;
  float2* ppart;
  double* dpart;
  float2 *wts, *sinv, *atoms;
  float* bg;
  long long* pidx;
  float* pval;
  uint8_t* topk;
  double* rho;
  float *beta, *init_norm, *rel, *best_rel;
  int *dmask, *active, *valid, *improved;
  int* any_active;
  float* hist;
  float *gsum, *dof, *change;
  static size_t layout(const BatchShape& s, int pmax, int rank, int max_iter, size_t* offs);
  void bind(const BatchShape& s, int pmax, int rank, int max_iter, uint8_t* w);
};

class CgEngine {
 public:
  CgEngine(const BatchShape& shape, const CgSettings& cfg, const DftTables& tabs, const float2* dir1,
           const float2* dir2, const CgBuffers& buffers);
  CgArgs args(int R, float tol) const;
  void matvec(int R, const float2* v, bool direction, float2* out, bool residual, cudaStream_t st);
  void precond_build(cudaStream_t st);
  void precondition(const CgArgs& A, cudaStream_t st);
  dim3 vec_grid(int R) const;
  int pcg(int R, float tol, bool warm, cudaStream_t st);
  ~CgEngine();
  // operator inputs of the next matvec / PCG solve
  const float* prior = nullptr;
  const float* noise = nullptr;
  int* host_flag = nullptr;  // pinned int for the restart test
  // Graph-resident PCG loop: the restart test runs on the device and a
  // graph WHILE node repeats chunks of check_interval iterations while any
  // right-hand side is active (an IF node runs the rest up to max_cg_iter);
  // pcg() then returns -1 and the iteration count stays in it_dev.
  bool graph_loop = false;
  float* tol_dev = nullptr;
  int* it_dev = nullptr;
  void pcg_iteration(int R, float tol, bool check, cudaStream_t st);
  cudaGraphExec_t loop_graph(int R);
  std::map<int, cudaGraphExec_t> loops;
  bool dev_tol = false;  // args() hands the kernels tol_dev
  BatchShape s;
  CgSettings c;
  DftTables t;
  const float2 *d1, *d2;
  CgBuffers buf;
  int nblk = 1;
  int rank = 0;
  int dcur = 0;
};

__global__ void cg_rank0_kernel(int B, const float* noise, const float* gsum, float* bg) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < B) bg[b] = noise[b] + gsum[b];
}

size_t CgBuffers::layout(const BatchShape& s, int pmax, int rank, int max_iter, size_t* offs) {
  size_t off = 0;
  int i = 0;
  auto take = [&](size_t bytes) {
    offs[i++] = off;
    off = (off + bytes + 255) & ~static_cast<size_t>(255);
  };
  const size_t B = s.B, N = s.n(), M = s.m();
  const size_t R = 1 + pmax, U = B * R;
  const size_t K = rank > 0 ? rank : 1;
  const size_t nblk = (M + kCgSlice - 1) / kCgSlice;
  take(B * N * sizeof(float2));              // 0 bp
  take(B * N * sizeof(float));               // 1 gamma
  take(10 * B * sizeof(float));              // 2 scalars
  take(B * kMaxTilesPerScene * kPartSlots * sizeof(double));  // 3 part
  take(B * kMaxTilesPerScene * kPartSlots * sizeof(double));  // 4 part2
  take(B * sizeof(int));                     // 5 status
  take(B * pmax * M * sizeof(float2) + 16);  // 6 pz
  take(B * pmax * N * sizeof(float2) + 16);  // 7 lp
  for (int v = 0; v < 8; ++v) take(U * M * sizeof(float2));  // 8..15 rhs x r z q d0 d1 best
  take(U * static_cast<size_t>(s.n2) * s.m1 * sizeof(float2));  // 16 t1
  take(U * N * sizeof(float2));              // 17 wide (prior-scaled / lifted)
  take(U * static_cast<size_t>(s.m2) * s.n1 * sizeof(float2));  // 18 t2
  take(B * N * sizeof(float2));              // 19 mean
  take(B * N * sizeof(float2));              // 20 prev
  take(B * N * sizeof(float));               // 21 relc
  take(U * kMaxTilesPerScene * kPartSlots * sizeof(double));  // 22 cpart
  take(B * nblk * R * K * sizeof(float2));   // 23 ppart
  take(B * nblk * R * kDSlots * sizeof(double));  // 24 dpart
  take(U * K * sizeof(float2));              // 25 w
  take(B * K * K * sizeof(float2));          // 26 sinv
  take(B * sizeof(float));                   // 27 bg
  take(B * K * sizeof(long long));           // 28 pidx
  take(B * K * sizeof(float));               // 29 pval
  take(topk_scratch_bytes(static_cast<long long>(N), static_cast<int>(K), s.B));  // 30 topk
  take(U * sizeof(double));                  // 31 rho
  take(6 * U * sizeof(float));               // 32 beta init_norm rel best_rel
  take(4 * U * sizeof(int));                 // 33 dmask active valid improved
  take(sizeof(int) * 4);                     // 34 any_active
  take(static_cast<size_t>(max_iter > 0 ? max_iter : 1) * 6 * sizeof(float));  // 35 history
  take(3 * B * sizeof(float));               // 36 gsum dof change
  take(B * M * kCgRankMax * sizeof(float2)); // 37 preconditioner atoms
  return off;
}

void CgBuffers::bind(const BatchShape& s, int pmax, int rank, int max_iter, uint8_t* w) {
  size_t o[kSlots];
  layout(s, pmax, rank, max_iter, o);
  const int B = s.B;
  const size_t U = static_cast<size_t>(B) * (1 + pmax);
  bp = reinterpret_cast<float2*>(w + o[0]);
  gamma = reinterpret_cast<float*>(w + o[1]);
  float* sc = reinterpret_cast<float*>(w + o[2]);
  scal = Scalars{sc, sc + B, sc + 2 * B, sc + 3 * B, sc + 4 * B,
                 sc + 5 * B, sc + 6 * B, sc + 7 * B, sc + 8 * B, sc + 9 * B};
  part = reinterpret_cast<double*>(w + o[3]);
  part2 = reinterpret_cast<double*>(w + o[4]);
  status = reinterpret_cast<int*>(w + o[5]);
  pz = reinterpret_cast<float2*>(w + o[6]);
  lp = reinterpret_cast<float2*>(w + o[7]);
  rhs = reinterpret_cast<float2*>(w + o[8]);
  x = reinterpret_cast<float2*>(w + o[9]);
  r = reinterpret_cast<float2*>(w + o[10]);
  z = reinterpret_cast<float2*>(w + o[11]);
  q = reinterpret_cast<float2*>(w + o[12]);
  d[0] = reinterpret_cast<float2*>(w + o[13]);
  d[1] = reinterpret_cast<float2*>(w + o[14]);
  best = reinterpret_cast<float2*>(w + o[15]);
  t1 = reinterpret_cast<float2*>(w + o[16]);
  wide = reinterpret_cast<float2*>(w + o[17]);
  t2 = reinterpret_cast<float2*>(w + o[18]);
  mean = reinterpret_cast<float2*>(w + o[19]);
  prev = reinterpret_cast<float2*>(w + o[20]);
  relc = reinterpret_cast<float*>(w + o[21]);
  cpart = reinterpret_cast<double*>(w + o[22]);
  ppart = reinterpret_cast<float2*>(w + o[23]);
  dpart = reinterpret_cast<double*>(w + o[24]);
  wts = reinterpret_cast<float2*>(w + o[25]);
  sinv = reinterpret_cast<float2*>(w + o[26]);
  bg = reinterpret_cast<float*>(w + o[27]);
  pidx = reinterpret_cast<long long*>(w + o[28]);
  pval = reinterpret_cast<float*>(w + o[29]);
  topk = w + o[30];
  rho = reinterpret_cast<double*>(w + o[31]);
  float* f = reinterpret_cast<float*>(w + o[32]);
  beta = f;
  init_norm = f + U;
  rel = f + 2 * U;
  best_rel = f + 3 * U;
  int* iv = reinterpret_cast<int*>(w + o[33]);
  dmask = iv;
  active = iv + U;
  valid = iv + 2 * U;
  improved = iv + 3 * U;
  any_active = reinterpret_cast<int*>(w + o[34]);
  hist = reinterpret_cast<float*>(w + o[35]);
  float* g3 = reinterpret_cast<float*>(w + o[36]);
  gsum = g3;
  dof = g3 + B;
  change = g3 + 2 * B;
  atoms = reinterpret_cast<float2*>(w + o[37]);
}

CgEngine::CgEngine(const BatchShape& shape, const CgSettings& cfg, const DftTables& tabs,
                   const float2* dir1, const float2* dir2, const CgBuffers& buffers)
    : s(shape), c(cfg), t(tabs), d1(dir1), d2(dir2), buf(buffers) {
  nblk = static_cast<int>((s.m() + kCgSlice - 1) / kCgSlice);
  rank = c.rank;
}

CgArgs CgEngine::args(int R, float tol) const {
  CgArgs A;
  A.s = s;
  A.R = R;
  A.K = rank;
  A.nblk = nblk;
  A.rhs = buf.rhs;
  A.x = buf.x;
  A.r = buf.r;
  A.z = buf.z;
  A.q = buf.q;
  A.d = buf.d[dcur];
  A.gamma = prior;
  A.noise = noise;
  A.pidx = buf.pidx;
  A.pval = buf.pval;
  A.bg = buf.bg;
  A.sinv = buf.sinv;
  A.F = buf.atoms;
  A.w = buf.wts;
  A.ppart = buf.ppart;
  A.dpart = buf.dpart;
  A.cpart = buf.cpart;
  const int nt = n_tile_of(c.terms);
  const DftGeom f2 = stage_geom_units(kFwd2, s, t, nt, s.B * R, R);
  A.ctiles = f2.row_tiles * f2.col_tiles;
  A.rho = buf.rho;
  A.beta = buf.beta;
  A.dmask = buf.dmask;
  A.active = buf.active;
  A.valid = buf.valid;
  A.improved = buf.improved;
  A.init_norm = buf.init_norm;
  A.rel = buf.rel;
  A.best_rel = buf.best_rel;
  A.any_active = buf.any_active;
  A.tol = tol;
  A.tol_dev = dev_tol ? tol_dev : nullptr;
  A.fixed = c.fixed_iterations > 0;
  return A;
}

// out = Q v over R right-hand sides per scene.  With `direction`, the
// adjoint-1 prologue first forms d[dcur^1] from z and d[dcur].
void CgEngine::matvec(int R, const float2* v, bool direction, float2* out, bool residual,
                      cudaStream_t st) {
  const int nt = n_tile_of(c.terms);
  const int U = s.B * R;
  const DftGeom a1 = stage_geom_units(kAdj1, s, t, nt, U, R);
  const DftGeom a2 = stage_geom_units(kAdj2, s, t, nt, U, R);
  const DftGeom f1 = stage_geom_units(kFwd1, s, t, nt, U, R);
  const DftGeom f2 = stage_geom_units(kFwd2, s, t, nt, U, R);
  const float2* src = v;
  if (direction) {
    run_stage(c.terms, a1,
              ProDirection{buf.z, buf.d[dcur], buf.d[dcur ^ 1], buf.beta, buf.dmask},
              EpiStoreT{buf.t1}, buf.status, st);
    dcur ^= 1;
    src = buf.d[dcur];
  } else {
    run_stage(c.terms, a1, ProPlain{v}, EpiStoreT{buf.t1}, buf.status, st);
  }
  run_stage(c.terms, a2, ProPlain{buf.t1}, EpiGamma{buf.wide, prior, R}, buf.status, st);
  run_stage(c.terms, f1, ProPlain{buf.wide}, EpiStoreT{buf.t2}, buf.status, st);
  if (residual)
    run_stage(c.terms, f2, ProPlain{buf.t2}, EpiResid{buf.r, buf.rhs, src, noise, R}, buf.status, st);
  else
    run_stage(c.terms, f2, ProPlain{buf.t2}, EpiCurv{out, src, noise, buf.cpart, R, 0.0}, buf.status,
              st);
}

void CgEngine::precond_build(cudaStream_t st) {
  if (rank <= 0) return;
  topk_scores(prior, s.n(), rank, s.B, buf.topk, reinterpret_cast<int64_t*>(buf.pidx), buf.pval, st);
  cg_precond_build_kernel<<<s.B, 32, 0, st>>>(s, rank, c.jitter, buf.pidx, buf.pval, buf.gsum, noise,
                                              d1, d2, buf.bg, buf.sinv, buf.status);
  const long long work = s.m() * kCgRankMax;
  cg_atoms_kernel<<<dim3(static_cast<unsigned>((work + 255) / 256), s.B), 256, 0, st>>>(
      s, rank, buf.pidx, buf.pval, buf.atoms);
}

dim3 CgEngine::vec_grid(int R) const {
  return dim3(nblk, s.B, (R + kCgChunk - 1) / kCgChunk);
}

void CgEngine::precondition(const CgArgs& A, cudaStream_t st) {
  const int units = s.B * A.R;
  if (rank > 0) cg_weights_kernel<<<units, 256, 0, st>>>(A);
  cg_precond_kernel<<<vec_grid(A.R), kCgThreads, 0, st>>>(A);
}

static const int kVecSmem = (kCgSlice * kFsLd + kCgChunk * kCgSlice) * static_cast<int>(sizeof(float2));

// Device side of the graph-resident PCG loop.
__global__ void cg_loop_init_kernel(float* tol_dev, float tol, int* it_dev) {
  *tol_dev = tol;
  *it_dev = 0;
}
// End of a chunk of `chunk` iterations (the last one a restart check):
// repeat while a right-hand side is active and a whole chunk still fits.
__global__ void cg_loop_cond_kernel(cudaGraphConditionalHandle h, const int* any_active, int* it_dev, int chunk,
                                    int limit) {
  const int it = *it_dev + chunk;
  *it_dev = it;
  cudaGraphSetConditional(h, (*any_active && it + chunk <= limit) ? 1u : 0u);
}
// After the chunks: the rest up to the limit, if still active.
__global__ void cg_tail_cond_kernel(cudaGraphConditionalHandle h, const int* any_active, const int* it_dev,
                                    int limit) {
  cudaGraphSetConditional(h, (*any_active && *it_dev < limit) ? 1u : 0u);
}
__global__ void cg_add_kernel(int* it_dev, int n) { *it_dev += n; }

// One PCG iteration (solver.py:5641-5721): the matvec along the direction,
// then either the plain step or, with `check`, the update, the residual
// recomputation and the restart test (any_active set by the finish kernel).
void CgEngine::pcg_iteration(int R, float tol, bool check, cudaStream_t st) {
  const int units = s.B * R;
  const int fin_blocks = (units + 7) / 8;
  matvec(R, nullptr, true, buf.q, false, st);
  CgArgs A = args(R, tol);
  if (!check) {
    cg_vector_kernel<true, true, false><<<vec_grid(R), kCgThreads, kVecSmem, st>>>(A);
    precondition(A, st);
    cg_finish_kernel<<<fin_blocks, 256, 0, st>>>(A, kFinishStep);
    return;
  }
  cg_vector_kernel<true, false, false><<<vec_grid(R), kCgThreads, 0, st>>>(A);
  matvec(R, buf.x, false, nullptr, true, st);
  A = args(R, tol);
  cudaMemsetAsync(buf.any_active, 0, sizeof(int), st);
  cg_vector_kernel<false, true, true><<<vec_grid(R), kCgThreads, kVecSmem, st>>>(A);
  precondition(A, st);
  cg_finish_kernel<<<fin_blocks, 256, 0, st>>>(A, kFinishRestart);
  if (c.fixed_iterations > 0) {
    const long long UM = static_cast<long long>(s.B) * R * s.m();
    cg_best_kernel<<<grid_for(UM), 256, 0, st>>>(s, R, buf.improved, buf.x, buf.best);
  }
}

// The loop of pcg() as a CUDA graph, for R right-hand sides: a WHILE node
// over chunks of check_interval iterations whose last kernel sets the
// condition from the device's restart test, then an IF node with the
// remaining max_cg_iter % check_interval iterations.  The tolerance is read
// from tol_dev, the count left in it_dev.  Chunks of an even length end on
// the direction buffer they started on.  nullptr if the graph cannot be
// built (the host loop runs instead).
cudaGraphExec_t CgEngine::loop_graph(int R) {
  auto found = loops.find(R);
  if (found != loops.end()) return found->second;
  const int interval = c.check_interval, limit = c.max_cg_iter, tail = limit % interval;
  cudaGraph_t g = nullptr;
  cudaStream_t cs = nullptr;
  cudaGraphExec_t exec = nullptr;
  const int saved = dcur;
  const bool saved_dev = dev_tol;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
            cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
  cudaGraphConditionalHandle hw{};
  cudaGraphNodeParams wp{};
  cudaGraphNode_t wn{};
  if (ok) {
    ok = cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    ok = ok && cudaGraphAddNode(&wn, g, nullptr, 0, &wp) == cudaSuccess;
  }
  dev_tol = true;
  if (ok) {
    ok = cudaStreamBeginCaptureToGraph(cs, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeRelaxed) == cudaSuccess;
    if (ok) {
      dcur = 0;
      for (int j = 1; j <= interval; ++j) pcg_iteration(R, 0.f, j == interval, cs);
      cg_loop_cond_kernel<<<1, 1, 0, cs>>>(hw, buf.any_active, it_dev, interval, limit);
      cudaGraph_t body = nullptr;
      ok = cudaStreamEndCapture(cs, &body) == cudaSuccess;
    }
  }
  if (ok && tail > 0) {
    cudaGraphConditionalHandle hi{};
    ok = cudaGraphConditionalHandleCreate(&hi, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
    const int* aa = buf.any_active;
    const int* itp = it_dev;
    int lim = limit;
    void* kargs[] = {&hi, &aa, &itp, &lim};
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void*>(cg_tail_cond_kernel);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.sharedMemBytes = 0;
    kp.kernelParams = kargs;
    cudaGraphNode_t kn{};
    ok = ok && cudaGraphAddKernelNode(&kn, g, &wn, 1, &kp) == cudaSuccess;
    cudaGraphNodeParams ip{};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hi;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t in{};
    ok = ok && cudaGraphAddNode(&in, g, &kn, 1, &ip) == cudaSuccess;
    ok = ok && cudaStreamBeginCaptureToGraph(cs, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeRelaxed) == cudaSuccess;
    if (ok) {
      dcur = 0;
      for (int j = 1; j <= tail; ++j) pcg_iteration(R, 0.f, j == tail, cs);
      cg_add_kernel<<<1, 1, 0, cs>>>(it_dev, tail);
      cudaGraph_t body = nullptr;
      ok = cudaStreamEndCapture(cs, &body) == cudaSuccess;
    }
  }
  dcur = saved;
  dev_tol = saved_dev;
  if (ok) ok = cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (cs) cudaStreamDestroy(cs);
  if (!ok) {
    cudaGetLastError();  // the host loop runs instead
    graph_loop = false;
    return nullptr;
  }
  loops[R] = exec;
  return exec;
}

CgEngine::~CgEngine() {
  for (auto& kv : loops)
    if (kv.second) cudaGraphExecDestroy(kv.second);
}

// One PCG solve over the R right-hand sides in buf.rhs (solver.py:5582-5723).
// Returns the iteration count of the loop, or -1 when the loop ran as the
// graph-resident loop (the count is then in it_dev).
int CgEngine::pcg(int R, float tol, bool warm, cudaStream_t st) {
  const long long UM = static_cast<long long>(s.B) * R * s.m();
  const int units = s.B * R;
  const int fin_blocks = (units + 7) / 8;
  CgArgs A = args(R, tol);
  if (rank <= 0)  // rank 0: the background alone, b = noise + sum(prior) (solver.py:5794-5801)
    cg_rank0_kernel<<<(s.B + 127) / 128, 128, 0, st>>>(s.B, noise, buf.gsum, buf.bg);
  if (warm) {
    matvec(R, buf.x, false, nullptr, true, st);
  } else {
    cudaMemsetAsync(buf.x, 0, UM * sizeof(float2), st);
    cudaMemcpyAsync(buf.r, buf.rhs, UM * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  }
  A = args(R, tol);
  cg_vector_kernel<false, true, true><<<vec_grid(R), kCgThreads, kVecSmem, st>>>(A);
  precondition(A, st);
  cg_finish_kernel<<<fin_blocks, 256, 0, st>>>(A, kFinishInit);
  const bool fixed = c.fixed_iterations > 0;
  if (fixed)
    cudaMemcpyAsync(buf.best, buf.x, UM * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  const int limit = fixed ? c.fixed_iterations : c.max_cg_iter;
  if (graph_loop && !fixed && c.check_interval % 2 == 0 && limit >= c.check_interval) {
    cudaGraphExec_t exec = loop_graph(R);
    if (exec) {
      cg_loop_init_kernel<<<1, 1, 0, st>>>(tol_dev, tol, it_dev);
      dcur = 0;
      cudaGraphLaunch(exec, st);
      dcur = 0;  // a finished loop's direction buffer is never read (beta = 0 at the next start)
      return -1;
    }
  }
  int it = 0;
  for (it = 1; it <= limit; ++it) {
    const bool check = (it % c.check_interval == 0) || it == limit;
    pcg_iteration(R, tol, check, st);
    if (check && !fixed) {
      cudaMemcpyAsync(host_flag, buf.any_active, sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      if (!*host_flag) break;
    }
  }
  if (it > limit) it = limit;
  if (fixed)
    cudaMemcpyAsync(buf.x, buf.best, UM * sizeof(float2), cudaMemcpyDeviceToDevice, st);
  return it;
}

// ---------------------------------------------------------------------------
// EM driver (fast_sbl mode="cg")
// ---------------------------------------------------------------------------

// Probe count and PCG tolerance of EM iteration `it` (solver.py:6086-6118).
static void cg_schedule(const FbmeCgConfig& c, int it, int* count, float* tol) {
  const int pmax = c.probes;
  if (!c.adaptive_cg) {
    *count = pmax;
    *tol = c.cg_tolerance;
    return;
  }
  const int initial = c.adaptive_probes ? std::min(c.initial_probes, pmax) : pmax;
  if (it <= 5) {
    *count = initial;
    *tol = std::max(c.cg_initial_tolerance, c.cg_tolerance);
    return;
  }
  if (it <= 15) {
    *count = c.adaptive_probes ? std::min(pmax, std::max(initial, std::min(24, pmax))) : pmax;
    *tol = static_cast<float>(std::max(static_cast<double>(c.cg_tolerance),
                                       std::sqrt(static_cast<double>(c.cg_initial_tolerance) *
                                                 c.cg_tolerance)));
    return;
  }
  *count = pmax;
  *tol = c.cg_tolerance;
}

// sum of the prior variances per scene (fbme_pcg_solve's preconditioner)
__global__ void __launch_bounds__(256) cg_gsum_kernel(long long n, const float* prior, float* gsum) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  double acc = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) acc += prior[b * n + i];
  const double v = block_sum(acc, red);
  if (threadIdx.x == 0) gsum[b] = static_cast<float>(v);
}

}  // namespace fbme

struct FbmeCgPlan {
  fbme::BatchShape s;
  FbmeCgConfig cfg;
  fbme::DevConfig dc;
  fbme::DftTables tables;
  float2 *dir1, *dir2;
  fbme::CgBuffers buf;
  fbme::DenseBufs dense{};  // mode="dense" buffers (cfg.dense)
  fbme::ActiveBufs act{};  // active-set switch (single-scene plans with active_set_start > 0)
  int act_kmax = 0;        // 0: the switch is off
  fbme::CgEngine* eng = nullptr;
  int* host = nullptr;  // pinned: [0] restart flag, [4] change, [8] active-set size
  ~FbmeCgPlan() {
    delete eng;
    if (host) cudaFreeHost(host);
  }
};

namespace {

using fbme::api_fail;

size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct CgLayout {
  size_t tab_f2, tab_a2, tab_f1, tab_a1, dir1, dir2, buffers, active, dense, total;
};

// Size of the active set the switch may select (0: the switch is off).
int active_kmax(const fbme::BatchShape& s, const FbmeCgConfig& c) {
  if (c.dense || c.active_set_start <= 0 || s.B != 1) return 0;
  return static_cast<int>(std::min<long long>(c.active_set_max_size, s.n()));
}

CgLayout cg_layout(const fbme::BatchShape& s, const FbmeCgConfig& c) {
  CgLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align256(off + bytes);
    return o;
  };
  L.tab_f2 = take(fbme::dft_table_bytes(s.n2, c.dft_terms));
  L.tab_a2 = take(fbme::dft_table_bytes(s.n2, c.dft_terms));
  if (s.n1 != s.n2) {
    L.tab_f1 = take(fbme::dft_table_bytes(s.n1, c.dft_terms));
    L.tab_a1 = take(fbme::dft_table_bytes(s.n1, c.dft_terms));
  } else {
    L.tab_f1 = L.tab_f2;
    L.tab_a1 = L.tab_a2;
  }
  L.dir1 = take(s.n1 * sizeof(float2));
  L.dir2 = take(s.n2 * sizeof(float2));
  size_t offs[fbme::CgBuffers::kSlots];
  const int rank = std::min<long long>(c.preconditioner_rank, std::min(s.m(), s.n()));
  L.buffers = take(fbme::CgBuffers::layout(s, c.probes, rank, c.max_iter, offs));
  const int kmax = active_kmax(s, c);
  L.active = kmax > 0 ? take(fbme::cg_active_bytes(s.n(), kmax)) : 0;
  L.dense = c.dense ? take(fbme::dense_bytes(s)) : 0;
  L.total = off;
  return L;
}

int cg_validate(const FbmeShape* shape, int n, const FbmeCgConfig* c, fbme::BatchShape* out) {
  if (!shape || !c || n < 1) return api_fail(FBME_ERR_INVALID, "shape, config and n_scenes >= 1 are required");
  const FbmeShape s = *shape;
  if (s.n1 < 1 || s.n2 < 1 || s.m1 < 1 || s.m2 < 1 || s.m1 > s.n1 || s.m2 > s.n2)
    return api_fail(FBME_ERR_INVALID, "Each sample dimension must satisfy 0 < M <= N.");
  const long long N = 1LL * s.n1 * s.n2;
  if (c->dft_terms != 3 && c->dft_terms != 6) return api_fail(FBME_ERR_INVALID, "dft_terms must be 3 or 6");
  if (c->max_iter < 1 || c->min_iter < 0) return api_fail(FBME_ERR_INVALID, "max_iter must be positive");
  if (c->dense && 1LL * s.m1 * s.m2 > 4096)
    return api_fail(FBME_ERR_UNSUPPORTED, "dense mode above 4096 samples is not built");
  if (c->probes < 1 && !c->dense) return api_fail(FBME_ERR_INVALID, "CG mode requires Hutchinson probes");
  if (c->probes > 128) return api_fail(FBME_ERR_UNSUPPORTED, "more than 128 Hutchinson probes");
  if (c->initial_probes < 1) return api_fail(FBME_ERR_INVALID, "initial_probes must be positive");
  if (c->preconditioner_rank < 0 || c->preconditioner_rank > 32)
    return api_fail(FBME_ERR_UNSUPPORTED, "preconditioner rank above 32 is not built");
  if (c->cg_max_iter < 1 || c->cg_check_interval < 1 || c->cg_fixed_iterations < 0)
    return api_fail(FBME_ERR_INVALID, "cg_max_iter and cg_check_interval must be positive");
  if (!(c->damping >= 0.f && c->damping < 1.f) || !(c->cg_damping >= 0.f && c->cg_damping < 1.f))
    return api_fail(FBME_ERR_INVALID, "damping values must be in [0, 1)");
  if (c->active_set_start > 0) {
    if (c->active_set_check_interval < 1 || c->active_set_min_size < 1 ||
        c->active_set_max_size < c->active_set_min_size ||
        !(c->active_set_tail_fraction > 0.f && c->active_set_tail_fraction < 1.f))
      return api_fail(FBME_ERR_INVALID,
                      "active set: check interval >= 1, 1 <= min_size <= max_size, tail fraction in (0, 1)");
    if (c->active_set_max_size > fbme::kActiveMax)
      return api_fail(FBME_ERR_UNSUPPORTED, "active_set_max_size above 1024 is not built");
  }
  if (N > 524288 || s.n2 > 512)
    return api_fail(FBME_ERR_UNSUPPORTED, "grids above 524288 points or N2 > 512 are not built");
  if (N * n * (1LL + c->probes) > (1LL << 36)) return api_fail(FBME_ERR_INVALID, "batch too large");
  out->B = n;
  out->n1 = s.n1;
  out->n2 = s.n2;
  out->m1 = s.m1;
  out->m2 = s.m2;
  return FBME_OK;
}

fbme::DevConfig cg_dev_config(const FbmeCgConfig& c) {
  fbme::DevConfig d{};
  d.blend = c.initialization_blend;
  d.init_noise = c.initial_noise_fraction;
  d.fixed_noise = c.fixed_noise_variance;
  d.min_var = c.min_variance;
  d.max_prec = c.max_precision;
  d.hyper_shape = c.hyper_shape;
  d.hyper_rate = c.hyper_rate;
  d.noise_shape = c.noise_shape;
  d.noise_rate = c.noise_rate;
  d.noise_evidence = c.noise_update;
  d.damping = c.damping;
  d.terms = c.dft_terms;
  d.jitter = c.jitter_multiplier;
  return d;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return api_fail(FBME_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FBME_OK;
}

// A^H over `units` transforms of shape s laid out back to back.
void adjoint_units(FbmeCgPlan* P, int units, int status_div, const float2* in, float2* out,
                   cudaStream_t st) {
  using namespace fbme;
  const int nt = n_tile_of(P->cfg.dft_terms);
  const DftGeom a1 = stage_geom_units(kAdj1, P->s, P->tables, nt, units, status_div);
  const DftGeom a2 = stage_geom_units(kAdj2, P->s, P->tables, nt, units, status_div);
  run_stage(P->cfg.dft_terms, a1, ProPlain{in}, EpiStoreT{P->buf.t1}, P->buf.status, st);
  run_stage(P->cfg.dft_terms, a2, ProPlain{P->buf.t1}, EpiStoreT{out}, P->buf.status, st);
}

// Lift the solutions, Hutchinson diagonal, mean, relevance (solver.py:3017-3036).
void lift_and_hutch(FbmeCgPlan* P, int R, int count, float* pv_out, cudaStream_t st) {
  using namespace fbme;
  adjoint_units(P, P->s.B * R, R, P->buf.x, P->buf.wide, st);
  const int nb = ew_blocks_host(P->s.n());
  cg_hutch_kernel<<<dim3(nb, P->s.B), kEwThreads, 0, st>>>(P->s, R, count, P->cfg.probes, P->buf.wide,
                                                           P->buf.lp, P->buf.gamma, P->buf.mean,
                                                           P->buf.relc, pv_out, P->buf.part);
}

int cg_solve(FbmeCgPlan* P, const float2* y, const float* probes, const FbmeCgOutputs* out,
             FbmeCgInfo* info, cudaStream_t st) {
  using namespace fbme;
  const BatchShape& s = P->s;
  const FbmeCgConfig& c = P->cfg;
  CgBuffers& bf = P->buf;
  CgEngine& E = *P->eng;
  const int B = s.B, pmax = c.probes;
  const long long N = s.n(), M = s.m();
  const int nt = n_tile_of(c.dft_terms);
  cudaMemsetAsync(bf.status, 0, B * sizeof(int), st);
  // initialisation shared with the UAMP path
  UampBuffers u{};
  u.y = y;
  u.bp = bf.bp;
  u.tmp = bf.t1;
  u.gamma = bf.gamma;
  u.part = bf.part;
  u.sc = bf.scal;
  u.status = bf.status;
  sbl_init(s, P->tables, P->dc, u, st);
  cudaMemcpyAsync(bf.gsum, bf.scal.dvar, B * sizeof(float), cudaMemcpyDeviceToDevice, st);
  const bool dense = c.dense != 0;
  // probes and their lift A^H z (solver.py:1209-1221)
  if (!dense) {
    cg_probe_kernel<<<grid_for(1LL * B * pmax * M), 256, 0, st>>>(1LL * B * pmax * M, probes, bf.pz);
    adjoint_units(P, B * pmax, pmax, bf.pz, bf.lp, st);
  }
  cudaMemsetAsync(bf.prev, 0, B * N * sizeof(float2), st);
  E.prior = bf.gamma;
  E.noise = bf.scal.noise;
  E.dcur = 0;
  // the PCG restart test runs on the device (graph-resident loop) where the
  // schedule allows: no fixed-iteration checkpointing, an even check interval
  E.graph_loop = c.cg_fixed_iterations == 0 && c.cg_check_interval % 2 == 0 && c.cg_max_iter >= c.cg_check_interval;
  // mode="dense": damping alone and min_iter as the minimum (solver.py:1287-1293, 1483-1487)
  const int minimum = dense ? c.min_iter : std::max(c.min_iter, c.cg_min_iter);
  const int limit = c.max_iter;
  const bool conv = c.tol > 0.f && minimum < limit;
  const float keep = dense ? c.damping : std::max(c.damping, c.cg_damping);
  const float floor_tol = 3.0f * std::sqrt(1.1920929e-07f);
  const int nb = ew_blocks_host(N);
  const DftGeom f1b = stage_geom_units(kFwd1, s, P->tables, nt, B, 1);
  const DftGeom f2b = stage_geom_units(kFwd2, s, P->tables, nt, B, 1);
  int R_cur = 0;
  bool warm = false;
  int streak = 0, converged = 0, it = 0, last_cg = 0;
  // active-set switch (single-scene plans): size and iteration once switched
  int act_size = 0, act_iter = 0;
  ActiveArgs aa{};
  if (P->act_kmax > 0) {
    aa.N = N;
    aa.n1 = s.n1;
    aa.n2 = s.n2;
    aa.nb = nb;
    aa.idx = P->act.idx;
    aa.gamma = bf.gamma;
    aa.bp = bf.bp;
    aa.noise = bf.scal.noise;
    aa.d1 = P->dir1;
    aa.d2 = P->dir2;
    aa.jitter = c.jitter_multiplier;
    aa.E = P->act.E;
    aa.X = P->act.X;
    aa.mean = bf.mean;
    aa.relc = bf.relc;
    aa.pv_out = nullptr;
    aa.part = bf.part;
    aa.status = bf.status;
  }
  std::vector<float> hchange(B);
  auto ensure_rhs = [&](int R) {
    if (R == R_cur) return;
    cg_rhs_kernel<<<grid_for(1LL * B * R * M), 256, 0, st>>>(s, R, pmax, y, bf.pz, bf.rhs);
    if (warm && R_cur > 0) {
      cg_resize_kernel<<<grid_for(1LL * B * R * M), 256, 0, st>>>(s, R_cur, R, bf.x, bf.z);
      cudaMemcpyAsync(bf.x, bf.z, 1LL * B * R * M * sizeof(float2), cudaMemcpyDeviceToDevice, st);
    }
    R_cur = R;
  };
  for (it = 1; it <= limit; ++it) {
    if (P->act_kmax > 0 && act_size == 0 && it >= c.active_set_start &&
        (it - c.active_set_start) % c.active_set_check_interval == 0) {
      // _select_active_indices on the current prior (solver.py:1316-1341);
      // the host reads the outcome, as the reference does
      cg_active_select(bf.gamma, N, P->act_kmax, c.active_set_min_size, c.active_set_tail_fraction, P->act, st);
      cudaMemcpyAsync(P->host + 8, P->act.sel, sizeof(int), cudaMemcpyDeviceToHost, st);
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return api_fail(FBME_ERR_CUDA, std::string("cg_solve: ") + cudaGetErrorString(e));
      if (P->host[8] > 0) {
        act_size = P->host[8];
        act_iter = it;
        aa.K = act_size;
        cg_active_mask(P->act, N, P->act_kmax, st);
      }
    }
    int count = pmax;
    float tolcg = c.cg_tolerance;
    cg_schedule(c, it, &count, &tolcg);
    tolcg = std::max(tolcg, floor_tol);
    if (dense) {
      dense_posterior(s, P->dense, bf.gamma, bf.scal.noise, y, c.jitter_multiplier, bf.mean, bf.relc, nullptr,
                      bf.part, nb, bf.status, st);
      last_cg = 0;
      count = 0;
    } else if (act_size > 0) {
      // exact reduced posterior on the active set: no PCG, no probes
      cg_active_posterior(aa, st);
      last_cg = 0;
      count = 0;
    } else {
      ensure_rhs(1 + count);
      const int R = R_cur;
      E.precond_build(st);
      last_cg = E.pcg(R, tolcg, warm, st);
      warm = c.warm_start != 0;
      lift_and_hutch(P, R, count, nullptr, st);
    }
    if (!dense) {  // residual energy (dense mode: from Q^-1 y, in dense_posterior)
      run_stage(c.dft_terms, f1b, ProPlain{bf.mean}, EpiStoreT{bf.t2}, bf.status, st);
      run_stage(c.dft_terms, f2b, ProPlain{bf.t2}, EpiEnergy{y, bf.part, 0.0}, bf.status, st);
    }
    CgEmArgs em;
    em.s = s;
    em.nb = nb;
    em.part = bf.part;
    em.part2 = bf.part2;
    em.mean = bf.mean;
    em.prev = bf.prev;
    em.relc = bf.relc;
    em.gamma = bf.gamma;
    em.floor_ = bf.scal.floor_;
    em.keep = keep;
    em.hyper_shape = c.hyper_shape;
    em.hyper_rate = c.hyper_rate;
    em.max_prec = c.max_precision;
    em.amask = act_size > 0 ? P->act.mask : nullptr;
    CgScalarArgs sa;
    sa.s = s;
    sa.nb = nb;
    sa.etiles = dense ? 1 : f2b.row_tiles * f2b.col_tiles;
    sa.part = bf.part;
    sa.part2 = bf.part2;
    sa.noise = bf.scal.noise;
    sa.floor_ = bf.scal.floor_;
    sa.gsum = bf.gsum;
    sa.dof = bf.dof;
    sa.change = bf.change;
    sa.hist = bf.hist + static_cast<long long>(it - 1) * 6;
    sa.keep = keep;
    sa.fixed_noise = c.fixed_noise_variance;
    sa.noise_shape = c.noise_shape;
    sa.noise_rate = c.noise_rate;
    sa.evidence = c.noise_update;
    sa.cg_iters = last_cg > 0 ? last_cg : 0;
    sa.cg_iters_dev = last_cg < 0 ? E.it_dev : nullptr;
    sa.probes = count;
    sa.cg_tol = tolcg;
    sa.update = 1;
    cg_em_kernel<<<dim3(nb, B), kEwThreads, 0, st>>>(em);
    cg_scalars_kernel<<<1, 256, 0, st>>>(sa);
    const bool should_check =
        conv && it >= minimum && ((it - minimum) % c.convergence_check_interval == 0 || it == limit);
    if (should_check) {
      cudaMemcpyAsync(P->host + 4, bf.hist + static_cast<long long>(it - 1) * 6, sizeof(float),
                      cudaMemcpyDeviceToHost, st);
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return api_fail(FBME_ERR_CUDA, std::string("cg_solve: ") + cudaGetErrorString(e));
      float ch;
      std::memcpy(&ch, P->host + 4, sizeof(float));
      streak = ch <= c.tol ? streak + 1 : 0;
      if (streak >= c.convergence_patience) {
        converged = 1;
        break;
      }
    }
  }
  const int iterations = it > limit ? limit : it;
  // final posterior: every probe, or the reduced posterior after a switch
  // (solver.py:2023-2080)
  if (dense) {
    dense_posterior(s, P->dense, bf.gamma, bf.scal.noise, y, c.jitter_multiplier, bf.mean, bf.relc,
                    out->posterior_variance, bf.part, nb, bf.status, st);
  } else if (act_size > 0) {
    aa.pv_out = out->posterior_variance;
    cg_active_posterior(aa, st);
  } else {
    ensure_rhs(1 + pmax);
    E.precond_build(st);
    E.pcg(R_cur, std::max(c.cg_tolerance, floor_tol), warm, st);
    lift_and_hutch(P, R_cur, pmax, out->posterior_variance, st);
  }
  {
    CgScalarArgs sa{};
    sa.s = s;
    sa.nb = nb;
    sa.part = bf.part;
    sa.part2 = bf.part2;
    sa.noise = bf.scal.noise;
    sa.floor_ = bf.scal.floor_;
    sa.gsum = bf.gsum;
    sa.dof = bf.dof;
    sa.change = bf.change;
    sa.hist = nullptr;
    sa.update = 0;
    cg_scalars_kernel<<<1, 256, 0, st>>>(sa);
  }
  cg_output_kernel<<<grid_for(1LL * B * N), 256, 0, st>>>(
      1LL * B * N, bf.gamma, bf.mean, out->precision, static_cast<float2*>(out->x),
      out->posterior_variance, out->support_mask, out->support_threshold);
  if (out->noise_variance)
    cudaMemcpyAsync(out->noise_variance, bf.scal.noise, B * sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (out->effective_dof)
    cudaMemcpyAsync(out->effective_dof, bf.dof, B * sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (out->status)
    cudaMemcpyAsync(out->status, bf.status, B * sizeof(int), cudaMemcpyDeviceToDevice, st);
  std::vector<float> hist(static_cast<size_t>(iterations) * 6);
  cudaMemcpyAsync(hist.data(), bf.hist, hist.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return api_fail(FBME_ERR_CUDA, std::string("cg_solve: ") + cudaGetErrorString(e));
  if (info) {
    info->iterations = iterations;
    info->converged = converged;
    info->relative_change = hist[static_cast<size_t>(iterations - 1) * 6];
    info->last_cg_iterations = last_cg >= 0 ? last_cg : static_cast<int>(hist[static_cast<size_t>(iterations - 1) * 6 + 3]);
    info->active_set_size = act_size;
    info->active_set_iteration = act_iter;
    if (info->history) std::memcpy(info->history, hist.data(), hist.size() * sizeof(float));
  }
  return check_launch("cg_solve");
}

}  // namespace

extern "C" {

size_t fbme_cg_workspace_bytes(const FbmeShape* shape, int32_t n_scenes, const FbmeCgConfig* cfg) {
  fbme::BatchShape s;
  if (cg_validate(shape, n_scenes, cfg, &s) != FBME_OK) return 0;
  return cg_layout(s, *cfg).total;
}

int fbme_cg_create(const FbmeShape* shape, int32_t n_scenes, const FbmeCgConfig* cfg, void* workspace,
                   size_t workspace_bytes, fbme_stream_t stream, FbmeCgPlan** plan) {
  if (!plan) return api_fail(FBME_ERR_INVALID, "plan output pointer is NULL");
  *plan = nullptr;
  fbme::BatchShape s;
  int rc = cg_validate(shape, n_scenes, cfg, &s);
  if (rc != FBME_OK) return rc;
  const CgLayout L = cg_layout(s, *cfg);
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255u) != 0)
    return api_fail(FBME_ERR_WORKSPACE, "workspace must be a 256-byte aligned device pointer");
  if (workspace_bytes < L.total)
    return api_fail(FBME_ERR_WORKSPACE, "workspace smaller than fbme_cg_workspace_bytes()");
  cudaError_t e = fbme::set_dft_attributes();
  if (e == cudaSuccess) e = fbme::set_cg_attributes();
  if (e != cudaSuccess)
    return api_fail(FBME_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  FbmeCgPlan* P = new (std::nothrow) FbmeCgPlan();
  if (!P) return api_fail(FBME_ERR_INVALID, "out of host memory");
  if (cudaMallocHost(&P->host, 64) != cudaSuccess) {
    P->host = nullptr;
    delete P;
    return api_fail(FBME_ERR_CUDA, "cudaMallocHost failed");
  }
  uint8_t* w = static_cast<uint8_t*>(workspace);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  P->s = s;
  P->cfg = *cfg;
  P->dc = cg_dev_config(*cfg);
  const int terms = cfg->dft_terms;
  const int nt = terms == 6 ? 128 : 256, parts = terms == 6 ? 3 : 2;
  auto cdiv = [](long long a, long long b) { return static_cast<int>((a + b - 1) / b); };
  auto build_table = [&](size_t off, int Lx, int sign) {
    fbme::launch_twiddle_table(w + off, Lx, sign, nt, cdiv(2LL * Lx, nt), cdiv(2LL * Lx, 64), parts, st);
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
  P->tables.kchunks_n1 = cdiv(2LL * s.n1, 64);
  P->tables.kchunks_n2 = cdiv(2LL * s.n2, 64);
  P->tables.n_tile = nt;
  P->dir1 = reinterpret_cast<float2*>(w + L.dir1);
  P->dir2 = reinterpret_cast<float2*>(w + L.dir2);
  fbme::launch_dirichlet(P->dir1, s.m1, s.n1, st);
  fbme::launch_dirichlet(P->dir2, s.m2, s.n2, st);
  const int rank = static_cast<int>(std::min<long long>(cfg->preconditioner_rank, std::min(s.m(), s.n())));
  P->buf.bind(s, cfg->probes, rank, cfg->max_iter, w + L.buffers);
  if (cfg->dense) P->dense = fbme::dense_bind(w + L.dense, s, st);
  P->act_kmax = active_kmax(s, *cfg);
  if (P->act_kmax > 0) P->act = fbme::cg_active_bind(w + L.active, s.n(), P->act_kmax);
  fbme::CgSettings cs;
  cs.terms = terms;
  cs.rank = rank;
  cs.fixed_iterations = cfg->cg_fixed_iterations;
  cs.max_cg_iter = cfg->cg_max_iter;
  cs.check_interval = cfg->cg_check_interval;
  cs.jitter = cfg->jitter_multiplier;
  P->eng = new (std::nothrow) fbme::CgEngine(s, cs, P->tables, P->dir1, P->dir2, P->buf);
  if (!P->eng) {
    delete P;
    return api_fail(FBME_ERR_INVALID, "out of host memory");
  }
  P->eng->host_flag = P->host;
  P->eng->it_dev = P->buf.any_active + 1;
  P->eng->tol_dev = reinterpret_cast<float*>(P->buf.any_active + 2);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    delete P;
    return api_fail(FBME_ERR_CUDA, std::string("cg plan tables: ") + cudaGetErrorString(e));
  }
  *plan = P;
  return FBME_OK;
}

int fbme_cg_destroy(FbmeCgPlan* plan) {
  delete plan;
  return FBME_OK;
}

int fbme_cg_solve(FbmeCgPlan* plan, const void* y, const float* probes, const FbmeCgOutputs* out,
                  FbmeCgInfo* info, fbme_stream_t stream) {
  if (!plan || !y || !probes || !out) return api_fail(FBME_ERR_INVALID, "NULL argument");
  if (!out->x || !out->posterior_variance || !out->precision)
    return api_fail(FBME_ERR_INVALID, "x, posterior_variance and precision outputs are required");
  return cg_solve(plan, static_cast<const float2*>(y), probes, out, info,
                  reinterpret_cast<cudaStream_t>(stream));
}

int fbme_cg_matvec(FbmeCgPlan* plan, const float* prior, const float* noise, const void* v,
                   int32_t rhs, void* out, fbme_stream_t stream) {
  if (!plan || !prior || !noise || !v || !out) return api_fail(FBME_ERR_INVALID, "NULL argument");
  if (rhs < 1 || rhs > 1 + plan->cfg.probes)
    return api_fail(FBME_ERR_INVALID, "rhs must be in [1, 1 + probes]");
  fbme::CgEngine& E = *plan->eng;
  E.prior = prior;
  E.noise = noise;
  E.matvec(rhs, static_cast<const float2*>(v), false, static_cast<float2*>(out), false,
           reinterpret_cast<cudaStream_t>(stream));
  return check_launch("fbme_cg_matvec");
}

int fbme_pcg_solve(FbmeCgPlan* plan, const float* prior, const float* noise, const void* rhs,
                   int32_t rhs_count, const void* initial, float tolerance, void* solution,
                   int32_t* iterations, fbme_stream_t stream) {
  if (!plan || !prior || !noise || !rhs || !solution) return api_fail(FBME_ERR_INVALID, "NULL argument");
  if (rhs_count < 1 || rhs_count > 1 + plan->cfg.probes)
    return api_fail(FBME_ERR_INVALID, "rhs_count must be in [1, 1 + probes]");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  fbme::CgEngine& E = *plan->eng;
  fbme::CgBuffers& bf = plan->buf;
  const fbme::BatchShape& s = plan->s;
  const size_t bytes = static_cast<size_t>(s.B) * rhs_count * s.m() * sizeof(float2);
  cudaMemsetAsync(bf.status, 0, s.B * sizeof(int), st);
  cudaMemcpyAsync(bf.rhs, rhs, bytes, cudaMemcpyDeviceToDevice, st);
  if (initial) cudaMemcpyAsync(bf.x, initial, bytes, cudaMemcpyDeviceToDevice, st);
  E.prior = prior;
  E.noise = noise;
  E.dcur = 0;
  fbme::cg_gsum_kernel<<<s.B, 256, 0, st>>>(s.n(), prior, bf.gsum);
  E.precond_build(st);
  const bool graph = E.graph_loop;
  E.graph_loop = false;  // this entry reports the iteration count on the host
  const int it = E.pcg(rhs_count, tolerance, initial != nullptr, st);
  E.graph_loop = graph;
  cudaMemcpyAsync(solution, bf.x, bytes, cudaMemcpyDeviceToDevice, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return api_fail(FBME_ERR_CUDA, std::string("fbme_pcg_solve: ") + cudaGetErrorString(e));
  if (iterations) *iterations = it;
  return check_launch("fbme_pcg_solve");
}

}  // extern "C"
