// Host-side geometry and launch helpers of the tcgen05 DFT stage kernel,
// plus the partial-sum and load helpers shared by the UAMP and PCG
// translation units.
//
// A "unit" is one independent 2-D transform: a scene for the UAMP sweeps,
// a (scene, right-hand side) pair for the PCG matvecs.  Units are laid out
// back to back, so every stage is described by its per-unit strides.
#pragma once

#include "dft_umma.cuh"
#include "kernels.cuh"

namespace fbme {

constexpr float kTiny = 1.17549435e-38f;  // FLT_MIN (torch.finfo(float32).tiny)
constexpr float kEps = 1.1920929e-07f;    // FLT_EPSILON

// ---------------------------------------------------------------------------
// partial-sum helpers
// ---------------------------------------------------------------------------
FBME_DEV double* part_slot(double* part, int unit, int tile, int slot) {
  return part + (static_cast<long long>(unit) * kMaxTilesPerScene + tile) * kPartSlots + slot;
}
FBME_DEV void write_block_partial(double v, double* red, double* part, int unit, int tile,
                                  int slot) {
  const double s = block_sum(v, red);
  if (threadIdx.x == 0) *part_slot(part, unit, tile, slot) = s;
}
// Reduction `sum` of one tile: warp `w` (of the stage's producer or
// epilogue group) writes its warp total to slot sum*kPartWarps + w.
FBME_DEV void warp_partial(double v, double* part, const TileCtx& t, int sum, int w, int lane) {
  v = warp_sum(v);
  if (lane == 0)
    *part_slot(part, t.scene, t.row_tile * t.g->col_tiles + t.col_tile, sum * kPartWarps + w) = v;
}
// Sum of reduction `sum` of one unit over `tiles` tiles x `warps` slots,
// in a fixed order.
FBME_DEV double unit_sum(const double* part, int unit, int sum, int tiles, int warps) {
  double v = 0.0;
  for (int t = 0; t < tiles; ++t)
    for (int w = 0; w < warps; ++w)
      v += part[(static_cast<long long>(unit) * kMaxTilesPerScene + t) * kPartSlots +
                sum * kPartWarps + w];
  return v;
}

FBME_DEV bool vec_ok(const DftGeom& g) { return g.vec4 != 0; }

// Two consecutive complex values at base[e] through the read-only path.
FBME_DEV void load2c(const float2* base, long long e, int avail, bool vec, float2& a, float2& b) {
  if (avail >= 2 && vec) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(base + e));
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
  } else {
    a = __ldg(base + e);
    b = avail >= 2 ? __ldg(base + e + 1) : make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------------------
// elementwise launch shape
// ---------------------------------------------------------------------------
constexpr int kEwThreads = 256;

FBME_DEV int ew_blocks_per_scene(long long n) {
  long long b = (n + 2047) / 2048;
  return static_cast<int>(b < kMaxTilesPerScene ? (b < 1 ? 1 : b) : kMaxTilesPerScene);
}
static inline int ew_blocks_host(long long n) {
  long long b = (n + 2047) / 2048;
  return static_cast<int>(b < kMaxTilesPerScene ? (b < 1 ? 1 : b) : kMaxTilesPerScene);
}

// Partial-sum source of one reduction: tiles x warps per tile.
struct PartSrc {
  int tiles, warps;
};

// ---------------------------------------------------------------------------
// stage geometry
// ---------------------------------------------------------------------------
static inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

static inline DftGeom make_geom(int units, int rows, int kcplx, int cols, int in_ld,
                                long long in_stride, int out_ld, long long out_stride,
                                const uint8_t* table, int table_kchunks, int n_tile,
                                int status_div = 1) {
  DftGeom g;
  g.n_scenes = units;
  g.rows = rows;
  g.row_tiles = ceil_div(rows, kTileRows);
  g.kcplx = kcplx;
  g.kchunks = ceil_div(2LL * kcplx, kKChunk);
  g.cols = cols;
  g.col_tiles = ceil_div(2LL * cols, n_tile);
  g.in_ld = in_ld;
  g.in_stride = in_stride;
  g.out_ld = out_ld;
  g.out_stride = out_stride;
  g.col_per_tile = n_tile / 2;
  g.vec4 = (in_ld % 2 == 0) && (in_stride % 2 == 0);
  g.table = table;
  g.table_kchunks = table_kchunks;
  g.status_div = status_div;
  return g;
}

enum Stage { kFwd1, kFwd2, kAdj1, kAdj2 };

// The four stages of the prefix operator for `units` transforms of shape s
// (s.B is ignored); status words are indexed by unit / status_div.
static inline DftGeom stage_geom_units(Stage st, const BatchShape& s, const DftTables& t,
                                       int n_tile, int units, int status_div) {
  const long long N = s.n(), M = s.m();
  switch (st) {
    case kFwd1:  // [n1][n2] -> [m2][n1], contract n2
      return make_geom(units, s.n1, s.n2, s.m2, s.n2, N, s.n1, 1LL * s.m2 * s.n1, t.fwd_n2,
                       t.kchunks_n2, n_tile, status_div);
    case kFwd2:  // [m2][n1] -> [m1][m2], contract n1
      return make_geom(units, s.m2, s.n1, s.m1, s.n1, 1LL * s.m2 * s.n1, s.m2, M, t.fwd_n1,
                       t.kchunks_n1, n_tile, status_div);
    case kAdj1:  // [m1][m2] -> [n2][m1], contract m2
      return make_geom(units, s.m1, s.m2, s.n2, s.m2, M, s.m1, 1LL * s.n2 * s.m1, t.adj_n2,
                       t.kchunks_n2, n_tile, status_div);
    default:     // [n2][m1] -> [n1][n2], contract m1
      return make_geom(units, s.n2, s.m1, s.n1, s.m1, 1LL * s.n2 * s.m1, s.n2, N, t.adj_n1,
                       t.kchunks_n1, n_tile, status_div);
  }
}
static inline DftGeom stage_geom(Stage st, const BatchShape& s, const DftTables& t, int n_tile) {
  return stage_geom_units(st, s, t, n_tile, s.B, 1);
}

static inline int tiles(const DftGeom& g) { return g.n_scenes * g.row_tiles * g.col_tiles; }

// Default stage tile width (real output columns): 256 for 3-term
// products, 128 for 6 (the 6-term operands fill shared memory sooner).
// Plans may lay their tables out for 64 or 128 columns with 3 terms
// instead (dft_n_tile_ok), which wastes less of a tile on short axes.
static inline int n_tile_of(int terms) { return terms == 6 ? 128 : 256; }

// A tile width a plan of this shape may use: 64, 128 or 256 with 3 terms,
// 128 with 6, and at most kMaxTilesPerScene tiles per scene in every stage.
static inline bool dft_n_tile_ok(int terms, int n_tile, const BatchShape& s) {
  if (terms == 6 ? n_tile != 128 : (n_tile != 64 && n_tile != 128 && n_tile != 256)) return false;
  const long long r[4][2] = {{s.n1, s.m2}, {s.m2, s.m1}, {s.m1, s.n2}, {s.n2, s.n1}};  // rows, cols
  for (const auto& rc : r)
    if (static_cast<long long>(ceil_div(rc[0], kTileRows)) * ceil_div(2 * rc[1], n_tile) > kMaxTilesPerScene)
      return false;
  return true;
}

template <int A_PARTS, int N_TILE, class Pro, class Epi, int NI>
static cudaError_t set_attr() {
  return cudaFuncSetAttribute(dft_stage_kernel<A_PARTS, N_TILE, Pro, Epi, NI>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              DftCfg<A_PARTS, N_TILE>::kSmemBytes);
}

template <int A_PARTS, int N_TILE, class Pro, class Epi, int NI>
static void launch_set(const StageSet<Pro, Epi, NI>& set, cudaStream_t st) {
  const int t = set.tile0[set.n], s = sm_count();
  dft_stage_kernel<A_PARTS, N_TILE, Pro, Epi, NI>
      <<<t < s ? t : s, kDftPersistThreads, DftCfg<A_PARTS, N_TILE>::kSmemBytes, st>>>(set);
}

template <int A_PARTS, int N_TILE, class Pro, class Epi>
static void launch_stage(const DftGeom& g, const Pro& pro, const Epi& epi, int* status, cudaStream_t st) {
  StageSet<Pro, Epi, 1> set;
  set.n = 1;
  set.tile0[0] = 0;
  set.tile0[1] = tiles(g);
  set.it[0] = StageItem<Pro, Epi>{g, pro, epi, status};
  launch_set<A_PARTS, N_TILE>(set, st);
}

// One stage launch; the tile width is the one the geometry was built for.
template <class Pro, class Epi>
static void run_stage(int terms, const DftGeom& g, const Pro& pro, const Epi& epi, int* status,
                      cudaStream_t st) {
  if (terms == 6) {
    launch_stage<3, 128>(g, pro, epi, status, st);
  } else if (g.col_per_tile == 32) {
    launch_stage<2, 64>(g, pro, epi, status, st);
  } else if (g.col_per_tile == 64) {
    launch_stage<2, 128>(g, pro, epi, status, st);
  } else {
    launch_stage<2, 256>(g, pro, epi, status, st);
  }
}

// Stage launches of several shape buckets merged into persistent launches
// of up to kStageSetMax items, one per tile width (and term count).
constexpr int kStageSetMax = 64;

template <class Pro, class Epi>
struct StageJob {
  int terms;
  StageItem<Pro, Epi> item;
};

template <int A_PARTS, int N_TILE, class Pro, class Epi>
static void launch_jobs(const StageJob<Pro, Epi>* jobs, int n, int terms, int col_per_tile,
                        cudaStream_t st) {
  StageSet<Pro, Epi, kStageSetMax> set;
  set.n = 0;
  set.tile0[0] = 0;
  for (int i = 0; i < n; ++i) {
    const StageJob<Pro, Epi>& j = jobs[i];
    if (j.terms != terms || j.item.g.col_per_tile != col_per_tile) continue;
    set.it[set.n] = j.item;
    set.tile0[set.n + 1] = set.tile0[set.n] + tiles(j.item.g);
    if (++set.n == kStageSetMax) {
      launch_set<A_PARTS, N_TILE>(set, st);
      set.n = 0;
    }
  }
  if (set.n > 0) launch_set<A_PARTS, N_TILE>(set, st);
}

template <class Pro, class Epi>
static void run_stage_multi(const StageJob<Pro, Epi>* jobs, int n, cudaStream_t st) {
  bool w6 = false, w64 = false, w128 = false, w256 = false;
  for (int i = 0; i < n; ++i) {
    const int c = jobs[i].item.g.col_per_tile;
    if (jobs[i].terms == 6) w6 = true;
    else if (c == 32) w64 = true;
    else if (c == 64) w128 = true;
    else w256 = true;
  }
  if (w6) launch_jobs<3, 128>(jobs, n, 6, 64, st);
  if (w64) launch_jobs<2, 64>(jobs, n, 3, 32, st);
  if (w128) launch_jobs<2, 128>(jobs, n, 3, 64, st);
  if (w256) launch_jobs<2, 256>(jobs, n, 3, 128, st);
}

template <class Pro, class Epi, bool kMulti = false>
static cudaError_t set_attr_both() {
  cudaError_t e;
  if ((e = set_attr<2, 256, Pro, Epi, 1>()) != cudaSuccess) return e;
  if ((e = set_attr<2, 128, Pro, Epi, 1>()) != cudaSuccess) return e;
  if ((e = set_attr<2, 64, Pro, Epi, 1>()) != cudaSuccess) return e;
  if ((e = set_attr<3, 128, Pro, Epi, 1>()) != cudaSuccess) return e;
  if constexpr (kMulti) {
    if ((e = set_attr<2, 256, Pro, Epi, kStageSetMax>()) != cudaSuccess) return e;
    if ((e = set_attr<2, 128, Pro, Epi, kStageSetMax>()) != cudaSuccess) return e;
    if ((e = set_attr<2, 64, Pro, Epi, kStageSetMax>()) != cudaSuccess) return e;
    if ((e = set_attr<3, 128, Pro, Epi, kStageSetMax>()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace fbme

namespace fbme {
struct DenoiseArgs;
// One FP32 FFT stage (fft.cu) with the geometry of the GEMM stage `g`: a
// length-L transform of sign `sign` per row, input zero-padded from g.kcplx,
// output truncated to g.cols.  Mode 3 (with `dn`) runs the UAMP denoiser on
// the outputs instead of storing them; fft_denoise_fused(L) says whether
// that is built for the length.
void fft_stage(const DftGeom& g, int L, int sign, const float2* tw, const float2* in, float2* out,
               const float2* y, const uint8_t* mask, double* part, int mode, int ysum, cudaStream_t st,
               const DenoiseArgs* dn = nullptr);
int fft_denoise_fused(int L);

// One shape bucket's stage in a merged FFT launch (fft_stage_set): the
// arguments fft_stage takes, per bucket.
struct FftSetJob {
  DftGeom g;
  const float2* tw;
  const float2* in;
  float2* out;
  const float2* y;
  const uint8_t* mask;
  double* part;
  int ysum;
  const DenoiseArgs* dn;  // mode 3
};
// The stages `jobs[0..n)` of one transform length L, sign and mode: in as
// few launches of the two-pass kernel as fit (64 buckets each) where L has
// it (fft_set_length_ok), else one fft_stage launch per bucket; every
// bucket's results and partial sums are those of its own fft_stage launch.
void fft_stage_set(const FftSetJob* jobs, int n, int L, int sign, int mode, cudaStream_t st);
int fft_set_length_ok(int L);
}  // namespace fbme
