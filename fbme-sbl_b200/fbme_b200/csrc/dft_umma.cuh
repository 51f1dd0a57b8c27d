// Prefix-DFT contraction on the 5th-generation tensor cores (tcgen05).
//
// One "DFT stage" contracts the contiguous axis of a batch of complex
// matrices with a DFT submatrix:
//
//     Out[r, c] = sum_k In[r, k] * w^(k*c),   w = exp(sign * 2*pi*i / L)
//
// written as a real GEMM on the interleaved (re, im) view: In is
// [rows, 2K] and the twiddles are expanded into a real [2K, 2C] matrix
// E[2k+a][2c+b] = [[Re w, Im w], [-Im w, Re w]][a][b].  Two stages make the
// 2-D prefix operator A(X) = F_M1 X F_M2^T (forward) and its adjoint.
//
// Precision: both operands are split into BF16 parts (x = hi + lo, or
// hi + mid + lo) and the tensor core accumulates in FP32 the products of
// order <= 1 (3 terms: hi*hi + hi*lo + lo*hi) or <= 2 (6 terms).  The FP32
// accumulation over the contracted axis, not the split, sets the error:
// measured against an FP64 DFT on B200, one 2-D transform is 5-6e-6
// relative L2 with 3 terms at 64^2/32^2 and 256^2/128^2, and 1-6e-6 with
// 6 terms (an FP32 FFT is ~5e-8).
//
// Kernel organisation (one CTA = one 128-row x N_TILE-column output tile):
//   warps 0-3  producer: read In through the prologue policy (fused
//              elementwise work), split to BF16 parts, store into the K-major
//              128-byte-swizzled operand layout; thread 0 bulk-copies the
//              pre-swizzled twiddle blocks for the same K chunk;
//   warp 4     allocates tensor memory; lane 0 issues tcgen05.mma;
//   all warps  epilogue: tcgen05.ld the FP32 accumulator and hand each
//              row's values to the epilogue policy.
// Epilogue stores put the tile row (the TMEM lane) on the contiguous memory
// axis, so a warp's 32 lanes write 32 consecutive elements.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace fbme {

// A prologue policy with `static constexpr bool kBulk = true` supplies its
// operand already split and swizzled: the producer only bulk-copies it.
template <class P, class = void>
struct ProBulk : std::false_type {};
template <class P>
struct ProBulk<P, std::void_t<decltype(P::kBulk)>> : std::bool_constant<P::kBulk> {};

constexpr int kTileRows = 128;  // UMMA M
constexpr int kKChunk = 64;     // real K per pipeline stage (one 128-byte row)
constexpr int kStages = 2;
constexpr int kDftThreads = 256;
constexpr int kPartBytesA = kTileRows * 128;  // 16 KiB

struct DftGeom {
  int n_scenes;
  int rows;                 // data rows per scene
  int row_tiles;            // ceil(rows / 128)
  int kcplx;                // contracted complex length
  int kchunks;              // ceil(2 * kcplx / 64)
  int cols;                 // complex output columns per scene
  int col_tiles;            // ceil(2 * cols / N_TILE)
  int in_ld;                // complex stride between input rows
  long long in_stride;      // complex elements between scenes (input)
  int out_ld;               // complex stride between output columns
  long long out_stride;     // complex elements between scenes (output)
  int col_per_tile;         // complex output columns per tile (N_TILE / 2)
  int vec4;                 // rows start on 16-byte boundaries (even strides)
  const uint8_t* table;     // pre-swizzled twiddle blocks
  int table_kchunks;        // K chunks per column tile in the table
  int status_div;           // status word of a unit: status[unit / status_div]
};

struct TileCtx {
  int scene, row_tile, col_tile;
  const DftGeom* g;
  __device__ int row0() const { return row_tile * kTileRows; }
  __device__ int col0() const { return col_tile * g->col_per_tile; }
};

template <int A_PARTS, int N_TILE>
struct DftCfg {
  static constexpr int kPartBytesB = N_TILE * 128;
  static constexpr int kStageBytes = A_PARTS * kPartBytesA + A_PARTS * kPartBytesB;
  static constexpr int kPairs = A_PARTS == 2 ? 3 : 6;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*bars*/ +
                                    32 * sizeof(double) /*reduction scratch*/;
  static constexpr uint32_t kIdesc = umma_idesc_bf16(kTileRows, N_TILE);
};

// (a-part, b-part) products of order <= 1 (A_PARTS=2) or <= 2 (A_PARTS=3).
__device__ __constant__ int8_t kPairA[6] = {0, 0, 1, 0, 1, 2};
__device__ __constant__ int8_t kPairB[6] = {0, 1, 0, 2, 1, 0};

FBME_DEV uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
FBME_DEV float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// Split four floats into A_PARTS packed bf16 quads (2 x uint32 each):
// part t holds bf16(x - sum of earlier parts); the subtraction is exact.
template <int A_PARTS>
FBME_DEV void split4(const float4 v, uint2* out) {
  float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
#pragma unroll
  for (int t = 0; t < A_PARTS; ++t) {
    const __nv_bfloat162 ha = __float22bfloat162_rn(a), hb = __float22bfloat162_rn(b);
    out[t].x = *reinterpret_cast<const uint32_t*>(&ha);
    out[t].y = *reinterpret_cast<const uint32_t*>(&hb);
    if (t + 1 < A_PARTS) {
      const float2 fa = __bfloat1622float2(ha), fb = __bfloat1622float2(hb);
      a = make_float2(a.x - fa.x, a.y - fa.y);
      b = make_float2(b.x - fb.x, b.y - fb.y);
    }
  }
}

// Persistent, warp-specialised stage kernel.  Each CTA loops over tiles
// (static round-robin); two TMEM accumulators let the epilogue of one tile
// overlap the tensor-core work of the next.
//   warps 0-3, 5-7  producer (224 threads): fetch the operand rows of a K
//               chunk into registers, then wait for the stage to be free,
//               split to BF16 parts and store; thread 0 also bulk-copies
//               the twiddle blocks;
//   warp 4      TMEM allocation; lane 0 issues tcgen05.mma;
//   warps 8-15  epilogue (256 threads): warp w reads TMEM lanes
//               32*(w%4).. (the lane quarter a warp may access) and half
//               (w-8)/4 of the tile's columns.
// Operand staging (load, split, swizzled store) limits the stages whose
// epilogue only stores, so every warp the issuer and the epilogue do not
// need works in the producer (measured: 7 producer warps beat 4 by 5-13%
// on those stages; 3 producer warps with 12 epilogue warps lost 30%).
// Per-tile sums are reduced per warp (shuffles only) and written to
// per-warp slots, so no role ever waits on a barrier another role could
// abandon after a bounded-wait timeout.
constexpr int kDftPersistThreads = 512;
constexpr int kProWarps = 7;
constexpr int kProThreads = 32 * kProWarps;
constexpr int kMmaWarp = 4;
constexpr int kEpiWarp0 = 8;
constexpr int kEpiThreads = 256;
constexpr int kRowPairs = kTileRows / 2;  // a producer warp covers 2 rows per fetch
constexpr int kProIters = (kRowPairs + kProWarps - 1) / kProWarps;

FBME_DEV TileCtx decode_tile(const DftGeom& g, int tile) {
  TileCtx t;
  t.col_tile = tile % g.col_tiles;
  tile /= g.col_tiles;
  t.row_tile = tile % g.row_tiles;
  t.scene = tile / g.row_tiles;
  t.g = &g;
  return t;
}

// One stage launch: geometry, prologue and epilogue policies, status words.
template <class Pro, class Epi>
struct StageItem {
  DftGeom g;
  Pro pro;
  Epi epi;
  int* status;
};

// Up to NI stage launches of one kind (same policies and tile width) as one
// persistent launch: item i owns the launch's tiles [tile0[i], tile0[i+1]).
// Shape buckets of an uneven plan run their stages this way, one launch
// for all buckets.
template <class Pro, class Epi, int NI>
struct StageSet {
  int n;
  int tile0[NI + 1];
  StageItem<Pro, Epi> it[NI];
  long long wait_cycles = kWaitCycles;  // limit of every mbarrier wait
  int hold = 0;  // nonzero: the producer issues nothing (failure-detection self-test)
  // Item of a tile: the last i with tile0[i] <= tile.
  FBME_DEV int find(int tile) const {
    if constexpr (NI == 1) {
      return 0;
    } else {
      int lo = 0, hi = n - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tile0[mid] <= tile) lo = mid;
        else hi = mid - 1;
      }
      return lo;
    }
  }
};

template <int A_PARTS, int N_TILE, class Pro, class Epi, int NI>
__global__ void __launch_bounds__(kDftPersistThreads, 1)
dft_stage_kernel(const __grid_constant__ StageSet<Pro, Epi, NI> set) {
  using C = DftCfg<A_PARTS, N_TILE>;
  extern __shared__ uint8_t smem_dyn[];
  const uint32_t base_u32 = smem_u32(smem_dyn);
  uint8_t* smem = smem_dyn + (((base_u32 + 1023u) & ~1023u) - base_u32);
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + kStages * C::kStageBytes);
  uint64_t* empty_bar = full_bar + kStages;
  uint64_t* accf_bar = empty_bar + kStages;  // [2]
  uint64_t* acce_bar = accf_bar + 2;         // [2]
  uint64_t* drain_bar = acce_bar + 2;        // MMA completion before TMEM release
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
  const long long wlim = set.wait_cycles;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = set.tile0[set.n];

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], ProBulk<Pro>::value ? 1 : kProThreads);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&accf_bar[a], 1);
      mbar_init(&acce_bar[a], kEpiThreads / 32);
    }
    mbar_init(drain_bar, 1);
    fence_mbar_init();
  }
  if (warp == kMmaWarp) tmem_alloc(tmem_slot, 2 * N_TILE);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (ProBulk<Pro>::value && warp < kEpiWarp0 && warp != kMmaWarp) {
    // ---------------- bulk producer ----------------
    // The operand is stored pre-split and pre-swizzled by the previous
    // stage's epilogue: [unit][row tile][K chunk][part][128 rows x 128 B].
    // Thread 0 copies a chunk's A parts (one contiguous block) and its
    // twiddle blocks, completing on the stage's full barrier; no register
    // work, so the stage runs at the copy engine's and the tensor core's pace.
    if constexpr (ProBulk<Pro>::value) {
      if (threadIdx.x == 0) {
        bool ok = true;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok && !set.hold; tile += gridDim.x) {
          const int ii = set.find(tile);
          const DftGeom& g = set.it[ii].g;
          const Pro& pro = set.it[ii].pro;
          const TileCtx t = decode_tile(g, tile - set.tile0[ii]);
          int* const st_scene = set.it[ii].status ? set.it[ii].status + t.scene / g.status_div : nullptr;
          constexpr uint32_t kABytes = A_PARTS * kPartBytesA;
          const uint8_t* a_src = pro.in + static_cast<size_t>(t.scene) * pro.unit_bytes +
                                 static_cast<size_t>(t.row_tile) * g.kchunks * kABytes;
          const uint8_t* b_src =
              g.table + static_cast<size_t>(t.col_tile) * g.table_kchunks * A_PARTS * C::kPartBytesB;
          for (int kc = 0; kc < g.kchunks && ok; ++kc, ++it) {
            const int s = it % kStages, use = it / kStages;
            uint8_t* st = smem + s * C::kStageBytes;
            if (it >= kStages) {
              ok = mbar_wait(&empty_bar[s], (use - 1) & 1, st_scene, wlim);
              if (!ok) break;
            }
            mbar_arrive_expect_tx(&full_bar[s], kABytes + A_PARTS * C::kPartBytesB);
            bulk_g2s(st, a_src + static_cast<size_t>(kc) * kABytes, kABytes, &full_bar[s]);
            for (int p = 0; p < A_PARTS; ++p)
              bulk_g2s(st + kABytes + p * C::kPartBytesB,
                       b_src + (static_cast<size_t>(kc) * A_PARTS + p) * C::kPartBytesB, C::kPartBytesB,
                       &full_bar[s]);
          }
        }
      }
    }
  } else if (warp < kEpiWarp0 && warp != kMmaWarp) {
    // ---------------- producer ----------------
    // Producer warp pw stages row pairs p = pw + kProWarps * i (tile rows 2p
    // and 2p + 1); lane l covers complex columns 2(l%16), 2(l%16)+1 of the
    // K chunk.  Shared-memory offsets are fixed per thread; element offsets
    // of the rows are computed once per tile, so a K chunk costs one add
    // per row before the load.
    const int pw = warp < kMmaWarp ? warp : warp - 1;  // producer warp 0..6
    const int tid = threadIdx.x;
    const int q = lane & 15;
    uint32_t soff[kProIters];
#pragma unroll
    for (int i = 0; i < kProIters; ++i)
      soff[i] = sw128_offset((pw + kProWarps * i) * 2 + (lane >> 4), q * 4);
    bool ok = true;
    int it = 0;
    // A held producer (self-test) issues no load, copy or arrive: the
    // issuer's and the epilogue's waits run out instead.
    for (int tile = blockIdx.x; tile < ntiles && ok && !set.hold; tile += gridDim.x) {
      const int ii = set.find(tile);
      const DftGeom& g = set.it[ii].g;
      Pro pro = set.it[ii].pro;  // per tile: accumulators start from the launch's values
      const TileCtx t = decode_tile(g, tile - set.tile0[ii]);
      int* const st_scene = set.it[ii].status ? set.it[ii].status + t.scene / g.status_div : nullptr;
      long long erow[kProIters];  // element offset of the row, -1 when outside
#pragma unroll
      for (int i = 0; i < kProIters; ++i) {
        const int pair = pw + kProWarps * i;
        const int r = t.row0() + pair * 2 + (lane >> 4);
        erow[i] = (pair < kRowPairs && r < g.rows)
                      ? t.scene * g.in_stride + static_cast<long long>(r) * g.in_ld
                      : -1;
      }
      if constexpr (Pro::kPipelined) {
        // Two register buffers, used in turn: the loads of chunk kc+1 are in
        // flight while chunk kc is converted and stored.
        typename Pro::Frag fa[kProIters], fb[kProIters];
        auto fetch_all = [&](int kcc, typename Pro::Frag(&f)[kProIters]) {
          const int j0 = kcc * (kKChunk / 2) + q * 2;
          const int avail = g.kcplx - j0;
#pragma unroll
          for (int i = 0; i < kProIters; ++i) pro.fetch(t, erow[i] + j0, erow[i] >= 0 ? avail : 0, f[i]);
        };
        auto store_all = [&](int kcc, const typename Pro::Frag(&f)[kProIters]) -> bool {
          const int s = it % kStages, use = it / kStages;
          uint8_t* st = smem + s * C::kStageBytes;
          if (it >= kStages && !mbar_wait(&empty_bar[s], (use - 1) & 1, st_scene, wlim)) return false;
          if (tid == 0) {
            asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;"
                         ::"r"(smem_u32(&full_bar[s])), "r"(uint32_t(A_PARTS * C::kPartBytesB))
                         : "memory");
            const uint8_t* src = g.table + (static_cast<size_t>(t.col_tile) * g.table_kchunks + kcc) *
                                               A_PARTS * C::kPartBytesB;
            for (int p = 0; p < A_PARTS; ++p)
              bulk_g2s(st + A_PARTS * kPartBytesA + p * C::kPartBytesB, src + p * C::kPartBytesB,
                       C::kPartBytesB, &full_bar[s]);
          }
          const int j0 = kcc * (kKChunk / 2) + q * 2;
          const int avail = g.kcplx - j0;
#pragma unroll
          for (int i = 0; i < kProIters; ++i) {
            if (pw + kProWarps * i >= kRowPairs) continue;
            const float4 v = pro.make(t, erow[i] + j0, erow[i] >= 0 ? avail : 0, f[i]);
            uint2 parts[A_PARTS];
            split4<A_PARTS>(v, parts);
#pragma unroll
            for (int p = 0; p < A_PARTS; ++p)
              *reinterpret_cast<uint2*>(st + p * kPartBytesA + soff[i]) = parts[p];
          }
          fence_proxy_async_smem();
          mbar_arrive(&full_bar[s]);
          ++it;
          return true;
        };
        fetch_all(0, fa);
        for (int kc = 0; kc < g.kchunks && ok; kc += 2) {
          if (kc + 1 < g.kchunks) fetch_all(kc + 1, fb);
          ok = store_all(kc, fa);
          if (!ok || kc + 1 >= g.kchunks) break;
          if (kc + 2 < g.kchunks) fetch_all(kc + 2, fa);
          ok = store_all(kc + 1, fb);
        }
        pro.tile_done(t, pw, lane);
        continue;
      }
      for (int kc = 0; kc < g.kchunks && ok; ++kc, ++it) {
        const int s = it % kStages, use = it / kStages;
        uint8_t* st = smem + s * C::kStageBytes;
        const int j0 = kc * (kKChunk / 2) + q * 2;  // complex column of this lane
        const int avail = g.kcplx - j0;
        constexpr int kB = Pro::kBatch < kProIters ? Pro::kBatch : kProIters;
#pragma unroll
        for (int b0 = 0; b0 < kProIters; b0 += kB) {
          typename Pro::Frag f[kB];
#pragma unroll
          for (int i = 0; i < kB; ++i) {
            if (b0 + i >= kProIters) continue;
            const long long er = erow[b0 + i];
            pro.fetch(t, er + j0, er >= 0 ? avail : 0, f[i]);
          }
          if (b0 == 0) {
            if (it >= kStages) ok = mbar_wait(&empty_bar[s], (use - 1) & 1, st_scene, wlim);
            if (!ok) break;
            if (tid == 0) {
              asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;"
                           ::"r"(smem_u32(&full_bar[s])), "r"(uint32_t(A_PARTS * C::kPartBytesB))
                           : "memory");
              const uint8_t* src = g.table + (static_cast<size_t>(t.col_tile) * g.table_kchunks +
                                              kc) * A_PARTS * C::kPartBytesB;
              for (int p = 0; p < A_PARTS; ++p)
                bulk_g2s(st + A_PARTS * kPartBytesA + p * C::kPartBytesB,
                         src + p * C::kPartBytesB, C::kPartBytesB, &full_bar[s]);
            }
          }
#pragma unroll
          for (int i = 0; i < kB; ++i) {
            if (b0 + i >= kProIters) continue;
            const int pair = pw + kProWarps * (b0 + i);
            if (pair >= kRowPairs) continue;
            const long long er = erow[b0 + i];
            const float4 v = pro.make(t, er + j0, er >= 0 ? avail : 0, f[i]);
            uint2 parts[A_PARTS];
            split4<A_PARTS>(v, parts);
#pragma unroll
            for (int p = 0; p < A_PARTS; ++p)
              *reinterpret_cast<uint2*>(st + p * kPartBytesA + soff[b0 + i]) = parts[p];
          }
        }
        if (!ok) break;
        fence_proxy_async_smem();
        mbar_arrive(&full_bar[s]);
      }
      pro.tile_done(t, pw, lane);
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      bool ok = true, issued = false;
      int it = 0, lt = 0;
      int* st_last = nullptr;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++lt) {
        const int ii = set.find(tile);
        const DftGeom& g = set.it[ii].g;
        const TileCtx t = decode_tile(g, tile - set.tile0[ii]);
        int* const st_scene = set.it[ii].status ? set.it[ii].status + t.scene / g.status_div : nullptr;
        st_last = st_scene;
        const int acc = lt & 1, ause = lt >> 1;
        if (lt >= 2) ok = mbar_wait(&acce_bar[acc], (ause - 1) & 1, st_scene, wlim);
        if (!ok) break;
        tc_fence_after();
        const uint32_t dtm = tmem + static_cast<uint32_t>(acc * N_TILE);
        for (int kc = 0; kc < g.kchunks && ok; ++kc, ++it) {
          const int s = it % kStages, use = it / kStages;
          ok = mbar_wait(&full_bar[s], use & 1, st_scene, wlim);
          if (!ok) break;
          issued = true;
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + s * C::kStageBytes);
          const uint32_t b0 = a0 + A_PARTS * kPartBytesA;
#pragma unroll
          for (int kk = 0; kk < kKChunk / 16; ++kk) {
#pragma unroll
            for (int pr = 0; pr < C::kPairs; ++pr) {
              const uint64_t ad = sw128_desc(a0 + kPairA[pr] * kPartBytesA + kk * 32);
              const uint64_t bd = sw128_desc(b0 + kPairB[pr] * C::kPartBytesB + kk * 32);
              umma_bf16(dtm, ad, bd, C::kIdesc, (kc | kk | pr) != 0);
            }
          }
          umma_commit(&empty_bar[s]);
        }
        if (ok) umma_commit(&accf_bar[acc]);
      }
      // After a timeout, MMAs issued before it may still be running: wait
      // (bounded) until they have completed, so tensor memory is released
      // only once nothing writes it.
      if (!ok && issued) {
        umma_commit(drain_bar);
        mbar_wait(drain_bar, 0, st_last, wlim);
      }
    }
    __syncwarp();
  } else if (warp >= kEpiWarp0) {
    // ---------------- epilogue ----------------
    const int q = warp & 3, h = (warp - kEpiWarp0) >> 2;
    const int row = q * 32 + lane;
    constexpr int kHalf = N_TILE / 2;
    bool ok = true;
    int lt = 0;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++lt) {
      const int ii = set.find(tile);
      const DftGeom& g = set.it[ii].g;
      Epi epi = set.it[ii].epi;
      const TileCtx t = decode_tile(g, tile - set.tile0[ii]);
      int* const st_scene = set.it[ii].status ? set.it[ii].status + t.scene / g.status_div : nullptr;
      const int acc = lt & 1;
      ok = mbar_wait(&accf_bar[acc], (lt >> 1) & 1, st_scene, wlim);
      tc_fence_after();
      if (ok) {
        const uint32_t base = tmem + static_cast<uint32_t>(acc * N_TILE) +
                              (static_cast<uint32_t>(q * 32) << 16);
        const int c_begin = h * kHalf, c_end = (h + 1) * kHalf;
        float va[16], vb[16];
        typename Epi::Pre pa, pb;
        epi.prefetch(t, row, c_begin, pa);
        tmem_ld16(base + static_cast<uint32_t>(c_begin), va);
#pragma unroll 1
        for (int c0 = c_begin; c0 < c_end; c0 += 32) {
          const bool more = c0 + 16 < c_end;
          if (more) {
            tmem_ld16_async(base + static_cast<uint32_t>(c0 + 16), vb);
            epi.prefetch(t, row, c0 + 16, pb);
          }
          epi.consume(t, row, c0, va, pa);
          if (more) {
            tmem_wait_ld(vb);
            const bool more2 = c0 + 32 < c_end;
            if (more2) {
              tmem_ld16_async(base + static_cast<uint32_t>(c0 + 32), va);
              epi.prefetch(t, row, c0 + 32, pa);
            }
            epi.consume(t, row, c0 + 16, vb, pb);
            if (more2) tmem_wait_ld(va);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce_bar[acc]);
      epi.tile_done(t, warp - kEpiWarp0, lane);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * N_TILE);
  }
}

// ---------------------------------------------------------------------------
// Prologue / epilogue policies shared by several stages
// ---------------------------------------------------------------------------

// Prologue policies: fetch(t, e, avail, f) issues the loads of two complex
// values at element offset e of the stage input (avail = complex columns
// left from there; <= 0 outside the matrix, which reads as zero); make(t,
// e, avail, f) turns the fetched values into the 4 floats fed to the tensor
// core.  The producer calls fetch for a batch of rows before it waits for a
// free stage, then make.

// Two complex values at base[e] (avail of them valid), zero outside.
FBME_DEV float4 load_pair(const float2* base, long long e, int avail, bool vec) {
  if (avail >= 2) {
    if (vec) return __ldg(reinterpret_cast<const float4*>(base + e));
    const float2 a = __ldg(base + e), b = __ldg(base + e + 1);
    return make_float4(a.x, a.y, b.x, b.y);
  }
  if (avail == 1) {
    const float2 a = __ldg(base + e);
    return make_float4(a.x, a.y, 0.f, 0.f);
  }
  return make_float4(0.f, 0.f, 0.f, 0.f);
}

struct ProPlain {
  static constexpr int kBatch = 16;
  static constexpr bool kPipelined = true;
  using Frag = float4;
  const float2* in;
  FBME_DEV void fetch(const TileCtx& t, long long e, int avail, Frag& f) const {
    f = load_pair(in, e, avail, t.g->vec4 != 0);
  }
  FBME_DEV float4 make(const TileCtx&, long long, int, const Frag& f) const { return f; }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Epilogue policies: prefetch(t, row, c0, pre) issues the global loads a
// 16-column chunk needs one chunk ahead; consume(t, row, c0, v, pre) gets
// the chunk's 16 accumulator values (8 complex) and the prefetched data.
struct NoPre {};

// Store Out[j][r] (lane-contiguous) as complex64.
struct EpiStoreT {
  using Pre = NoPre;
  float2* out;
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) const {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= g.rows) return;
    float2* o = out + t.scene * g.out_stride + r;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (jb + i < g.cols) o[(jb + i) * g.out_ld] = make_float2(v[2 * i], v[2 * i + 1]);
    }
  }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Intermediate of a two-stage transform stored as the next stage's operand:
// element (r, c) of this stage's output is row c, complex column r of the
// next stage's A, written as its two BF16 parts (hi = bf16(x), lo = bf16(x -
// hi), the split the producer would otherwise do) straight into the
// K-major 128-byte-swizzled layout
//   [unit][c / 128][r / 32][part][c % 128 rows x 128 B].
// A warp's 32 lanes hold 32 consecutive r, one 128-byte operand row per
// column and part: fully coalesced stores.  Rows r past this stage's rows
// carry exact zeros (their inputs read as zero), which is the next stage's
// K padding; columns past `cols` are never written, and the next stage's
// rows that read them are discarded by its epilogue.
struct EpiSplitT {
  using Pre = NoPre;
  uint8_t* out;
  long long unit_bytes;  // row_tiles2 * kchunks2 * 2 * 16 KiB
  int kchunks2;          // K chunks of the next stage (32 complex each)
  FBME_DEV void prefetch(const TileCtx&, int, int, Pre&) const {}
  FBME_DEV void consume(const TileCtx& t, int row, int c0, const float* v, const Pre&) const {
    const DftGeom& g = *t.g;
    const int r = t.row0() + row;
    if (r >= kchunks2 * 32) return;
    const int kc = r >> 5, w = r & 31;
    uint8_t* base = out + t.scene * unit_bytes + static_cast<size_t>(kc) * 2 * kPartBytesA;
    const int jb = t.col0() + (c0 >> 1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int c = jb + i;
      if (c >= g.cols) continue;
      const float2 x = make_float2(v[2 * i], v[2 * i + 1]);
      const __nv_bfloat162 hi = __float22bfloat162_rn(x);
      const float2 h = __bfloat1622float2(hi);
      const __nv_bfloat162 lo = __float22bfloat162_rn(make_float2(x.x - h.x, x.y - h.y));
      const int cr = c & 127;
      uint8_t* blk = base + static_cast<size_t>(c >> 7) * kchunks2 * 2 * kPartBytesA;
      const uint32_t off = cr * 128u + ((((w >> 2) ^ (cr & 7)) & 7) << 4) + (w & 3) * 4u;
      *reinterpret_cast<__nv_bfloat162*>(blk + off) = hi;
      *reinterpret_cast<__nv_bfloat162*>(blk + kPartBytesA + off) = lo;
    }
  }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Prologue of a stage whose A operand EpiSplitT wrote (3-term products).
struct ProSplit {
  static constexpr bool kBulk = true;
  // unused register-producer interface (the bulk producer copies instead)
  static constexpr int kBatch = 1;
  static constexpr bool kPipelined = false;
  using Frag = float4;
  const uint8_t* in;
  long long unit_bytes;
  FBME_DEV void fetch(const TileCtx&, long long, int, Frag& f) const { f = make_float4(0.f, 0.f, 0.f, 0.f); }
  FBME_DEV float4 make(const TileCtx&, long long, int, const Frag& f) const { return f; }
  FBME_DEV void tile_done(const TileCtx&, int, int) {}
};

// Bytes per unit of the split operand of a stage with `rows` rows and a
// contracted length of `kcplx` complex values.
__host__ __device__ inline long long split_unit_bytes(int rows, int kcplx) {
  return static_cast<long long>((rows + kTileRows - 1) / kTileRows) * ((kcplx + 31) / 32) * 2 * kPartBytesA;
}

}  // namespace fbme
