// Block-wide top-k (k <= 32) over order-preserving 32-bit keys held in
// registers, with the index-order tie break of a stable descending sort.
//
// Used twice per selection: many CTAs per scene each reduce a slice of the
// grid to k candidates, then one CTA per scene merges the candidates; the
// result is exactly the k largest keys of the scene (largest first, ties by
// lower index), which is what torch.topk returns at solver.py:1931/4410.
#pragma once

#include "common.cuh"

namespace fbme {

FBME_DEV uint32_t float_key_t(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
FBME_DEV float key_to_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

struct TopkShared {
  uint32_t hist[256];
  uint32_t prefix, mask;
  int remaining, ngt, neq, filled, nvalid;
  int red_idx[32];
  uint32_t sel_key[32];
  int sel_idx[32];
};

// Warp 0, after a radix pass's histogram: the digit bin that holds the
// remaining-th largest key; narrows prefix/mask and the remaining count.
FBME_DEV void radix_pick_bin(TopkShared& S, int shift, uint32_t prefix, uint32_t mask) {
  const int lane = threadIdx.x & 31;
  const int hi = 256 - 8 * lane;  // lane owns bins [hi-8, hi), counted from the top
  uint32_t local = 0;
#pragma unroll
  for (int b = 1; b <= 8; ++b) local += S.hist[hi - b];
  uint32_t incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t excl = incl - local;
  const int rem = S.remaining;
  const bool here = excl < static_cast<uint32_t>(rem) && incl >= static_cast<uint32_t>(rem);
  const unsigned ball = __ballot_sync(0xffffffffu, here);
  const int owner = ball ? __ffs(ball) - 1 : 31;
  if (lane == owner) {
    uint32_t cum = excl;
    int sel = hi - 8;
    for (int b = hi - 1; b >= hi - 8; --b) {
      if (cum + S.hist[b] >= static_cast<uint32_t>(rem)) {
        sel = b;
        break;
      }
      cum += S.hist[b];
    }
    S.remaining = rem - static_cast<int>(cum);
    S.prefix = prefix | (static_cast<uint32_t>(sel) << shift);
    S.mask = mask | (255u << shift);
  }
}

// k-th largest of the valid keys held one per thread (1 <= k <= their
// number): radix select with 8-bit digits, histogram counts aggregated per
// warp (the keys crowd into few top-byte bins).  Ends on a barrier.
FBME_DEV uint32_t block_kth_key(uint32_t key, bool valid, int k, TopkShared& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    S.prefix = 0;
    S.mask = 0;
    S.remaining = k;
  }
#pragma unroll 1
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    for (int b = tid; b < 256; b += blockDim.x) S.hist[b] = 0;
    __syncthreads();
    const uint32_t prefix = S.prefix, mask = S.mask;
    const bool part = valid && (key & mask) == prefix;
    const unsigned act = __ballot_sync(0xffffffffu, part);
    if (part) {
      const uint32_t bin = (key >> shift) & 255u;
      const unsigned peers = __match_any_sync(act, bin);
      if (__ffs(peers) - 1 == lane) atomicAdd(&S.hist[bin], static_cast<uint32_t>(__popc(peers)));
    }
    __syncthreads();
    if (warp == 0) radix_pick_bin(S, shift, prefix, mask);
    __syncthreads();
  }
  return S.prefix;
}

// Block-wide top-k (k <= 32) of the valid (key, gidx) pairs held KPT per
// thread.  Radix select with 8-bit digits finds the k-th largest key T;
// keys above T are all taken; among keys equal to T the lowest indices are
// taken.  Writes k winners, sorted (key desc, index asc), to out_key/out_idx.
// AGG: warp-aggregated histogram atomics (lanes whose keys share a bin add
// once); pays where the keys crowd into few bins, costs where they spread.
// Entries are read through valid(i) and gidx(i), so callers can compute
// them instead of holding arrays.
template <int KPT, bool AGG, typename Valid, typename GIdx>
FBME_DEV void block_topk_fn(const uint32_t (&key)[KPT], Valid valid, GIdx gidx, int k, TopkShared& S,
                            uint32_t* out_key, int* out_idx) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  if (tid == 0) {
    S.prefix = 0;
    S.mask = 0;
    S.ngt = 0;
    S.neq = 0;
    S.filled = 0;
    S.nvalid = 0;
  }
  __syncthreads();
  {
    int nv = 0;
#pragma unroll
    for (int i = 0; i < KPT; ++i) nv += valid(i) ? 1 : 0;
    nv = warp_sum(nv);
    if (lane == 0 && nv) atomicAdd(&S.nvalid, nv);
  }
  __syncthreads();
  const int k_out = k;
  k = min(k, S.nvalid);  // fewer valid entries than k: pad the output
  if (tid == 0) S.remaining = k;
  if (k == 0) {
    if (tid < k_out) {
      out_key[tid] = 0u;
      out_idx[tid] = 0x7fffffff;
    }
    __syncthreads();
    return;
  }
#pragma unroll 1
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    for (int b = tid; b < 256; b += blockDim.x) S.hist[b] = 0;
    __syncthreads();
    const uint32_t prefix = S.prefix, mask = S.mask;
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const bool part = valid(i) && (key[i] & mask) == prefix;
      if constexpr (AGG) {
        const unsigned act = __ballot_sync(0xffffffffu, part);
        if (part) {
          const uint32_t bin = (key[i] >> shift) & 255u;
          const unsigned peers = __match_any_sync(act, bin);
          if (__ffs(peers) - 1 == lane) atomicAdd(&S.hist[bin], static_cast<uint32_t>(__popc(peers)));
        }
      } else if (part) {
        atomicAdd(&S.hist[(key[i] >> shift) & 255u], 1u);
      }
    }
    __syncthreads();
    if (warp == 0) radix_pick_bin(S, shift, prefix, mask);
    __syncthreads();
  }
  const uint32_t T = S.prefix;
  const int need_eq = S.remaining;  // >= 1
  int my_eq = 0;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    if (valid(i) && key[i] > T) {
      const int pos = atomicAdd(&S.ngt, 1);
      if (pos < 32) {
        S.sel_key[pos] = key[i];
        S.sel_idx[pos] = gidx(i);
      }
    }
    my_eq += (valid(i) && key[i] == T) ? 1 : 0;
  }
  my_eq = warp_sum(my_eq);
  if (lane == 0 && my_eq) atomicAdd(&S.neq, my_eq);
  __syncthreads();
  const int base = k - need_eq;
  if (S.neq == need_eq) {
    // every tie is a winner
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      if (valid(i) && key[i] == T) {
        const int pos = atomicAdd(&S.filled, 1);
        S.sel_key[base + pos] = T;
        S.sel_idx[base + pos] = gidx(i);
      }
    }
  } else {
    // more ties than places: take the lowest indices, one per round
    int taken_below = -1;  // indices <= taken_below are already taken
    for (int r = 0; r < need_eq; ++r) {
      int best = 0x7fffffff;
#pragma unroll
      for (int i = 0; i < KPT; ++i)
        if (valid(i) && key[i] == T && gidx(i) > taken_below && gidx(i) < best) best = gidx(i);
      for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
      if (lane == 0) S.red_idx[warp] = best;
      __syncthreads();
      int b2 = 0x7fffffff;
      for (int w = 0; w < nwarps; ++w) b2 = min(b2, S.red_idx[w]);
      if (tid == 0) {
        S.sel_key[base + r] = T;
        S.sel_idx[base + r] = b2;
      }
      taken_below = b2;
      __syncthreads();
    }
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t kk = lane < k ? S.sel_key[lane] : 0u;
    int ii = lane < k ? S.sel_idx[lane] : 0x7fffffff;
    for (int size = 2; size <= 32; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const uint32_t ok = __shfl_xor_sync(0xffffffffu, kk, stride);
        const int oi = __shfl_xor_sync(0xffffffffu, ii, stride);
        const bool other_first = (ok > kk) || (ok == kk && oi < ii);
        const bool lower = (lane & stride) == 0;
        const bool asc = (lane & size) == 0;
        if (lower == asc ? other_first : !other_first) {
          kk = ok;
          ii = oi;
        }
      }
    if (lane < k_out) {
      out_key[lane] = lane < k ? kk : 0u;
      out_idx[lane] = lane < k ? ii : 0x7fffffff;
    }
  }
  __syncthreads();
}

template <int KPT, bool AGG = false>
FBME_DEV void block_topk(const uint32_t (&key)[KPT], const int (&gidx)[KPT], const bool (&valid)[KPT],
                         int k, TopkShared& S, uint32_t* out_key, int* out_idx) {
  block_topk_fn<KPT, AGG>(
      key, [&](int i) { return valid[i]; }, [&](int i) { return gidx[i]; }, k, S, out_key, out_idx);
}

constexpr int kPrunedCap = 256;
constexpr int kPrunedLaneMax = 256;  // warps x k lane maxima ranked for the bound

struct TopkPrunedShared {
  TopkShared radix;  // the fallback's
  uint32_t lane_max[kPrunedLaneMax];
  uint32_t t0;
  int ncand;
  uint2 cand[kPrunedCap];  // (key, index)
};

// How block_topk_pruned finds its bound T0: kWarpSort sorts each warp's
// lane maxima and ranks the warps' k largest by counting (few warps x small
// k); kRadix runs a radix select over the lane maxima (large k).
enum class TopkBound { kWarpSort, kRadix };

// Block-wide top-k (k <= 32) with the result of block_topk, for key sets
// whose k best are few among many.  Every thread's largest key is a lane
// maximum; the k-th largest lane maximum T0 is a lower bound on the
// block's k-th key (k different threads hold a key >= T0), so the block's
// top k are among the keys >= T0, typically little more than k of them.
// The keys >= T0 go on a shared list, where each finds its output place by
// counting the entries ahead of it (key desc, index asc).  A zero bound,
// fewer than k threads with a key, or a list longer than kPrunedCap falls
// back to the radix select over all keys.  valid: bit i set when entry i
// counts; gidx(i): its index.  The block is whole warps.
template <int KPT, bool AGG, TopkBound BOUND = TopkBound::kWarpSort, typename GIdx>
FBME_DEV void block_topk_pruned(const uint32_t (&key)[KPT], uint32_t valid, GIdx gidx, int k,
                                TopkPrunedShared& P, uint32_t* out_key, int* out_idx) {
  static_assert(KPT <= 32, "the valid mask holds 32 entries");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto radix = [&]() {
    block_topk_fn<KPT, AGG>(
        key, [&](int i) { return ((valid >> i) & 1u) != 0u; }, gidx, k, P.radix, out_key, out_idx);
  };
  uint32_t m = 0u;
#pragma unroll
  for (int i = 0; i < KPT; ++i)
    if ((valid >> i) & 1u) m = max(m, key[i]);
  uint32_t t0 = 0u;
  if constexpr (BOUND == TopkBound::kWarpSort) {
    // each warp offers its k largest lane maxima, which hold the block's k
    // largest; T0 is found among them by counting
    const int offered = (blockDim.x >> 5) * k;
    if (offered > kPrunedLaneMax) {
      radix();
      return;
    }
    // bitonic sort of the warp's lane maxima, descending
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const uint32_t o = __shfl_xor_sync(0xffffffffu, m, stride);
        const bool keep_max = ((lane & stride) == 0) == ((lane & size) == 0);
        m = keep_max ? max(m, o) : min(m, o);
      }
    if (lane < k) P.lane_max[warp * k + lane] = m;
    if (tid == 0) {
      P.t0 = 0u;
      P.ncand = 0;
    }
    __syncthreads();
    if (tid < offered) {
      // place among the offered maxima, ties by position: unique
      const uint32_t me = P.lane_max[tid];
      int rank = 0;
      for (int j = 0; j < offered; ++j) {
        const uint32_t o = P.lane_max[j];
        rank += (o > me || (o == me && j < tid)) ? 1 : 0;
      }
      if (rank == k - 1) P.t0 = me;
    }
    __syncthreads();
    t0 = P.t0;
  } else {
    if (tid == 0) P.ncand = 0;
    if (__syncthreads_count(valid != 0u) < k) {
      radix();
      return;
    }
    t0 = block_kth_key(m, valid != 0u, k, P.radix);
  }
  if (t0 == 0u) {
    radix();
    return;
  }
#pragma unroll
  for (int i = 0; i < KPT; ++i)
    if (((valid >> i) & 1u) && key[i] >= t0) {
      const int pos = atomicAdd(&P.ncand, 1);
      if (pos < kPrunedCap) P.cand[pos] = make_uint2(key[i], static_cast<uint32_t>(gidx(i)));
    }
  __syncthreads();
  const int n = P.ncand;  // >= k: k threads hold a valid key >= t0
  if (n > kPrunedCap) {
    radix();
    return;
  }
  for (int c = tid; c < n; c += blockDim.x) {
    const uint2 me = P.cand[c];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const uint2 o = P.cand[j];
      rank += (o.x > me.x || (o.x == me.x && static_cast<int>(o.y) < static_cast<int>(me.y))) ? 1 : 0;
    }
    if (rank < k) {
      out_key[rank] = me.x;
      out_idx[rank] = static_cast<int>(me.y);
    }
  }
  __syncthreads();
}

}  // namespace fbme
