// Per-scene top-K selection over order-preserving 32-bit float keys.
//
// Replaces torch.topk(score, K) at torch_sbl/solver.py:1931 (active set),
// 4410 (residual exchange additions).  One CTA per scene: a 3-pass radix
// select (11/11/10-bit digits, most significant first) finds the key of the
// K-th largest element; elements above it are collected directly, ties at
// that key are taken in increasing index order, and the K winners are
// sorted descending (ties by lower index).
#include "common.cuh"
#include "kernels.cuh"

namespace fbme {

constexpr int kTopkThreads = 1024;

FBME_DEV float key_to_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__global__ void __launch_bounds__(kTopkThreads)
topk_select_kernel(const uint32_t* keys, long long n, int k, int* out_idx, float* out_val) {
  __shared__ uint32_t hist[2048];
  __shared__ uint32_t s_prefix, s_mask;
  __shared__ int s_remaining;
  __shared__ int sel_idx[32];
  __shared__ uint32_t sel_key[32];
  __shared__ int s_ngt, s_filled;
  __shared__ int warp_cnt[32];
  const int scene = blockIdx.x;
  const uint32_t* kp = keys + scene * n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    s_prefix = 0;
    s_mask = 0;
    s_remaining = k;
  }
  const int shifts[3] = {21, 10, 0};
  const int widths[3] = {11, 11, 10};
  for (int pass = 0; pass < 3; ++pass) {
    const int shift = shifts[pass], nb = 1 << widths[pass];
    for (int b = tid; b < 2048; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    const uint32_t prefix = s_prefix, mask = s_mask;
    for (long long i = tid; i < n; i += blockDim.x) {
      const uint32_t key = kp[i];
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & (nb - 1)], 1u);
    }
    __syncthreads();
    if (warp == 0) {
      // lane l owns bins [nb - per*(l+1), nb - per*l) counted from the top
      const int per = nb / 32;
      const int hi = nb - per * lane;
      uint32_t local = 0;
      for (int b = hi - 1; b >= hi - per; --b) local += hist[b];
      // inclusive scan from the top (lane 0 = highest bins)
      uint32_t incl = local;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t excl = incl - local;
      const int rem = s_remaining;
      const bool here = excl < static_cast<uint32_t>(rem) && incl >= static_cast<uint32_t>(rem);
      const unsigned ball = __ballot_sync(0xffffffffu, here);
      const int owner = ball ? __ffs(ball) - 1 : 31;
      if (lane == owner) {
        uint32_t cum = excl;
        int sel = hi - per;
        for (int b = hi - 1; b >= hi - per; --b) {
          if (cum + hist[b] >= static_cast<uint32_t>(rem)) {
            sel = b;
            break;
          }
          cum += hist[b];
        }
        s_remaining = rem - static_cast<int>(cum);
        s_prefix = prefix | (static_cast<uint32_t>(sel) << shift);
        s_mask = mask | (static_cast<uint32_t>(nb - 1) << shift);
      }
    }
    __syncthreads();
  }
  const uint32_t T = s_prefix;
  const int need_eq = s_remaining;  // elements equal to T to take
  if (tid == 0) {
    s_ngt = 0;
    s_filled = 0;
  }
  __syncthreads();
  for (long long i = tid; i < n; i += blockDim.x) {
    const uint32_t key = kp[i];
    if (key > T) {
      const int pos = atomicAdd(&s_ngt, 1);
      if (pos < 32) {
        sel_idx[pos] = static_cast<int>(i);
        sel_key[pos] = key;
      }
    }
  }
  __syncthreads();
  const int base = k - need_eq;
  for (long long start = 0; start < n; start += blockDim.x) {
    if (s_filled >= need_eq) break;  // uniform: read after a barrier
    const long long i = start + tid;
    const bool eq = i < n && kp[i] == T;
    const unsigned ball = __ballot_sync(0xffffffffu, eq);
    if (lane == 0) warp_cnt[warp] = __popc(ball);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += warp_cnt[w];
    const int rank = before + __popc(ball & ((1u << lane) - 1u));
    const int filled = s_filled;
    if (eq && filled + rank < need_eq) {
      sel_idx[base + filled + rank] = static_cast<int>(i);
      sel_key[base + filled + rank] = T;
    }
    __syncthreads();
    if (tid == 0) {
      int tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += warp_cnt[w];
      s_filled = filled + tot;
    }
    __syncthreads();
  }
  // sort the k winners: key descending, index ascending (warp bitonic sort)
  if (warp == 0) {
    uint32_t key = lane < k ? sel_key[lane] : 0u;
    int idx = lane < k ? sel_idx[lane] : 0x7fffffff;
    for (int size = 2; size <= 32; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const uint32_t ok = __shfl_xor_sync(0xffffffffu, key, stride);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, stride);
        // "a before b" when key larger, or equal key and smaller index
        const bool other_first = (ok > key) || (ok == key && oi < idx);
        const bool lower = (lane & stride) == 0;
        const bool ascending_block = (lane & size) == 0;  // block order: "first" at low lanes
        const bool take = lower == ascending_block ? other_first : !other_first;
        if (take) {
          key = ok;
          idx = oi;
        }
      }
    }
    if (lane < k) {
      out_idx[scene * k + lane] = idx;
      out_val[scene * k + lane] = key_to_float(key);
    }
  }
}

void launch_topk(const uint32_t* keys, long long n, int k, int B, int* out_idx, float* out_val,
                 cudaStream_t st) {
  topk_select_kernel<<<B, kTopkThreads, 0, st>>>(keys, n, k, out_idx, out_val);
}

}  // namespace fbme
