// Active-set switch of single-scene cg runs (torch_sbl/solver.py:1316-1341):
// from EM iteration `active_set_start`, every `active_set_check_interval`
// iterations until it switches, the ARD active set is selected from the
// prior variances (_select_active_indices, solver.py:3184-3216); once
// selected, every remaining EM iteration and the final posterior use the
// exact reduced posterior on it (_active_posterior, solver.py:3897-3920 over
// 3591-3779 with the omitted prior variance as an isotropic loading), and
// the prior variances outside it stay fixed (solver.py:1684-1693).
//
// Both kernels are one CTA of 1024 threads for the one scene:
//   cg_select_kernel     radix select of the K_max largest prior variances
//                        (4 passes of 8-bit digits over order-preserving
//                        keys), ties taken in index order, a bitonic sort
//                        (value descending, index ascending), then the
//                        tail test on the cumulative sums in FP64;
//   cg_active_kernel     the reduced system S = diag(1/gamma_a) + G / nu
//                        (G from the separable Dirichlet tables, nu = noise
//                        + omitted variance), equilibrated, loaded with the
//                        deterministic jitter of the CUDA Cholesky branch,
//                        factored (right-looking, column-major in the plan
//                        workspace), inverted (L^-1, for diag(S^-1)), and
//                        the mean, posterior variance and clipped relevance
//                        scattered back to the grid.
#include <math.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.cuh"
#include "stage.cuh"

namespace fbme {

constexpr int kActThreads = 1024;
constexpr int kActMax = 1024;  // largest supported active_set_max_size

size_t cg_active_bytes(long long N, int kmax) {
  const size_t K = static_cast<size_t>(kmax);
  auto up = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  return up(16 * sizeof(int)) + up(K * sizeof(int)) + up(static_cast<size_t>(N)) + 2 * up(K * K * sizeof(float2));
}

ActiveBufs cg_active_bind(uint8_t* w, long long N, int kmax) {
  const size_t K = static_cast<size_t>(kmax);
  auto up = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  ActiveBufs a;
  size_t o = 0;
  a.sel = reinterpret_cast<int*>(w + o);
  o += up(16 * sizeof(int));
  a.idx = reinterpret_cast<int*>(w + o);
  o += up(K * sizeof(int));
  a.mask = w + o;
  o += up(static_cast<size_t>(N));
  a.E = reinterpret_cast<float2*>(w + o);
  o += up(K * K * sizeof(float2));
  a.X = reinterpret_cast<float2*>(w + o);
  return a;
}

namespace {

// Block-wide sum of a double (1024 threads).
__device__ double block_sum_d(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < (kActThreads >> 5) ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[0] = t;
  }
  __syncthreads();
  t = red[0];
  __syncthreads();
  return t;
}

// Order-preserving key of a non-negative float (larger value, larger key).
__device__ __forceinline__ uint32_t pos_key(float f) { return __float_as_uint(f); }

// _select_active_indices for one scene: sel[0] = size (0: no switch),
// idx[0..K) the K = min(kmax, N) largest prior variances in order.
__global__ void __launch_bounds__(kActThreads)
cg_select_kernel(const float* gamma, long long N, int kmax, int min_size, float tail, ActiveBufs ab) {
  __shared__ double red[32];
  __shared__ int hist[256];
  __shared__ int s_digit, s_need;
  __shared__ uint32_t keys[kActMax];
  __shared__ int ids[kActMax];
  __shared__ int s_count;
  __shared__ int wsum[32];
  const int tid = threadIdx.x;
  const int K = static_cast<int>(kmax < N ? kmax : N);
  // finite check and total (FP64)
  double tot = 0.0;
  int bad = 0;
  for (long long n = tid; n < N; n += kActThreads) {
    const float g = gamma[n];
    if (!isfinite(g)) bad = 1;
    tot += g;
  }
  bad = __syncthreads_or(bad);
  const double total = block_sum_d(tot, red);
  if (bad) {
    if (tid == 0) {
      ab.sel[0] = 0;
      ab.sel[1] = 1;
    }
    return;
  }
  // radix select of the K-th largest key
  uint32_t prefix = 0, pmask = 0;
  int need = K;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = tid; i < 256; i += kActThreads) hist[i] = 0;
    __syncthreads();
    for (long long n = tid; n < N; n += kActThreads) {
      const uint32_t k = pos_key(gamma[n]);
      if ((k & pmask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1);
    }
    __syncthreads();
    if (tid == 0) {
      int run = 0, d = 255;
      for (; d > 0; --d) {
        if (run + hist[d] >= need) break;
        run += hist[d];
      }
      s_digit = d;
      s_need = need - run;
    }
    __syncthreads();
    prefix |= static_cast<uint32_t>(s_digit) << shift;
    pmask |= 255u << shift;
    need = s_need;
    __syncthreads();
  }
  const uint32_t T = prefix;  // the K-th largest key; `need` of its ties are taken
  // the keys above T (K - need of them), in any order
  if (tid == 0) s_count = 0;
  __syncthreads();
  for (long long n = tid; n < N; n += kActThreads) {
    const uint32_t k = pos_key(gamma[n]);
    if (k > T) {
      const int p = atomicAdd(&s_count, 1);
      keys[p] = k;
      ids[p] = static_cast<int>(n);
    }
  }
  __syncthreads();
  // the first `need` ties in index order (ordered block compaction)
  const int base = s_count;
  int taken = 0;  // uniform over the block
  const int lane = tid & 31, wid = tid >> 5;
  for (long long c0 = 0; c0 < N && taken < need; c0 += kActThreads) {
    const long long n = c0 + tid;
    const bool tie = n < N && pos_key(gamma[n]) == T;
    const unsigned bal = __ballot_sync(0xffffffffu, tie);
    if (lane == 0) wsum[wid] = __popc(bal);
    __syncthreads();
    if (tid == 0) {  // exclusive scan over the warps; the chunk's total in s_digit
      int run = 0;
      for (int w = 0; w < kActThreads / 32; ++w) {
        const int v = wsum[w];
        wsum[w] = run;
        run += v;
      }
      s_digit = run;
    }
    __syncthreads();
    if (tie) {
      const int pos = taken + wsum[wid] + __popc(bal & ((1u << lane) - 1u));
      if (pos < need) {
        keys[base + pos] = T;
        ids[base + pos] = static_cast<int>(n);
      }
    }
    taken += s_digit;
    __syncthreads();  // wsum and s_digit are rewritten by the next chunk
  }
  // pad and sort: value descending, index ascending
  for (int i = K + tid; i < kActMax; i += kActThreads) {
    keys[i] = 0u;
    ids[i] = 0x7fffffff;
  }
  __syncthreads();
  for (int size = 2; size <= kActMax; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < kActMax; i += kActThreads) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;  // this run sorts "first-before-second" ascending in rank
          const uint32_t ki = keys[i], kj = keys[j];
          const int ii = ids[i], ij = ids[j];
          // rank order: larger key first, then smaller index
          const bool j_first = kj > ki || (kj == ki && ij < ii);
          if (j_first == up) {
            keys[i] = kj;
            keys[j] = ki;
            ids[i] = ij;
            ids[j] = ii;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < K; i += kActThreads) ab.idx[i] = ids[i];
  if (tid == 0) {
    const double target = (1.0 - static_cast<double>(tail)) * total;
    double top = 0.0;
    for (int i = 0; i < K; ++i) top += static_cast<double>(__uint_as_float(keys[i]));
    int size = 0;
    if (!(top < target)) {
      double cum = 0.0;
      int first = K - 1;
      for (int i = 0; i < K; ++i) {
        cum += static_cast<double>(__uint_as_float(keys[i]));
        if (cum >= target) {
          first = i;
          break;
        }
      }
      const int required = (first < K - 1 ? first : K - 1) + 1;
      size = required > min_size ? required : min_size;
      if (size > K) size = K;
    }
    ab.sel[0] = size;
    ab.sel[1] = 0;
  }
}

__global__ void cg_active_scatter_kernel(const int* idx, const int* sel, uint8_t* mask) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < sel[0]) mask[idx[k]] = 1;
}

// Gram entry G[i][k] = a_i^H a_k of atoms (i1, i2), (k1, k2): the separable
// Dirichlet product D1(i1 - k1) D2(i2 - k2) over the prefix block.
__device__ __forceinline__ float2 gram_entry(const ActiveArgs& a, int i1, int i2, int k1, int k2) {
  int d1 = i1 - k1, d2 = i2 - k2;
  if (d1 < 0) d1 += a.n1;
  if (d2 < 0) d2 += a.n2;
  return cmul(__ldg(a.d1 + d1), __ldg(a.d2 + d2));
}

// The reduced posterior on the active set (one scene, 1024 threads).
__global__ void __launch_bounds__(kActThreads) cg_active_kernel(const ActiveArgs a) {
  __shared__ double red[32];
  __shared__ float dsc[kActMax], ga[kActMax];
  __shared__ int n1s[kActMax], n2s[kActMax];
  __shared__ float2 colq[kActMax];
  __shared__ float2 zvec[kActMax], bvec[kActMax];
  __shared__ float s_piv;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int K = a.K;
  const long long N = a.N;
  // omitted prior variance as an isotropic loading of the noise
  double tot = 0.0;
  for (long long n = tid; n < N; n += kActThreads) tot += a.gamma[n];
  double act = 0.0;
  for (int i = tid; i < K; i += kActThreads) {
    const int n = a.idx[i];
    const float g = a.gamma[n];
    ga[i] = g;
    n1s[i] = n / a.n2;
    n2s[i] = n - (n / a.n2) * a.n2;
    act += g;
  }
  const double total = block_sum_d(tot, red);
  const double active = block_sum_d(act, red);
  const float omitted = fmaxf(static_cast<float>(total) - static_cast<float>(active), 0.f);
  const float nu = a.noise[0] + omitted;
  // outputs off the active set: zero mean and relevance, prior variance
  for (long long n = tid; n < N; n += kActThreads) {
    a.mean[n] = make_float2(0.f, 0.f);
    a.relc[n] = 0.f;
    if (a.pv_out) a.pv_out[n] = a.gamma[n];
  }
  __syncthreads();
  // S = diag(1/gamma) + G / nu (Hermitian part); equilibration scale d
  for (int i = tid; i < K; i += kActThreads) {
    const float2 g = gram_entry(a, n1s[i], n2s[i], n1s[i], n2s[i]);
    const float sii = g.x / nu + 1.0f / ga[i];
    dsc[i] = sqrtf(fmaxf(sii, kTiny));
  }
  __syncthreads();
  // equilibrated lower triangle, column-major: E[k * K + i], i >= k
  double dsum = 0.0;
  for (int k = ty; k < K; k += kActThreads / 32) {
    for (int i = k + tx; i < K; i += 32) {
      const float2 g = gram_entry(a, n1s[i], n2s[i], n1s[k], n2s[k]);
      const float2 h = gram_entry(a, n1s[k], n2s[k], n1s[i], n2s[i]);
      float2 sv = make_float2(0.5f * (g.x + h.x) / nu, 0.5f * (g.y - h.y) / nu);
      if (i == k) sv = make_float2(sv.x + 1.0f / ga[i], 0.f);
      sv = make_float2(sv.x / dsc[i] / dsc[k], sv.y / dsc[i] / dsc[k]);
      a.E[static_cast<long long>(k) * K + i] = sv;
      if (i == k) dsum += fabsf(sv.x);
    }
  }
  // deterministic loading of the CUDA Cholesky branch: m * eps * mean|diag|
  const double dmean = block_sum_d(dsum, red) / K;
  const float jit = a.jitter * (kEps * fmaxf(static_cast<float>(dmean), kTiny));
  for (int i = tid; i < K; i += kActThreads) a.E[static_cast<long long>(i) * K + i].x += jit;
  __syncthreads();
  // Cholesky, right-looking, in place (lower)
  int stat = 0;
  for (int q = 0; q < K; ++q) {
    if (tid == 0) {
      float sdiag = a.E[static_cast<long long>(q) * K + q].x;
      if (!(sdiag > 0.f)) {
        stat |= isfinite(sdiag) ? FBME_STATUS_CHOLESKY : FBME_STATUS_NONFINITE;
        sdiag = kTiny;
      }
      const float piv = sqrtf(sdiag);
      a.E[static_cast<long long>(q) * K + q] = make_float2(piv, 0.f);
      s_piv = piv;
    }
    __syncthreads();
    const float piv = s_piv;
    for (int i = q + 1 + tid; i < K; i += kActThreads) {
      float2 v = a.E[static_cast<long long>(q) * K + i];
      v = make_float2(v.x / piv, v.y / piv);
      a.E[static_cast<long long>(q) * K + i] = v;
      colq[i] = v;
    }
    __syncthreads();
    for (int k = q + 1 + ty; k < K; k += kActThreads / 32) {
      const float2 bk = colq[k];
      float2* col = a.E + static_cast<long long>(k) * K;
      for (int i = k + tx; i < K; i += 32) {
        const float2 ai = colq[i];
        float2 v = col[i];
        v.x -= ai.x * bk.x + ai.y * bk.y;  // ai * conj(bk)
        v.y -= ai.y * bk.x - ai.x * bk.y;
        col[i] = v;
      }
    }
    __syncthreads();
  }
  if (tid == 0 && stat && a.status) atomicOr(a.status, stat);
  // X = L^-1 (lower, column-major X[j * K + i]): rows in order, each
  // divided by its pivot once final, then eliminated from the rows below
  for (int j = ty; j < K; j += kActThreads / 32)
    for (int i = j + tx; i < K; i += 32)
      a.X[static_cast<long long>(j) * K + i] = make_float2(i == j ? 1.f : 0.f, 0.f);
  __syncthreads();
  for (int k = 0; k < K; ++k) {
    const float rk = 1.0f / a.E[static_cast<long long>(k) * K + k].x;
    for (int j = tid; j <= k; j += kActThreads) {
      float2* x = a.X + static_cast<long long>(j) * K + k;
      *x = make_float2(x->x * rk, x->y * rk);
    }
    __syncthreads();
    const float2* lk = a.E + static_cast<long long>(k) * K;
    for (int j = ty; j <= k; j += kActThreads / 32) {
      float2* col = a.X + static_cast<long long>(j) * K;
      const float2 xk = col[k];
      for (int i = k + 1 + tx; i < K; i += 32) {
        const float2 l = lk[i];
        float2 v = col[i];
        v.x -= l.x * xk.x - l.y * xk.y;  // l * xk
        v.y -= l.x * xk.y + l.y * xk.x;
        col[i] = v;
      }
    }
    __syncthreads();
  }
  // mean: S^-1 b = D^-1 X^H X D^-1 (c / nu), c = A_a^H y (the backprojection)
  for (int j = tid; j < K; j += kActThreads) {
    const float2 c = __ldg(a.bp + a.idx[j]);
    bvec[j] = make_float2(c.x / nu / dsc[j], c.y / nu / dsc[j]);
  }
  __syncthreads();
  for (int i = tid; i < K; i += kActThreads) {
    float2 z = make_float2(0.f, 0.f);
    for (int j = 0; j <= i; ++j) {
      const float2 b = bvec[j];
      const float2 x = a.X[static_cast<long long>(j) * K + i];
      z.x += x.x * b.x - x.y * b.y;
      z.y += x.x * b.y + x.y * b.x;
    }
    zvec[i] = z;
  }
  __syncthreads();
  double rsum = 0.0;
  for (int j = tid; j < K; j += kActThreads) {
    const float2* col = a.X + static_cast<long long>(j) * K;
    float2 w = make_float2(0.f, 0.f);
    float var = 0.f;
    for (int i = j; i < K; ++i) {
      const float2 x = col[i], z = zvec[i];
      w.x += x.x * z.x + x.y * z.y;  // conj(x) * z
      w.y += x.x * z.y - x.y * z.x;
      var += x.x * x.x + x.y * x.y;
    }
    const float d = dsc[j], g = ga[j];
    const float2 mean = make_float2(w.x / d, w.y / d);
    const float pv = fmaxf(var / (d * d), 0.f);
    const float dd = fmaxf((g - pv) / (g * g), 0.f);
    const float rc = fminf(fmaxf(g * dd, 0.f), 1.f);
    const int n = a.idx[j];
    a.mean[n] = mean;
    a.relc[n] = rc;
    if (a.pv_out) a.pv_out[n] = pv;
    rsum += rc;
  }
  const double rel = block_sum_d(rsum, red);
  // relevance sum in partial slot 0 of tile 0 (the other tiles of the EM
  // kernels' partial layout hold zero)
  for (int t = tid; t < a.nb; t += kActThreads)
    a.part[static_cast<long long>(t) * kPartSlots + 0] = t == 0 ? rel : 0.0;
}

}  // namespace

void cg_active_select(const float* gamma, long long N, int kmax, int min_size, float tail, const ActiveBufs& ab,
                      cudaStream_t st) {
  cg_select_kernel<<<1, kActThreads, 0, st>>>(gamma, N, kmax, min_size, tail, ab);
}

void cg_active_mask(const ActiveBufs& ab, long long N, int kmax, cudaStream_t st) {
  cudaMemsetAsync(ab.mask, 0, static_cast<size_t>(N), st);
  cg_active_scatter_kernel<<<(kmax + 255) / 256, 256, 0, st>>>(ab.idx, ab.sel, ab.mask);
}

void cg_active_posterior(const ActiveArgs& a, cudaStream_t st) {
  cg_active_kernel<<<1, kActThreads, 0, st>>>(a);
}

}  // namespace fbme
