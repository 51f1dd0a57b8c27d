// FP32 FFT form of the prefix operator's stages (the "fp32-fft" precision
// mode, dft_terms = 0).
//
// A stage of the prefix operator contracts the contiguous axis of each row
// with a DFT submatrix (csrc/dft_umma.cuh):
//     Out[r, c] = sum_{k < K} In[r, k] w^(k c),  c < C,  w = exp(sign 2 pi i / L)
// Here it is computed as a length-L FFT per row (input zero-padded from K,
// output truncated to C), L = 2^a 3^b (b <= 1): for 32 <= L <= 512 in two
// register passes around one shared-memory exchange (fft_fast_kernel), for
// shorter rows as mixed radix 4 / 2 / 3 Stockham passes on shared memory
// (fft_stage_kernel); the twiddles between the passes come from an
// FP64-evaluated table of the L roots of unity.  The error against an FP64
// DFT is that of an FP32 FFT (1.1-1.5e-7 relative L2 for one 2-D prefix
// transform of a random complex input, where cuFFT in FP32 gives
// 1.8-2.6e-7), while the split-BF16 tensor-core products stop at 1-6e-6.
//
// A CTA of 256 threads takes 256 / P rows (P threads per row) in the
// two-pass kernel, RT = 4096 / L (power of two) in the Stockham one; outputs
// are stored with the row on the contiguous axis, as the tensor-core stages store them, and the
// stage's prologue / epilogue sums go to the same per-tile, per-warp partial
// slots (8 warps per tile), so the scalar updates read them unchanged.
#include <math.h>

#include <utility>

#include "common.cuh"
#include "denoise.cuh"
#include "kernels.cuh"
#include "stage.cuh"

namespace fbme {

namespace {

constexpr int kFftThreads = 256;
constexpr int kFftMaxPasses = 12;

struct FftPlan {
  int L;                       // transform length
  int passes;
  int radix[kFftMaxPasses];    // radices in pass order
  int rows_per_cta;            // RT
  float sign;                  // -1 forward, +1 adjoint
  const float2* tw;            // FP64-evaluated roots of unity (fft_twiddle_kernel's layout)
};

// One stage over `units` transforms: geometry of the GEMM stage it replaces.
struct FftStage {
  FftPlan p;
  int rows, kin, cols;         // rows, contracted length K, outputs C
  int in_ld, out_ld;
  long long in_stride, out_stride;
  int tiles;                   // row tiles per transform
  int units;                   // transforms
};

FBME_DEV float2 twiddle(const FftPlan& p, long long idx) {
  const float2 w = __ldg(p.tw + (idx % p.L));
  return make_float2(w.x, p.sign < 0.f ? w.y : -w.y);
}

// radix-R DFT in registers with exponent sign s (w = exp(s 2 pi i / R))
FBME_DEV void dft2(float2* v) {
  const float2 a = v[0], b = v[1];
  v[0] = make_float2(a.x + b.x, a.y + b.y);
  v[1] = make_float2(a.x - b.x, a.y - b.y);
}
FBME_DEV void dft4(float2* v, float s) {
  const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
  const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
  const float2 b0 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
  const float2 b1 = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
  // (s i) * b1
  const float2 ib1 = make_float2(-s * b1.y, s * b1.x);
  v[0] = make_float2(a0.x + b0.x, a0.y + b0.y);
  v[2] = make_float2(a0.x - b0.x, a0.y - b0.y);
  v[1] = make_float2(a1.x + ib1.x, a1.y + ib1.y);
  v[3] = make_float2(a1.x - ib1.x, a1.y - ib1.y);
}
FBME_DEV void dft3(float2* v, float s) {
  // w = -1/2 + s i sqrt(3)/2
  const float c = -0.5f, d = s * 0.86602540378443864676f;
  const float2 t = make_float2(v[1].x + v[2].x, v[1].y + v[2].y);
  const float2 u = make_float2(v[1].x - v[2].x, v[1].y - v[2].y);
  const float2 m = make_float2(v[0].x + c * t.x, v[0].y + c * t.y);
  const float2 iu = make_float2(-d * u.y, d * u.x);
  v[0] = make_float2(v[0].x + t.x, v[0].y + t.y);
  v[1] = make_float2(m.x + iu.x, m.y + iu.y);
  v[2] = make_float2(m.x - iu.x, m.y - iu.y);
}

// In-place-free Stockham passes over RT rows of `pitch` complex values:
// data in `a`, result left in *out (a or b).
FBME_DEV float2* fft_rows(const FftPlan& p, int rt, int pitch, float2* a, float2* b) {
  const int L = p.L;
  int ns = 1;
  for (int ps = 0; ps < p.passes; ++ps) {
    const int R = p.radix[ps];
    const int m = L / R;
    const int stride = L / (ns * R);  // twiddle table step for this pass
    for (int idx = threadIdx.x; idx < rt * m; idx += blockDim.x) {
      const int row = idx / m, j = idx - row * m;
      const float2* src = a + row * pitch;
      float2* dst = b + row * pitch;
      const int k = j % ns;
      float2 v[4];
      for (int r = 0; r < R; ++r) {
        const float2 x = src[j + r * m];
        if (r == 0 || k == 0) {
          v[r] = x;
        } else {
          const float2 w = twiddle(p, static_cast<long long>(r) * k * stride);
          v[r] = cmul(x, w);
        }
      }
      if (R == 4) dft4(v, p.sign);
      else if (R == 2) dft2(v);
      else dft3(v, p.sign);
      const int base = (j / ns) * ns * R + k;
      for (int r = 0; r < R; ++r) dst[base + r * ns] = v[r];
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    ns *= R;
  }
  return a;
}

// Prologue / epilogue of an FFT stage (the stage kernels' policies):
//   mode 0  store                       (EpiStoreT)
//   mode 1  store A^H y, sum |A^H y|^2  (EpiBackprojection, slot 1)
//   mode 2  store p, sum |y - p|^2      (EpiPredict, slot 2; masked)
// and `ysum`: sum |In|^2 of the input rows (ProYPower, slot 3).
//   mode 3  the UAMP denoiser on A^H m in place of storing it (two-pass
//           kernel only): mean, variance, prior and score keys updated as
//           denoise_kernel does, per-tile sums of relevance (slot 0) and
//           variance (slot 1)
struct FftIo {
  const float2* in;
  float2* out;
  const float2* y;        // mode 2: the observations (output layout)
  const uint8_t* mask;    // mode 2: observation mask (or nullptr)
  double* part;
  int mode;
  int ysum;
  DenoiseArgs dn;         // mode 3
};

// The stages of one launch of the two-pass kernel: item i owns the launch's
// tiles [tile0[i], tile0[i + 1]) (one item: a single stage; several: the
// same-length stages of an uneven plan's shape buckets, each computed
// exactly as its own launch computes it).
constexpr int kFftSetMax = 64;
template <int NMAX>
struct FftSet {
  int n;
  int tile0[NMAX + 1];
  FftStage st[NMAX];
  FftIo io[NMAX];
};

template <int NMAX>
FBME_DEV int fft_set_item(const FftSet<NMAX>& set, int t) {
  if constexpr (NMAX == 1) {
    return 0;
  } else {
    int lo = 0, hi = set.n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (set.tile0[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
}

__global__ void __launch_bounds__(kFftThreads) fft_stage_kernel(const FftStage S, const FftIo io) {
  extern __shared__ float2 fsm[];
  const int unit = blockIdx.y, tile = blockIdx.x;
  const int rt = S.p.rows_per_cta, L = S.p.L, pitch = L + 1;
  float2* a = fsm;
  float2* b = fsm + rt * pitch;
  const int r0 = tile * rt;
  const float2* in = io.in + unit * S.in_stride;
  // load rows r0.. (K valid values, zero-padded to L)
  float acc = 0.f;
  for (int idx = threadIdx.x; idx < rt * L; idx += blockDim.x) {
    const int row = idx / L, k = idx - row * L;
    const int r = r0 + row;
    float2 v = make_float2(0.f, 0.f);
    if (r < S.rows && k < S.kin) v = __ldg(in + static_cast<long long>(r) * S.in_ld + k);
    if (io.ysum) acc += abs_sq(v);
    a[row * pitch + k] = v;
  }
  if (io.ysum) {
    const double w = warp_sum(static_cast<double>(acc));
    if ((threadIdx.x & 31) == 0)
      *part_slot(io.part, unit, tile, 3 * kPartWarps + (threadIdx.x >> 5)) = w;
  }
  __syncthreads();
  const float2* res = fft_rows(S.p, rt, pitch, a, b);
  // outputs c < C, row on the contiguous axis
  float2* out = io.out + unit * S.out_stride;
  const float2* ys = io.y ? io.y + unit * S.out_stride : nullptr;
  acc = 0.f;
  for (int idx = threadIdx.x; idx < rt * S.cols; idx += blockDim.x) {
    const int c = idx / rt, row = idx - c * rt;
    const int r = r0 + row;
    if (r >= S.rows) continue;
    const float2 v = res[row * pitch + c];
    const long long o = static_cast<long long>(c) * S.out_ld + r;
    out[o] = v;
    if (io.mode == 1) {
      acc += abs_sq(v);
    } else if (io.mode == 2 && (!io.mask || io.mask[o])) {
      const float2 yy = __ldg(ys + o);
      const float dr = yy.x - v.x, di = yy.y - v.y;
      acc += dr * dr + di * di;
    }
  }
  if (io.mode != 0) {
    const double w = warp_sum(static_cast<double>(acc));
    if ((threadIdx.x & 31) == 0)
      *part_slot(io.part, unit, tile, (io.mode == 1 ? 1 : 2) * kPartWarps + (threadIdx.x >> 5)) = w;
  }
}

// ---------------------------------------------------------------------------
// Register-resident two-pass FFT rows (L >= 32)
// ---------------------------------------------------------------------------
// L = P x Q.  With n = p + P q and k = k1 + Q k2 (p, k2 < P; q, k1 < Q),
//     X[k1 + Q k2] = sum_p w_P^(p k2) [ w_L^(p k1) sum_q x[p + P q] w_Q^(q k1) ],
// so P threads per row each load the Q samples x[p + P q] straight from
// global memory (P consecutive samples per row and q: coalesced), transform
// them in registers (DFT-Q), apply w_L^(p k1) from the FP64-evaluated table
// and exchange through shared memory; each thread then owns the DFT-P of
// ceil(Q / P) output columns k1.  The outputs are staged in shared memory
// and stored with the row on the contiguous axis.  One shared-memory round
// trip per element instead of one per radix pass.
//
// The small DFTs use twiddles that are compile-time constants: cos / sin of
// 2 pi k / n from an octant reduction and Taylor series evaluated in double
// by the compiler, rounded once to float.
constexpr double kPiD = 3.14159265358979323846;

__host__ __device__ constexpr double ct_sin_taylor(double x) {
  double term = x, sum = x;
  for (int i = 1; i < 12; ++i) {
    term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double ct_cos_taylor(double x) {
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 12; ++i) {
    term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    sum += term;
  }
  return sum;
}
struct CtRoot {
  double c, s;
};
// exp(2 pi i k / n) for integers k, n > 0
__host__ __device__ constexpr CtRoot ct_root(int k, int n) {
  k %= n;
  if (k < 0) k += n;
  const int q = (4 * k) / n;    // quarter turns
  const int r = 4 * k - q * n;  // the rest: (pi / 2) r / n, 0 <= r < n
  double c = 0.0, s = 0.0;
  if (2 * r <= n) {
    const double x = 0.5 * kPiD * r / n;
    c = ct_cos_taylor(x);
    s = ct_sin_taylor(x);
  } else {
    const double x = 0.5 * kPiD * (n - r) / n;
    c = ct_sin_taylor(x);
    s = ct_cos_taylor(x);
  }
  if (q == 1) return CtRoot{-s, c};
  if (q == 2) return CtRoot{-c, -s};
  if (q == 3) return CtRoot{s, -c};
  return CtRoot{c, s};
}

// a * exp(S 2 pi i K / N) with the exact rotations done without rounding
template <int N, int S, int K>
FBME_DEV float2 tw_mul(float2 a) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (2 * k == N) {
    return make_float2(-a.x, -a.y);
  } else if constexpr (4 * k == N) {  // S i
    return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
  } else if constexpr (4 * k == 3 * N) {  // -S i
    return S > 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
  } else {
    constexpr CtRoot w = ct_root(k, N);
    constexpr float c = static_cast<float>(w.c);
    constexpr float s = static_cast<float>(S * w.s);
    return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

// In-register DFT of N = 2^a 3^b (b <= 1) values, exponent sign S, natural
// order in and out: radix-4 (else radix-2) decimation in time down to
// DFT-2 / 3 / 4.
template <int N, int S>
struct RegDft {
  template <int K>
  static FBME_DEV void bfly4(float2 (&a)[4][N / 4], float2 (&v)[N]) {
    float2 b[4] = {a[0][K], tw_mul<N, S, K>(a[1][K]), tw_mul<N, S, 2 * K>(a[2][K]),
                   tw_mul<N, S, 3 * K>(a[3][K])};
    dft4(b, static_cast<float>(S));
    v[K] = b[0];
    v[K + N / 4] = b[1];
    v[K + N / 2] = b[2];
    v[K + 3 * N / 4] = b[3];
  }
  template <int K>
  static FBME_DEV void bfly2(float2 (&a)[2][N / 2], float2 (&v)[N]) {
    float2 b[2] = {a[0][K], tw_mul<N, S, K>(a[1][K])};
    dft2(b);
    v[K] = b[0];
    v[K + N / 2] = b[1];
  }
  template <int... K>
  static FBME_DEV void combine4(float2 (&a)[4][N / 4], float2 (&v)[N], std::integer_sequence<int, K...>) {
    (bfly4<K>(a, v), ...);
  }
  template <int... K>
  static FBME_DEV void combine2(float2 (&a)[2][N / 2], float2 (&v)[N], std::integer_sequence<int, K...>) {
    (bfly2<K>(a, v), ...);
  }
  static FBME_DEV void run(float2 (&v)[N]) {
    if constexpr (N == 2) {
      dft2(v);
    } else if constexpr (N == 3) {
      dft3(v, static_cast<float>(S));
    } else if constexpr (N == 4) {
      dft4(v, static_cast<float>(S));
    } else if constexpr (N % 4 == 0) {
      float2 a[4][N / 4];
#pragma unroll
      for (int j = 0; j < N / 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) a[r][j] = v[4 * j + r];
      RegDft<N / 4, S>::run(a[0]);
      RegDft<N / 4, S>::run(a[1]);
      RegDft<N / 4, S>::run(a[2]);
      RegDft<N / 4, S>::run(a[3]);
      combine4(a, v, std::make_integer_sequence<int, N / 4>{});
    } else {
      static_assert(N % 2 == 0, "RegDft: N must be 2^a 3^b with b <= 1");
      float2 a[2][N / 2];
#pragma unroll
      for (int j = 0; j < N / 2; ++j) {
        a[0][j] = v[2 * j];
        a[1][j] = v[2 * j + 1];
      }
      RegDft<N / 2, S>::run(a[0]);
      RegDft<N / 2, S>::run(a[1]);
      combine2(a, v, std::make_integer_sequence<int, N / 2>{});
    }
  }
};

// Threads per row P of the two-pass kernel for a length L (0: not built)
__host__ __device__ constexpr int fast_threads_per_row(int L) {
  return L == 512 || L == 384 || L == 256 ? 16 : L == 192 || L == 128 || L == 96 || L == 64 ? 8
                                                 : L == 48 || L == 32 ? 4 : 0;
}
// Complex values of one row's area: at least Q (P + 2) for the exchange
// (column k1 at k1 (P + 2): 16-byte aligned for the pass-2 vector reads,
// whose 8-lane phases then fall on distinct banks) and L + ROWS for the
// output staging (row lr stages its outputs at offset lr, so that the ROWS
// rows read in one pass fall on distinct banks), and = P mod 16 so that the
// 16 / P rows served in one 64-bit shared-memory phase of the exchange fall
// on disjoint banks.
__host__ __device__ constexpr int fast_row_area(int L) {
  const int P = fast_threads_per_row(L), Q = L / P, ROWS = kFftThreads / P;
  int a = Q * (P + 2) > L + ROWS ? Q * (P + 2) : L + ROWS;
  while (a % 16 != P % 16) ++a;
  return a;
}
// two buffers of ROWS rows (the input rows, then in place the exchange
// and the output staging)
constexpr size_t fast_smem_bytes(int L) {
  return 2 * static_cast<size_t>(kFftThreads / fast_threads_per_row(L)) * fast_row_area(L) * sizeof(float2);
}

FBME_DEV void cp_async8(float2* dst, const float2* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
FBME_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
FBME_DEV void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
template <int N>
FBME_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Asynchronous copy of the values thread (lr, p) transforms in tile t:
// x[p + P q] of row lr with p + P q < K (the rest of the row is zero and is
// never copied); one commit group.
template <int L>
FBME_DEV void fast_issue(const FftStage& st, const FftIo& io, int t, float2* buf, int lr, int p) {  // t: the item's tile
  constexpr int P = fast_threads_per_row(L), Q = L / P, ROWS = kFftThreads / P, A = fast_row_area(L);
  const int unit = t / st.tiles, tile = t - unit * st.tiles;
  const int r = tile * ROWS + lr;
  if (r < st.rows) {
    const float2* src = io.in + unit * st.in_stride + static_cast<long long>(r) * st.in_ld + p;
    float2* dst = buf + lr * A + p;
#pragma unroll
    for (int q = 0; q < Q; ++q)
      if (p + P * q < st.kin) cp_async8(dst + P * q, src + P * q);
  }
  cp_async_commit();
}

// Persistent: CTA b takes tiles b, b + gridDim.x, ... (tile t = unit x
// tiles + row tile); the copy of its next tile is in flight while the
// current one is transformed.
// EPI: 0 store (modes 0 and 1), 1 residual (mode 2), 2 denoiser (mode 3)
template <int L, int S, int EPI>
__global__ void __launch_bounds__(kFftThreads, 2) fft_fast_kernel(const FftStage st, const FftIo io) {
  constexpr int P = fast_threads_per_row(L), Q = L / P, ROWS = kFftThreads / P;
  constexpr int J = (Q + P - 1) / P;     // output columns k1 per thread in pass 2
  constexpr int A = fast_row_area(L);    // row stride of a buffer
  constexpr int BUF = ROWS * A;
  extern __shared__ float2 fsm[];
  const int lr = threadIdx.x / P, p = threadIdx.x % P;
  const int total = st.tiles * st.units;
  int t = blockIdx.x;
  if (t < total) fast_issue<L>(st, io, t, fsm, lr, p);
  for (int it = 0; t < total; ++it, t += gridDim.x) {
    float2* buf = fsm + (it & 1) * BUF;
    if (t + static_cast<int>(gridDim.x) < total)
      fast_issue<L>(st, io, t + gridDim.x, fsm + ((it + 1) & 1) * BUF, lr, p);
    else
      cp_async_commit();  // empty group: the wait below counts the same
    if constexpr (EPI != 0) {
      // the next tile's epilogue operands (observations; prior, mean and
      // variance) into L2, one line per output column and array, so their
      // DRAM reads overlap this tile's transform
      const int tn = t + gridDim.x;
      if (tn < total) {
        const int un = tn / st.tiles;
        const long long bn = un * st.out_stride + static_cast<long long>(tn - un * st.tiles) * ROWS;
        for (int c = threadIdx.x; c < st.cols; c += kFftThreads) {
          const long long o = bn + static_cast<long long>(c) * st.out_ld;
          if constexpr (EPI == 1) {
            prefetch_l2(io.y + o);
          } else {
            prefetch_l2(io.dn.gamma + o);
            prefetch_l2(io.dn.mu + o);
            prefetch_l2(io.dn.var + o);
          }
        }
      }
    }
    cp_async_wait<1>();   // this thread's copies of tile t (it reads only its own)
    const int unit = t / st.tiles, tile = t - unit * st.tiles;
    const int r0 = tile * ROWS;
    const bool live = r0 + lr < st.rows;
    float2* ya = buf + lr * A;

    // pass 1: DFT-Q of x[p + P q] in registers
    float2 v[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
      v[q] = (live && p + P * q < st.kin) ? ya[p + P * q] : make_float2(0.f, 0.f);
    if (io.ysum) {
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q < Q; ++q) acc += abs_sq(v[q]);
      const double w = warp_sum(static_cast<double>(acc));
      if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 3 * kPartWarps + (threadIdx.x >> 5)) = w;
    }
    __syncwarp();  // the row's inputs are read before the exchange overwrites them
    RegDft<Q, S>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < Q; ++k1) {
      float2 y = v[k1];
      if (k1 > 0) {  // w_L^(p k1), stored at k1 P + p
        const float2 w = __ldg(st.p.tw + k1 * P + p);
        y = cmul(y, S < 0 ? w : make_float2(w.x, -w.y));
      }
      ya[k1 * (P + 2) + p] = y;
    }
    __syncwarp();

    // pass 2: DFT-P over p for the columns k1 = p + j P
    float2 u[J][P];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k1 = p + j * P;
      if (Q % P == 0 || k1 < Q) {
        const float4* col = reinterpret_cast<const float4*>(ya + k1 * (P + 2));
#pragma unroll
        for (int pp = 0; pp < P / 2; ++pp) {
          const float4 t = col[pp];
          u[j][2 * pp] = make_float2(t.x, t.y);
          u[j][2 * pp + 1] = make_float2(t.z, t.w);
        }
        RegDft<P, S>::run(u[j]);
      }
    }
    __syncwarp();  // the row's exchange values are read before its staging overwrites them
    float2* xo = ya + lr;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k1 = p + j * P;
      if (Q % P == 0 || k1 < Q) {
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) {
          const int c = k1 + Q * k2;
          if (c < st.cols) xo[c] = u[j][k2];
        }
      }
    }

    // outputs c < C, row on the contiguous axis: thread (c0, row) handles
    // columns c0 + P i (i < L / P) of row r0 + row (ROWS consecutive rows).
    // The epilogue's other operands (the residual's observations and mask
    // bits, the denoiser's prior, mean and variance) are loaded a chunk of
    // CH columns ahead, the first chunk before the barrier, so that their
    // latency overlaps it.
    constexpr int NC = L / P;
    constexpr int CH = NC <= 16 ? NC : (NC % 16 == 0 ? 16 : 8);
    const int row = threadIdx.x % ROWS, c0 = threadIdx.x / ROWS;
    const int rr = r0 + row;
    const bool live_out = rr < st.rows;
    const long long base = unit * st.out_stride;
    const long long o0 = static_cast<long long>(c0) * st.out_ld + rr;
    const long long step = static_cast<long long>(P) * st.out_ld;
    const float2* sp = buf + row * A + row;
    if constexpr (EPI == 0) {
      __syncthreads();
      float acc = 0.f;
      if (live_out) {
        long long o = base + o0;
        for (int c = c0; c < st.cols; c += P, o += step) {
          const float2 x = sp[c];
          io.out[o] = x;
          if (io.mode == 1) acc += abs_sq(x);
        }
      }
      if (io.mode == 1) {
        const double w = warp_sum(static_cast<double>(acc));
        if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 1 * kPartWarps + (threadIdx.x >> 5)) = w;
      }
    } else if constexpr (EPI == 1) {
      float2 yv[CH];
      uint32_t obs = 0;
      auto load_chunk = [&](int g) {
        obs = 0;
        if (live_out) {
#pragma unroll
          for (int i = 0; i < CH; ++i) {
            const int ii = g * CH + i;
            const long long o = o0 + ii * step;
            if (c0 + P * ii < st.cols && (!io.mask || io.mask[o])) {
              yv[i] = __ldg(io.y + base + o);
              obs |= 1u << i;
            }
          }
        }
      };
      load_chunk(0);
      __syncthreads();
      float acc = 0.f;
#pragma unroll
      for (int g = 0; g < NC / CH; ++g) {
        if (g > 0) load_chunk(g);
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          const int ii = g * CH + i;
          const int c = c0 + P * ii;
          if (live_out && c < st.cols) {
            const float2 x = sp[c];
            io.out[base + o0 + ii * step] = x;
            if (obs >> i & 1u) {
              const float dr = yv[i].x - x.x, di = yv[i].y - x.y;
              acc += dr * dr + di * di;
            }
          }
        }
      }
      const double w = warp_sum(static_cast<double>(acc));
      if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 2 * kPartWarps + (threadIdx.x >> 5)) = w;
    } else {
      // four registers a column: chunks of at most 8 columns
      constexpr int CD = NC % 8 == 0 ? 8 : (NC % 4 == 0 ? 4 : NC);
      const DenoiseArgs& dn = io.dn;
      float gv[CD], vv[CD];
      float2 mv[CD];
      auto load_chunk = [&](int g) {
        if (live_out) {
#pragma unroll
          for (int i = 0; i < CD; ++i) {
            const int ii = g * CD + i;
            if (c0 + P * ii < st.cols) {
              const long long o = base + o0 + ii * step;
              gv[i] = dn.gamma[o];
              mv[i] = dn.mu[o];
              vv[i] = dn.var[o];
            }
          }
        }
      };
      load_chunk(0);
      __syncthreads();
      const float pv = dn.pv[unit], fl = dn.floor_[unit];
      float dof = 0.f, sv = 0.f;
#pragma unroll
      for (int g = 0; g < NC / CD; ++g) {
        if (g > 0) load_chunk(g);
#pragma unroll
        for (int i = 0; i < CD; ++i) {
          const int ii = g * CD + i;
          const int c = c0 + P * ii;
          if (live_out && c < st.cols) {
            const DenoiseOut r = denoise_math(dn, gv[i], mv[i], vv[i], sp[c], pv, fl);
            const long long o = base + o0 + ii * step;
            dn.mu[o] = r.mean;
            dn.var[o] = r.variance;
            if (dn.update_prior) dn.gamma[o] = r.gamma;
            if (dn.keys) dn.keys[o] = float_key(abs_sq(r.mean) + r.variance);
            dof += r.rel;
            sv += r.variance;
          }
        }
      }
      const double w0 = warp_sum(static_cast<double>(dof));
      const double w1 = warp_sum(static_cast<double>(sv));
      if ((threadIdx.x & 31) == 0) {
        *part_slot(io.part, unit, tile, 0 * kPartWarps + (threadIdx.x >> 5)) = w0;
        *part_slot(io.part, unit, tile, 1 * kPartWarps + (threadIdx.x >> 5)) = w1;
      }
    }
    __syncthreads();  // this buffer takes the copy issued at the top of the next tile
  }
  cp_async_wait<0>();
}

// The same kernel over a set of same-length stages (uneven plans' shape
// buckets): tile t belongs to the item whose tile range holds it, and is
// computed exactly as that item's own launch computes it.  A separate
// kernel, so that the single-stage kernel keeps its code.
template <int L, int S, int EPI, int NMAX>
__global__ void __launch_bounds__(kFftThreads, 2) fft_fast_set_kernel(const FftSet<NMAX> set) {
  constexpr int P = fast_threads_per_row(L), Q = L / P, ROWS = kFftThreads / P;
  constexpr int J = (Q + P - 1) / P;     // output columns k1 per thread in pass 2
  constexpr int A = fast_row_area(L);    // row stride of a buffer
  constexpr int BUF = ROWS * A;
  extern __shared__ float2 fsm[];
  const int lr = threadIdx.x / P, p = threadIdx.x % P;
  const int total = set.tile0[set.n];
  int t = blockIdx.x;
  if (t < total) {
    const int i = fft_set_item(set, t);
    fast_issue<L>(set.st[i], set.io[i], t - set.tile0[i], fsm, lr, p);
  }
  for (int it = 0; t < total; ++it, t += gridDim.x) {
    const int item = fft_set_item(set, t);
    const FftStage& st = set.st[item];
    const FftIo& io = set.io[item];
    float2* buf = fsm + (it & 1) * BUF;
    const int tn = t + gridDim.x;
    if (tn < total) {
      const int in_ = fft_set_item(set, tn);
      const FftStage& sn = set.st[in_];
      const int tl = tn - set.tile0[in_];
      fast_issue<L>(sn, set.io[in_], tl, fsm + ((it + 1) & 1) * BUF, lr, p);
      if constexpr (EPI != 0) {
        // the next tile's epilogue operands (observations; prior, mean and
        // variance) into L2, one line per output column and array, so their
        // DRAM reads overlap this tile's transform
        const FftIo& ion = set.io[in_];
        const int un = tl / sn.tiles;
        const long long bn = un * sn.out_stride + static_cast<long long>(tl - un * sn.tiles) * ROWS;
        for (int c = threadIdx.x; c < sn.cols; c += kFftThreads) {
          const long long o = bn + static_cast<long long>(c) * sn.out_ld;
          if constexpr (EPI == 1) {
            prefetch_l2(ion.y + o);
          } else {
            prefetch_l2(ion.dn.gamma + o);
            prefetch_l2(ion.dn.mu + o);
            prefetch_l2(ion.dn.var + o);
          }
        }
      }
    } else {
      cp_async_commit();  // empty group: the wait below counts the same
    }
    cp_async_wait<1>();   // this thread's copies of tile t (it reads only its own)
    const int tloc = t - set.tile0[item];
    const int unit = tloc / st.tiles, tile = tloc - unit * st.tiles;
    const int r0 = tile * ROWS;
    const bool live = r0 + lr < st.rows;
    float2* ya = buf + lr * A;

    // pass 1: DFT-Q of x[p + P q] in registers
    float2 v[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q)
      v[q] = (live && p + P * q < st.kin) ? ya[p + P * q] : make_float2(0.f, 0.f);
    if (io.ysum) {
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q < Q; ++q) acc += abs_sq(v[q]);
      const double w = warp_sum(static_cast<double>(acc));
      if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 3 * kPartWarps + (threadIdx.x >> 5)) = w;
    }
    __syncwarp();  // the row's inputs are read before the exchange overwrites them
    RegDft<Q, S>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < Q; ++k1) {
      float2 y = v[k1];
      if (k1 > 0) {  // w_L^(p k1), stored at k1 P + p
        const float2 w = __ldg(st.p.tw + k1 * P + p);
        y = cmul(y, S < 0 ? w : make_float2(w.x, -w.y));
      }
      ya[k1 * (P + 2) + p] = y;
    }
    __syncwarp();

    // pass 2: DFT-P over p for the columns k1 = p + j P
    float2 u[J][P];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k1 = p + j * P;
      if (Q % P == 0 || k1 < Q) {
        const float4* col = reinterpret_cast<const float4*>(ya + k1 * (P + 2));
#pragma unroll
        for (int pp = 0; pp < P / 2; ++pp) {
          const float4 t = col[pp];
          u[j][2 * pp] = make_float2(t.x, t.y);
          u[j][2 * pp + 1] = make_float2(t.z, t.w);
        }
        RegDft<P, S>::run(u[j]);
      }
    }
    __syncwarp();  // the row's exchange values are read before its staging overwrites them
    float2* xo = ya + lr;
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int k1 = p + j * P;
      if (Q % P == 0 || k1 < Q) {
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) {
          const int c = k1 + Q * k2;
          if (c < st.cols) xo[c] = u[j][k2];
        }
      }
    }

    // outputs c < C, row on the contiguous axis: thread (c0, row) handles
    // columns c0 + P i (i < L / P) of row r0 + row (ROWS consecutive rows).
    // The epilogue's other operands (the residual's observations and mask
    // bits, the denoiser's prior, mean and variance) are loaded a chunk of
    // CH columns ahead, the first chunk before the barrier, so that their
    // latency overlaps it.
    constexpr int NC = L / P;
    constexpr int CH = NC <= 16 ? NC : (NC % 16 == 0 ? 16 : 8);
    const int row = threadIdx.x % ROWS, c0 = threadIdx.x / ROWS;
    const int rr = r0 + row;
    const bool live_out = rr < st.rows;
    const long long base = unit * st.out_stride;
    const long long o0 = static_cast<long long>(c0) * st.out_ld + rr;
    const long long step = static_cast<long long>(P) * st.out_ld;
    const float2* sp = buf + row * A + row;
    if constexpr (EPI == 0) {
      __syncthreads();
      float acc = 0.f;
      if (live_out) {
        long long o = base + o0;
        for (int c = c0; c < st.cols; c += P, o += step) {
          const float2 x = sp[c];
          io.out[o] = x;
          if (io.mode == 1) acc += abs_sq(x);
        }
      }
      if (io.mode == 1) {
        const double w = warp_sum(static_cast<double>(acc));
        if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 1 * kPartWarps + (threadIdx.x >> 5)) = w;
      }
    } else if constexpr (EPI == 1) {
      float2 yv[CH];
      uint32_t obs = 0;
      auto load_chunk = [&](int g) {
        obs = 0;
        if (live_out) {
#pragma unroll
          for (int i = 0; i < CH; ++i) {
            const int ii = g * CH + i;
            const long long o = o0 + ii * step;
            if (c0 + P * ii < st.cols && (!io.mask || io.mask[o])) {
              yv[i] = __ldg(io.y + base + o);
              obs |= 1u << i;
            }
          }
        }
      };
      load_chunk(0);
      __syncthreads();
      float acc = 0.f;
#pragma unroll
      for (int g = 0; g < NC / CH; ++g) {
        if (g > 0) load_chunk(g);
#pragma unroll
        for (int i = 0; i < CH; ++i) {
          const int ii = g * CH + i;
          const int c = c0 + P * ii;
          if (live_out && c < st.cols) {
            const float2 x = sp[c];
            io.out[base + o0 + ii * step] = x;
            if (obs >> i & 1u) {
              const float dr = yv[i].x - x.x, di = yv[i].y - x.y;
              acc += dr * dr + di * di;
            }
          }
        }
      }
      const double w = warp_sum(static_cast<double>(acc));
      if ((threadIdx.x & 31) == 0) *part_slot(io.part, unit, tile, 2 * kPartWarps + (threadIdx.x >> 5)) = w;
    } else {
      // four registers a column: chunks of at most 8 columns
      constexpr int CD = NC % 8 == 0 ? 8 : (NC % 4 == 0 ? 4 : NC);
      const DenoiseArgs& dn = io.dn;
      float gv[CD], vv[CD];
      float2 mv[CD];
      auto load_chunk = [&](int g) {
        if (live_out) {
#pragma unroll
          for (int i = 0; i < CD; ++i) {
            const int ii = g * CD + i;
            if (c0 + P * ii < st.cols) {
              const long long o = base + o0 + ii * step;
              gv[i] = dn.gamma[o];
              mv[i] = dn.mu[o];
              vv[i] = dn.var[o];
            }
          }
        }
      };
      load_chunk(0);
      __syncthreads();
      const float pv = dn.pv[unit], fl = dn.floor_[unit];
      float dof = 0.f, sv = 0.f;
#pragma unroll
      for (int g = 0; g < NC / CD; ++g) {
        if (g > 0) load_chunk(g);
#pragma unroll
        for (int i = 0; i < CD; ++i) {
          const int ii = g * CD + i;
          const int c = c0 + P * ii;
          if (live_out && c < st.cols) {
            const DenoiseOut r = denoise_math(dn, gv[i], mv[i], vv[i], sp[c], pv, fl);
            const long long o = base + o0 + ii * step;
            dn.mu[o] = r.mean;
            dn.var[o] = r.variance;
            if (dn.update_prior) dn.gamma[o] = r.gamma;
            if (dn.keys) dn.keys[o] = float_key(abs_sq(r.mean) + r.variance);
            dof += r.rel;
            sv += r.variance;
          }
        }
      }
      const double w0 = warp_sum(static_cast<double>(dof));
      const double w1 = warp_sum(static_cast<double>(sv));
      if ((threadIdx.x & 31) == 0) {
        *part_slot(io.part, unit, tile, 0 * kPartWarps + (threadIdx.x >> 5)) = w0;
        *part_slot(io.part, unit, tile, 1 * kPartWarps + (threadIdx.x >> 5)) = w1;
      }
    }
    __syncthreads();  // this buffer takes the copy issued at the top of the next tile
  }
  cp_async_wait<0>();
}

template <int L, int S, int EPI>
void launch_fast_as(const FftStage& S_, const FftIo& io, cudaStream_t st) {
  auto kern = fft_fast_kernel<L, S, EPI>;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFftThreads, fast_smem_bytes(L)) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long total = static_cast<long long>(S_.tiles) * S_.units;
  const long long cap = static_cast<long long>(sm_count()) * per_sm;
  const int grid = static_cast<int>(total < cap ? total : cap);
  if (grid > 0) kern<<<grid, kFftThreads, fast_smem_bytes(L), st>>>(S_, io);
}

template <int L, int S, int EPI>
void launch_fast_set_as(const FftSet<kFftSetMax>& set, cudaStream_t st) {
  auto kern = fft_fast_set_kernel<L, S, EPI, kFftSetMax>;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kFftThreads, fast_smem_bytes(L)) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long total = set.tile0[set.n];
  const long long cap = static_cast<long long>(sm_count()) * per_sm;
  const int grid = static_cast<int>(total < cap ? total : cap);
  if (grid > 0) kern<<<grid, kFftThreads, fast_smem_bytes(L), st>>>(set);
}

// Forward stages store or take the residual; adjoint stages store or run
// the denoiser (the combinations the UAMP sweeps use).
template <int L>
void launch_fast(const FftStage& S, const FftIo& io, int sign, cudaStream_t st) {
  if (sign < 0) {
    if (io.mode == 2) launch_fast_as<L, -1, 1>(S, io, st);
    else launch_fast_as<L, -1, 0>(S, io, st);
  } else {
    if (io.mode == 3) launch_fast_as<L, 1, 2>(S, io, st);
    else launch_fast_as<L, 1, 0>(S, io, st);
  }
}
template <int L>
void launch_fast_set(const FftSet<kFftSetMax>& set, int sign, int mode, cudaStream_t st) {
  if (sign < 0) {
    if (mode == 2) launch_fast_set_as<L, -1, 1>(set, st);
    else launch_fast_set_as<L, -1, 0>(set, st);
  } else {
    if (mode == 3) launch_fast_set_as<L, 1, 2>(set, st);
    else launch_fast_set_as<L, 1, 0>(set, st);
  }
}

template <typename K>
cudaError_t smem_attr(K kern, int bytes) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <int L>
cudaError_t set_fast_attr() {
  const int bytes = static_cast<int>(fast_smem_bytes(L));
  cudaError_t e = smem_attr(fft_fast_kernel<L, -1, 0>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_kernel<L, -1, 1>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_kernel<L, 1, 0>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_kernel<L, 1, 2>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_set_kernel<L, -1, 0, kFftSetMax>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_set_kernel<L, -1, 1, kFftSetMax>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_set_kernel<L, 1, 0, kFftSetMax>, bytes);
  if (e == cudaSuccess) e = smem_attr(fft_fast_set_kernel<L, 1, 2, kFftSetMax>, bytes);
  return e;
}

}  // namespace

// Radix plan of a length L = 2^a 3^b (b <= 1, L <= 512), 0 when L has
// another factor.
int fft_length_ok(int L) {
  if (L < 2 || L > 512) return 0;
  int v = L;
  if (v % 3 == 0) v /= 3;
  return (v & (v - 1)) == 0 ? 1 : 0;
}

static FftPlan make_plan(int L, int sign, const float2* tw) {
  FftPlan p{};
  p.L = L;
  p.sign = static_cast<float>(sign);
  p.tw = tw;
  int v = L;
  while (v % 4 == 0) {
    p.radix[p.passes++] = 4;
    v /= 4;
  }
  if (v % 2 == 0) {
    p.radix[p.passes++] = 2;
    v /= 2;
  }
  if (v % 3 == 0) {
    p.radix[p.passes++] = 3;
    v /= 3;
  }
  int rt = 4096 / L;
  int pow2 = 1;
  while (pow2 * 2 <= rt) pow2 *= 2;
  p.rows_per_cta = pow2 < 1 ? 1 : pow2;
  return p;
}

int fft_rows_per_cta(int L) {
  const int P = fast_threads_per_row(L);
  return P ? kFftThreads / P : make_plan(L, -1, nullptr).rows_per_cta;
}

size_t fft_smem_bytes(int L) {
  return static_cast<size_t>(2) * fft_rows_per_cta(L) * (L + 1) * sizeof(float2);
}

cudaError_t set_fft_attributes() {
  // the largest footprint over the supported lengths (short rows pack more
  // of them to a CTA: L = 2 needs 96 KB)
  size_t most = 0;
  for (int L = 2; L <= 512; ++L)
    if (fft_length_ok(L) && fft_smem_bytes(L) > most) most = fft_smem_bytes(L);
  cudaError_t e = cudaFuncSetAttribute(fft_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(most));
  if (e == cudaSuccess) e = set_fast_attr<512>();
  if (e == cudaSuccess) e = set_fast_attr<384>();
  if (e == cudaSuccess) e = set_fast_attr<256>();
  if (e == cudaSuccess) e = set_fast_attr<192>();
  if (e == cudaSuccess) e = set_fast_attr<128>();
  if (e == cudaSuccess) e = set_fast_attr<96>();
  if (e == cudaSuccess) e = set_fast_attr<64>();
  if (e == cudaSuccess) e = set_fast_attr<48>();
  if (e == cudaSuccess) e = set_fast_attr<32>();
  return e;
}

// One FFT stage of `units` transforms (the geometry of the GEMM stage `g`,
// whose contracted length K is padded to the transform length L).
// The fused denoiser epilogue pays where two CTAs fit on an SM; at L = 512
// (one CTA of 147 KB) its loads find too few warps, and the elementwise
// denoiser at full occupancy is faster.
int fft_denoise_fused(int L) { return fast_threads_per_row(L) != 0 && L < 512; }

static FftStage fft_stage_of(const DftGeom& g, int L, int sign, const float2* tw) {
  FftStage S;
  S.p = make_plan(L, sign, tw);
  S.rows = g.rows;
  S.kin = g.kcplx;
  S.cols = g.cols;
  S.in_ld = g.in_ld;
  S.out_ld = g.out_ld;
  S.in_stride = g.in_stride;
  S.out_stride = g.out_stride;
  S.tiles = ceil_div(g.rows, fft_rows_per_cta(L));
  S.units = g.n_scenes;
  return S;
}

static void launch_fast_set_len(const FftSet<kFftSetMax>& set, int L, int sign, int mode, cudaStream_t st) {
  switch (L) {
    case 512: launch_fast_set<512>(set, sign, mode, st); return;
    case 384: launch_fast_set<384>(set, sign, mode, st); return;
    case 256: launch_fast_set<256>(set, sign, mode, st); return;
    case 192: launch_fast_set<192>(set, sign, mode, st); return;
    case 128: launch_fast_set<128>(set, sign, mode, st); return;
    case 96: launch_fast_set<96>(set, sign, mode, st); return;
    case 64: launch_fast_set<64>(set, sign, mode, st); return;
    case 48: launch_fast_set<48>(set, sign, mode, st); return;
    case 32: launch_fast_set<32>(set, sign, mode, st); return;
    default: return;
  }
}

void fft_stage(const DftGeom& g, int L, int sign, const float2* tw, const float2* in, float2* out,
               const float2* y, const uint8_t* mask, double* part, int mode, int ysum, cudaStream_t st,
               const DenoiseArgs* dn) {
  const FftStage S = fft_stage_of(g, L, sign, tw);
  FftIo io{in, out, y, mask, part, mode, ysum};
  if (dn) io.dn = *dn;
  switch (L) {
    case 512: launch_fast<512>(S, io, sign, st); return;
    case 384: launch_fast<384>(S, io, sign, st); return;
    case 256: launch_fast<256>(S, io, sign, st); return;
    case 192: launch_fast<192>(S, io, sign, st); return;
    case 128: launch_fast<128>(S, io, sign, st); return;
    case 96: launch_fast<96>(S, io, sign, st); return;
    case 64: launch_fast<64>(S, io, sign, st); return;
    case 48: launch_fast<48>(S, io, sign, st); return;
    case 32: launch_fast<32>(S, io, sign, st); return;
    default: break;
  }
  fft_stage_kernel<<<dim3(S.tiles, g.n_scenes), kFftThreads, fft_smem_bytes(L), st>>>(S, io);
}

// The same-length stages of several shape buckets in one launch of the
// two-pass kernel where L has it (fft_set_length_ok).  Each item is
// computed as fft_stage computes it alone.
int fft_set_length_ok(int L) { return fast_threads_per_row(L) != 0; }

void fft_stage_set(const FftSetJob* jobs, int n, int L, int sign, int mode, cudaStream_t st) {
  if (!fft_set_length_ok(L)) {
    // lengths without the two-pass kernel (below 32): one Stockham launch
    // per bucket, as fft_stage runs it
    for (int i = 0; i < n; ++i) {
      const FftSetJob& j = jobs[i];
      fft_stage(j.g, L, sign, j.tw, j.in, j.out, j.y, j.mask, j.part, mode, j.ysum, st, j.dn);
    }
    return;
  }
  for (int j0 = 0; j0 < n; j0 += kFftSetMax) {
    const int cnt = n - j0 < kFftSetMax ? n - j0 : kFftSetMax;
    FftSet<kFftSetMax> set;
    set.n = cnt;
    set.tile0[0] = 0;
    for (int i = 0; i < cnt; ++i) {
      const FftSetJob& j = jobs[j0 + i];
      set.st[i] = fft_stage_of(j.g, L, sign, j.tw);
      set.io[i] = FftIo{j.in, j.out, j.y, j.mask, j.part, mode, j.ysum};
      if (mode == 3) set.io[i].dn = *j.dn;
      set.tile0[i + 1] = set.tile0[i] + set.st[i].tiles * set.st[i].units;
    }
    launch_fast_set_len(set, L, sign, mode, st);
  }
}

int fft_stage_tiles(int rows, int L) { return ceil_div(rows, fft_rows_per_cta(L)); }

namespace {
// The twiddles of one transform length, FP64-evaluated: for the two-pass
// kernel (P threads per row) entry k1 P + p is w_L^(p k1), so that the P
// threads of a row read one contiguous run per k1; for the Stockham kernel
// entry k is w_L^k.
__global__ void fft_twiddle_kernel(float2* dst, int L, int P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= L) return;
  const int e = P ? ((i % P) * (i / P)) % L : i;
  double s, c;
  sincospi(-2.0 * static_cast<double>(e) / static_cast<double>(L), &s, &c);
  dst[i] = make_float2(static_cast<float>(c), static_cast<float>(s));
}
}  // namespace

void launch_fft_twiddles(float2* dst, int L, cudaStream_t st) {
  fft_twiddle_kernel<<<(L + 255) / 256, 256, 0, st>>>(dst, L, fast_threads_per_row(L));
}

}  // namespace fbme
