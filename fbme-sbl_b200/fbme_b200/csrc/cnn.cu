// Learned warm start: a 3-layer 3x3 convolutional network on the
// reconstruction grid that predicts the initial log prior variance of a
// scene from its backprojection A^H y (no counterpart in the reference; it
// replaces the initial prior of torch_sbl/solver.py:1072-1099).
//
//   x   = features(A^H y)                       [B][H][W][8]  BF16 (2 used)
//   h1  = relu(conv(x, W1) + b1)                [B][H][W][8]  BF16
//   h2  = relu(conv(h1, W2) + b2)               [B][H][W][8]  BF16
//   out = conv(h2, W3) + b3                     [B][H][W]     FP32
//   prior0 = max(data_power / N * exp(out), floor)
//
// The forward pass (training and inference) is one kernel per 32 x 32
// output tile with all three layers on the tensor cores (mma.sync, BF16
// operands, FP32 accumulation; net_tile_kernel below).  The backward pass's
// input gradients are the same convolutions with flipped, transposed
// weights, as implicit GEMMs on the tensor cores (M = 16 pixels of one tile
// row, N = 8 output channels, K = (tap, input channel) with the channel
// fastest, so an operand pair is one 32-bit load from the NHWC tile in
// shared memory); the weight gradient is a reduction over pixels on the
// CUDA cores with fixed-order block partials.  Parameters are an FP32
// master vector; the kernels round them to BF16 where they read them.
#include <cuda_bf16.h>
#include <type_traits>
#include <math.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace fbme {
namespace cnn {

constexpr int kHid = 8;    // hidden channels
constexpr int kInP = 8;    // input feature channels, padded (2 used)
constexpr int kIn = 2;
constexpr int kTileH = 8, kTileW = 16;
constexpr int kConvThreads = 128;

__host__ __device__ constexpr int kpad(int cin) { return (9 * cin + 15) / 16 * 16; }

// FP32 master parameter layout: W[dy][dx][ci][co] then bias, per layer.
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + 9 * kIn * kHid;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + 9 * kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + 9 * kHid;
constexpr int kNParams = kOffB3 + 1;

constexpr int kK2 = kpad(kHid);   // 80: (tap, channel) of an 8-channel input, padded
constexpr int kKb3 = kpad(8);     // 80: layer-3 backward, input = 8 padded gradient channels

// BF16 operand matrices [Cout][K] of the backward pass's input gradients.
struct Packed {
  __nv_bfloat16* wb3;  // [8][80]  d h2 = conv(d out, W3 flipped)
  __nv_bfloat16* wb2;  // [8][80]  d h1 = conv(d a2, W2 flipped)
};

__global__ void pack_kernel(const float* p, Packed P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * kK2) {
    // row = input channel of the forward layer 2, column k = (flipped tap, its output channel)
    const int cin2 = i / kK2, k = i % kK2, tap = k / kHid, cout2 = k % kHid;
    const float v = k < 9 * kHid ? p[kOffW2 + ((8 - tap) * kHid + cin2) * kHid + cout2] : 0.f;
    P.wb2[i] = __float2bfloat16_rn(v);
  }
  if (i < kHid * kKb3) {
    const int ci = i / kKb3, k = i % kKb3, tap = k / 8, co = k % 8;
    const float v = (k < 72 && co == 0) ? p[kOffW3 + (8 - tap) * kHid + ci] : 0.f;
    P.wb3[i] = __float2bfloat16_rn(v);
  }
}

// Sum of a scene's n <= 64 FP64 feature partials p[0..n) in one fixed
// order (two per lane, then the warp butterfly); every lane of the calling
// warp returns the same value, so all kernels that read the partials agree.
FBME_DEV double parts_sum(const double* p, int n) {
  const int lane = threadIdx.x & 31;
  const double v = (lane < n ? p[lane] : 0.0) + (lane + 32 < n ? p[lane + 32] : 0.0);
  return warp_sum(v);
}

FBME_DEV uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

FBME_DEV void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                             uint32_t b0, uint32_t b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Two channels (c, c+1) of pixel e of an NHWC tensor as a BF16 pair.
FBME_DEV uint32_t load_pair(const __nv_bfloat16* x, long long e) {
  return *reinterpret_cast<const uint32_t*>(x + e);
}
FBME_DEV uint32_t load_pair(const float* x, long long e) {
  const float2 v = *reinterpret_cast<const float2*>(x + e);
  return pack_bf16x2(v.x, v.y);
}

enum OutMode { kOutReluBf16 = 0, kOutF32Ch0 = 1, kOutF32All = 2 };

// 3x3 convolution, zero padding 1, on an 8 x 16 pixel tile per block.
// x: NHWC [B][H][W][CIN]; mask (optional, NHWC BF16 [CIN]): input values
// where mask <= 0 read as 0 (the ReLU derivative of the backward pass);
// wt: [COUTP][kpad(CIN)] BF16; bias: [COUTP] or nullptr.
template <typename TIn, int CIN, int COUTP, int MODE>
__global__ void __launch_bounds__(kConvThreads)
conv3x3_kernel(const TIn* x, const __nv_bfloat16* mask, const __nv_bfloat16* wt, const float* bias,
               void* out, int H, int W) {
  constexpr int KP = kpad(CIN);
  constexpr int HW = kTileH + 2, WW = kTileW + 2;
  constexpr int WPP = CIN / 2;  // 32-bit words per pixel
  __shared__ uint32_t xs[HW * WW * WPP];
  __shared__ uint32_t ws[COUTP * KP / 2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int x0 = blockIdx.x * kTileW, y0 = blockIdx.y * kTileH, b = blockIdx.z;
  const long long img = static_cast<long long>(b) * H * W;
  if (std::is_same<TIn, __nv_bfloat16>::value && CIN % 8 == 0 && !mask) {
    // BF16 input without a mask: 16-byte loads, all of a thread's issued
    // before any is stored.
    constexpr int V = CIN / 8, NV = HW * WW * V, IT = (NV + kConvThreads - 1) / kConvThreads;
    uint4 v[IT];
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const int i = tid + j * kConvThreads, pix = i / V;
      const int gy = y0 - 1 + pix / WW, gx = x0 - 1 + pix % WW;
      v[j] = make_uint4(0u, 0u, 0u, 0u);
      if (i < NV && gy >= 0 && gy < H && gx >= 0 && gx < W)
        v[j] = *reinterpret_cast<const uint4*>(x + (img + static_cast<long long>(gy) * W + gx) * CIN + 8 * (i % V));
    }
#pragma unroll
    for (int j = 0; j < IT; ++j) {
      const int i = tid + j * kConvThreads;
      if (i < NV) reinterpret_cast<uint4*>(xs)[i] = v[j];
    }
  } else
  for (int i = tid; i < HW * WW * WPP; i += kConvThreads) {
    const int pix = i / WPP, w2 = i % WPP;
    const int gy = y0 - 1 + pix / WW, gx = x0 - 1 + pix % WW;
    uint32_t v = 0u;
    if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
      const long long e = (img + static_cast<long long>(gy) * W + gx) * CIN + 2 * w2;
      v = load_pair(x, e);
      if (mask) {
        const uint32_t mk = load_pair(mask, e);
        const __nv_bfloat162 m2 = *reinterpret_cast<const __nv_bfloat162*>(&mk);
        const float2 mf = __bfloat1622float2(m2);
        const __nv_bfloat162 v2 = *reinterpret_cast<const __nv_bfloat162*>(&v);
        const float2 vf = __bfloat1622float2(v2);
        v = pack_bf16x2(mf.x > 0.f ? vf.x : 0.f, mf.y > 0.f ? vf.y : 0.f);
      }
    }
    xs[i] = v;
  }
  const uint32_t* wt32 = reinterpret_cast<const uint32_t*>(wt);
  for (int i = tid; i < COUTP * KP / 2; i += kConvThreads) ws[i] = wt32[i];
  __syncthreads();

  const int g = lane >> 2, t = lane & 3;
  float acc[2][COUTP / 8][4];
#pragma unroll
  for (int mf = 0; mf < 2; ++mf)
#pragma unroll
    for (int nf = 0; nf < COUTP / 8; ++nf)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[mf][nf][j] = 0.f;
#pragma unroll
  for (int ks = 0; ks < KP / 16; ++ks) {
    uint32_t bq[COUTP / 8][2];
#pragma unroll
    for (int nf = 0; nf < COUTP / 8; ++nf) {
      bq[nf][0] = ws[((nf * 8 + g) * KP + ks * 16 + t * 2) / 2];
      bq[nf][1] = ws[((nf * 8 + g) * KP + ks * 16 + t * 2 + 8) / 2];
    }
    int tapv[2], civ[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = ks * 16 + t * 2 + h * 8;
      tapv[h] = k / CIN;
      civ[h] = k % CIN;
    }
#pragma unroll
    for (int mf = 0; mf < 2; ++mf) {
      const int yy = warp * 2 + mf;
      uint32_t a[4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t lo = 0u, hi = 0u;
        if (tapv[h] < 9) {
          const int dy = tapv[h] / 3, dx = tapv[h] % 3;
          lo = xs[((yy + dy) * WW + g + dx) * WPP + civ[h] / 2];
          hi = xs[((yy + dy) * WW + g + 8 + dx) * WPP + civ[h] / 2];
        }
        a[h * 2] = lo;      // rows g   (pixel g),   k = t*2 (+8)
        a[h * 2 + 1] = hi;  // rows g+8 (pixel g+8)
      }
#pragma unroll
      for (int nf = 0; nf < COUTP / 8; ++nf)
        mma_bf16_16816(acc[mf][nf], a[0], a[1], a[2], a[3], bq[nf][0], bq[nf][1]);
    }
  }
#pragma unroll
  for (int mf = 0; mf < 2; ++mf) {
    const int gy = y0 + warp * 2 + mf;
    if (gy >= H) continue;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int gx = x0 + g + half * 8;
      if (gx >= W) continue;
      const long long pix = img + static_cast<long long>(gy) * W + gx;
#pragma unroll
      for (int nf = 0; nf < COUTP / 8; ++nf) {
        const int co = nf * 8 + t * 2;
        float v0 = acc[mf][nf][half * 2], v1 = acc[mf][nf][half * 2 + 1];
        if (bias) {
          v0 += bias[co];
          v1 += bias[co + 1];
        }
        if (MODE == kOutReluBf16) {
          reinterpret_cast<uint32_t*>(static_cast<__nv_bfloat16*>(out) + pix * COUTP + co)[0] =
              pack_bf16x2(fmaxf(v0, 0.f), fmaxf(v1, 0.f));
        } else if (MODE == kOutF32Ch0) {
          if (co == 0) static_cast<float*>(out)[pix] = v0;
        } else {
          *reinterpret_cast<float2*>(static_cast<float*>(out) + pix * COUTP + co) = make_float2(v0, v1);
        }
      }
    }
  }
}

FBME_DEV void ldmatrix_x4(uint32_t addr, uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
               : "r"(addr));
}
FBME_DEV void ldmatrix_x2(uint32_t addr, uint32_t& a0, uint32_t& a1) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(a0), "=r"(a1) : "r"(addr));
}



// Weight gradient of one layer: dW[tap][ci][co] = sum_p x[p + shift(tap)][ci]
// * g[p][co] (g masked by mask > 0 when a mask is given) and db[co] =
// sum_p g[p][co].  Each block loops over tiles and writes its partial sums;
// grad_reduce_kernel adds them in block order.
template <typename TX, int CIN, int COUT>
__global__ void __launch_bounds__(256)
wgrad_kernel(const TX* x, const float* gin, const __nv_bfloat16* mask, int B, int H, int W,
             float* partial) {
  constexpr int NW = 9 * CIN * COUT;
  constexpr int NOUT = NW + COUT;
  constexpr int PER = (NOUT + 255) / 256;
  constexpr int HW = kTileH + 2, WW = kTileW + 2;
  __shared__ float xs[HW * WW * CIN];
  __shared__ float gs[kTileH * kTileW * COUT];
  const int tid = threadIdx.x;
  float acc[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) acc[j] = 0.f;
  const int tx_n = W / kTileW, ty_n = H / kTileH;
  const long long ntiles = static_cast<long long>(B) * tx_n * ty_n;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int b = static_cast<int>(tile / (tx_n * ty_n));
    const int rem = static_cast<int>(tile % (tx_n * ty_n));
    const int y0 = (rem / tx_n) * kTileH, x0 = (rem % tx_n) * kTileW;
    const long long img = static_cast<long long>(b) * H * W;
    __syncthreads();
    for (int i = tid; i < HW * WW * CIN; i += 256) {
      const int pix = i / CIN, c = i % CIN;
      const int gy = y0 - 1 + pix / WW, gx = x0 - 1 + pix % WW;
      float v = 0.f;
      if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
        const long long e = (img + static_cast<long long>(gy) * W + gx) * CIN + c;
        if constexpr (sizeof(TX) == 2) v = __bfloat162float(x[e]);
        else v = x[e];
      }
      xs[i] = v;
    }
    for (int i = tid; i < kTileH * kTileW * COUT; i += 256) {
      const int pix = i / COUT, c = i % COUT;
      const long long e = (img + static_cast<long long>(y0 + pix / kTileW) * W + x0 + pix % kTileW) * COUT + c;
      float v = gin[e];
      if (mask && !(__bfloat162float(mask[e]) > 0.f)) v = 0.f;
      gs[i] = v;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int o = tid + j * 256;
      if (o >= NOUT) continue;
      float a = 0.f;
      if (o < NW) {
        const int co = o % COUT, ci = (o / COUT) % CIN, tap = o / (COUT * CIN);
        const int dy = tap / 3, dx = tap % 3;
        for (int py = 0; py < kTileH; ++py)
#pragma unroll 4
          for (int px = 0; px < kTileW; ++px)
            a += xs[((py + dy) * WW + px + dx) * CIN + ci] * gs[(py * kTileW + px) * COUT + co];
      } else {
        const int co = o - NW;
        for (int p = 0; p < kTileH * kTileW; ++p) a += gs[p * COUT + co];
      }
      acc[j] += a;
    }
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int o = tid + j * 256;
    if (o < NOUT) partial[static_cast<long long>(blockIdx.x) * NOUT + o] = acc[j];
  }
}

// Sum the block partials of a layer into the flat gradient (FP64 sums in
// block order).  `cin_used` drops padded input channels; weights land at
// flat offset woff as [tap][ci][co], biases at boff.
__global__ void grad_reduce_kernel(const float* partial, int nblocks, int cin, int cin_used, int cout,
                                   int cout_used, int woff, int boff, float* grad) {
  const int nw = 9 * cin * cout;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nw + cout) return;
  double s = 0.0;
  for (int k = 0; k < nblocks; ++k) s += partial[static_cast<long long>(k) * (nw + cout) + o];
  if (o < nw) {
    const int co = o % cout, ci = (o / cout) % cin, tap = o / (cout * cin);
    if (ci < cin_used && co < cout_used) grad[woff + (tap * cin_used + ci) * cout_used + co] = static_cast<float>(s);
  } else {
    const int co = o - nw;
    if (co < cout_used) grad[boff + co] = static_cast<float>(s);
  }
}

// Loss mean((out - target)^2) and d out (channel 0 of an 8-channel FP32
// NHWC gradient); per-block FP64 partial sums of the loss.
__global__ void __launch_bounds__(256) loss_kernel(const float* out, const float* target, long long n,
                                                   float* dout8, double* lpart) {
  __shared__ double red[32];
  double acc = 0.0;
  const float scale = 2.0f / static_cast<float>(n);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float d = out[i] - target[i];
    acc += static_cast<double>(d) * d;
    float4* g = reinterpret_cast<float4*>(dout8 + i * 8);
    g[0] = make_float4(scale * d, 0.f, 0.f, 0.f);
    g[1] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) lpart[blockIdx.x] = s;
}

__global__ void loss_sum_kernel(const double* lpart, int n, double scale, double* loss_out) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += lpart[i];
  *loss_out = s * scale;
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Features of the backprojection (see the header comment of the oracle
// restatement): pass 0 sums |A^H y|^2, pass 1 writes f0 and sums it, pass 2
// writes f1 = mean f0.  part: [B][64] FP64 block partials per pass.
// compact (inference): pass 1 writes f0 alone, one BF16 per pixel, to the
// start of x8 -- the network's first layer takes f1 from the partials.
__global__ void __launch_bounds__(256) features_kernel(int pass, const float2* bp, int B, long long N,
                                                       __nv_bfloat16* x8, double* part, bool compact = false) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  double acc = 0.0;
  double mean = 0.0, f1 = 0.0;
  if (pass >= 1) mean = fmax(parts_sum(part + b * 128, gridDim.x) / static_cast<double>(N), 1e-30);
  if (pass == 2) f1 = parts_sum(part + b * 128 + 64, gridDim.x) / static_cast<double>(N);
  if (pass == 1 && compact && (N & 3) == 0) {
    // four pixels a step: two 16-byte loads, one 8-byte store of BF16 f0
    const float4* src = reinterpret_cast<const float4*>(bp + b * N);
    uint2* dst = reinterpret_cast<uint2*>(x8 + b * N);
#pragma unroll 4
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < N / 4;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
      const float4 u = src[2 * q], w = src[2 * q + 1];
      const float px[4] = {u.x, u.z, w.x, w.z}, py[4] = {u.y, u.w, w.y, w.w};
      float f[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double e = static_cast<double>(px[i]) * px[i] + static_cast<double>(py[i]) * py[i];
        f[i] = logf(static_cast<float>(e / mean) + 1e-3f);
        acc += f[i];
      }
      dst[q] = make_uint2(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]));
    }
    const double sum = block_sum(acc, red);
    if (threadIdx.x == 0) part[b * 128 + pass * 64 + blockIdx.x] = sum;
    return;
  }
#pragma unroll 4
  for (long long n = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 v = bp[b * N + n];
    const double e = static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
    if (pass == 0) {
      acc += e;
    } else if (pass == 1) {
      const float f0 = logf(static_cast<float>(e / mean) + 1e-3f);
      acc += f0;
      if (compact) {
        x8[b * N + n] = __float2bfloat16_rn(f0);
      } else {
        uint4 w;
        w.x = pack_bf16x2(f0, 0.f);
        w.y = w.z = w.w = 0u;
        *reinterpret_cast<uint4*>(x8 + (b * N + n) * 8) = w;
      }
    } else {
      x8[(b * N + n) * 8 + 1] = __float2bfloat16_rn(static_cast<float>(f1));
    }
  }
  if (pass < 2) {
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) part[b * 128 + pass * 64 + blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// The whole network on 32 x 32 output tiles, all three layers on the
// tensor cores (mma.sync, BF16 operands, FP32 accumulation), every
// intermediate in shared memory.  Per tile:
//   x  : the f0 halo, 38 x 38 pixels of (f0, f1) BF16 pairs (f1 = the
//        scene constant), zero outside the image;
//   h1 : layer 1 on the 36 x 36 region, 16-pixel fragments in raster
//        order, K = (tap, channel) = 18, padded to 32;
//   h2 : layer 2 on the 34 x 34 region, A fragments by ldmatrix from h1
//        (as conv3x3_kernel), K = 72 (four m16n8k16 steps and an m16n8k8);
//   z  : the accumulator fragment of layer 2, relu'd and rounded to BF16,
//        is the A fragment of an m16n8k8 product with W3 (K = 8 channels,
//        N = 9 taps): z[tap][q] = sum_c W3[tap][c] h2[q][c];
//   out: b3 + sum over the 9 taps of z[tap][q + shift(tap)].
// Biases are the accumulators' initial values (FP32).  Region pixels
// outside the image are zero, as the convolution's zero padding
// reads them.  Inference writes prior0 = max(data_power / N * exp(out),
// floor) and its partial sums; training writes h1, h2 (NHWC BF16) and out
// (FP32) for the backward pass.  Traffic: 2 bytes of f0 read and 4 bytes
// of prior written per pixel.
// ---------------------------------------------------------------------------
constexpr int kFT = 32, kFThreads = 256, kFStrip = 4;   // the gather: 4-row strips per thread
// x halo: 38 rows of 40 pixels (columns x0 - 4 ...), in rows of 48 words
// (48 = 16 mod 32 banks: layer 1's taps of 8 pixels fall on distinct banks)
constexpr int kFXH = kFT + 6, kFXC = kFT + 8, kFXP = 48;
constexpr int kFXN = kFXH * kFXP, kFXChunks = kFXH * (kFXC / 4);  // 4-pixel chunks
constexpr int kF1W = kFT + 4, kF1N = kF1W * kF1W;       // h1 region
constexpr int kF2W = kFT + 2, kF2N = kF2W * kF2W;       // h2 / z region
constexpr int kFFrag1 = (kF1N + 15) / 16, kFFrag2 = (kF2N + 15) / 16;
// dynamic shared memory: z [9][kF2N] FP32 (the x halo [kFXN] BF16 pairs
// lies under it until layer 1 is done; its rows are 16-byte aligned), h1
// [kF1N] NHWC BF16 pixels, then two address tables built once per CTA:
// layer 1, per fragment and row g < 8, the halo indices of its pixels g and
// g + 8 (16 bits each); layer 2, per fragment and row, the h1 index of the
// pixel's first tap (16 bits).
constexpr int kFTab1 = kFFrag1 * 8, kFTab2 = kFFrag2 * 16;
constexpr size_t kFSmemA = sizeof(float) * 9 * kF2N;
constexpr size_t kFSmemB = sizeof(uint4) * kF1N;
constexpr size_t kFSmem = kFSmemA + kFSmemB + sizeof(uint32_t) * kFTab1 + sizeof(uint16_t) * kFTab2;
static_assert(kFSmemA >= sizeof(uint32_t) * kFXN, "the x halo fits under z");
static_assert(kFXChunks <= 2 * kFThreads, "the x halo: two chunks per thread at most");
static_assert(kFSmemA % 16 == 0, "16-byte aligned h1");
static_assert(kFThreads == kFT * (kFT / kFStrip), "the gather: one strip per thread");

// Prior of the strip (gy0 + p, gx), p < kFStrip, from the network outputs
// o[p]: stores gamma and adds the priors to acc in pixel order (both
// warm-prior tile kernels use it, so their partial sums agree bit for bit).
FBME_DEV void prior_strip(const float (&o)[kFStrip], float base, float fl, float* gamma_img, int H, int W,
                          int gy0, int gx, double& acc) {
  if (gx >= W) return;
#pragma unroll
  for (int p = 0; p < kFStrip; ++p) {
    const int gy = gy0 + p;
    if (gy >= H) break;
    const float gm = fmaxf(base * expf(fminf(fmaxf(o[p], -40.f), 40.f)), fl);
    gamma_img[static_cast<long long>(gy) * W + gx] = gm;
    acc += gm;
  }
}

// The same prior from a caller's [B][H][W] map, over the same tiles, strips
// and partial-sum slots as net_tile_kernel<false, 1>.
__global__ void __launch_bounds__(kFThreads) warm_map_kernel(const float* map, int H, int W,
                                                            const float* data_power, const float* floor_,
                                                            float* gamma, double* upart, int nslots) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const long long img = static_cast<long long>(b) * H * W;
  const float base = data_power[b] / static_cast<float>(static_cast<long long>(H) * W), fl = floor_[b];
  const int tx_n = (W + kFT - 1) / kFT, ntiles = tx_n * ((H + kFT - 1) / kFT);
  const int col = threadIdx.x % kFT, r0 = (threadIdx.x / kFT) * kFStrip;
  double acc = 0.0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int y0 = (tile / tx_n) * kFT, x0 = (tile % tx_n) * kFT;
    const int gx = x0 + col;
    float o[kFStrip];
#pragma unroll
    for (int p = 0; p < kFStrip; ++p) {
      const int gy = y0 + r0 + p;
      o[p] = (gy < H && gx < W) ? map[img + static_cast<long long>(gy) * W + gx] : 0.f;
    }
    prior_strip(o, base, fl, gamma + img, H, W, y0 + r0, gx, acc);
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0)
    for (int k = blockIdx.x; k < nslots; k += gridDim.x)
      upart[(static_cast<long long>(b) * kMaxTilesPerScene + k) * kPartSlots] = k == blockIdx.x ? s : 0.0;
}

// CTAs per scene of the two warm-prior tile kernels: about four tiles each
// (amortising the per-CTA setup and prefetching the next tile's halo), at
// most the `nslots` partial-sum slots the initialisation reads.
inline int warm_ctas(int H, int W, int nslots) {
  const int ntiles = ((H + kFT - 1) / kFT) * ((W + kFT - 1) / kFT);
  return std::max(1, std::min(nslots, (ntiles + 3) / 4));
}

FBME_DEV void mma_bf16_1688(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm(
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0));
}

// relu(BF16(a)), relu(BF16(b)) as a BF16 pair.
FBME_DEV uint32_t relu_bf16x2(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  v = __hmax2(v, __float2bfloat162_rn(0.f));
  return *reinterpret_cast<const uint32_t*>(&v);
}

FBME_DEV bool in_image(int y, int x, int H, int W) {
  return static_cast<unsigned>(y) < static_cast<unsigned>(H) && static_cast<unsigned>(x) < static_cast<unsigned>(W);
}

struct NetArgs {
  const __nv_bfloat16* x;  // f0 at x[pixel * CSTR]
  const double* fpart;     // feature partials [B][128]; f1 = the pass-1 sum / N
  int nparts;
  const float* params;     // FP32 master parameters
  int H, W;
  // inference: the prior and its partial sums
  const float* data_power;
  const float* floor_;
  float* gamma;
  double* upart;
  int nslots;  // partial-sum slots per scene (>= gridDim.x; the rest are zeroed)
  // training: the activations for the backward pass
  __nv_bfloat16* h1;
  __nv_bfloat16* h2;
  float* out;
};

static_assert(kF1N % 16 == 0, "layer 1: every fragment row is a region pixel");

template <bool TRAIN, int CSTR>
__global__ void __launch_bounds__(kFThreads, 3) net_tile_kernel(NetArgs a) {
  extern __shared__ __align__(16) uint8_t fsm[];
  __shared__ double red[32];
  float* z = reinterpret_cast<float*>(fsm);         // [9][kF2N]
  uint32_t* xs = reinterpret_cast<uint32_t*>(fsm);  // [kFXN] (f0, f1) pairs
  uint4* h1 = reinterpret_cast<uint4*>(fsm + kFSmemA);
  uint32_t* h1w = reinterpret_cast<uint32_t*>(h1);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int b = blockIdx.y, H = a.H, W = a.W;
  const long long N = static_cast<long long>(H) * W, img = static_cast<long long>(b) * N;
  const float* p = a.params;
  const uint32_t c1hi = static_cast<uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(
                            static_cast<float>(parts_sum(a.fpart + b * 128 + 64, a.nparts) / static_cast<double>(N)))))
                        << 16;
  // B fragments (lane: n = g, k = 2 t4 (+1), + 8 for the second register)
  const uint32_t l1b0 = pack_bf16x2(p[kOffW1 + (t4 * kIn) * kHid + g], p[kOffW1 + (t4 * kIn + 1) * kHid + g]);
  const uint32_t l1b1 =
      pack_bf16x2(p[kOffW1 + ((t4 + 4) * kIn) * kHid + g], p[kOffW1 + ((t4 + 4) * kIn + 1) * kHid + g]);
  const uint32_t l1b2 =
      t4 == 0 ? pack_bf16x2(p[kOffW1 + (8 * kIn) * kHid + g], p[kOffW1 + (8 * kIn + 1) * kHid + g]) : 0u;
  constexpr int KP2 = kpad(kHid);
  uint32_t bq[KP2 / 16][2];
#pragma unroll
  for (int ks = 0; ks < KP2 / 16; ++ks)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = ks * 16 + 2 * t4 + 8 * h;  // k = tap * 8 + channel
      bq[ks][h] = k < 9 * kHid ? pack_bf16x2(p[kOffW2 + k * kHid + g], p[kOffW2 + (k + 1) * kHid + g]) : 0u;
    }
  const uint32_t bz0 = pack_bf16x2(p[kOffW3 + g * kHid + 2 * t4], p[kOffW3 + g * kHid + 2 * t4 + 1]);
  const uint32_t bz1 =
      g == 0 ? pack_bf16x2(p[kOffW3 + 8 * kHid + 2 * t4], p[kOffW3 + 8 * kHid + 2 * t4 + 1]) : 0u;
  const float b3 = p[kOffB3];
  // biases of this lane's accumulator columns (channels 2 t4, 2 t4 + 1)
  const float b1a = p[kOffB1 + 2 * t4], b1b = p[kOffB1 + 2 * t4 + 1];
  const float b2a = p[kOffB2 + 2 * t4], b2b = p[kOffB2 + 2 * t4 + 1];
  float base = 0.f, fl = 0.f;
  if constexpr (!TRAIN) {
    base = a.data_power[b] / static_cast<float>(N);
    fl = a.floor_[b];
  }
  // per-lane constants: layer-1 tap offsets in the x halo (the second k
  // step holds tap 8 in lanes t4 = 0, zero elsewhere); layer-2 ldmatrix row
  // and tap offsets in h1 (the fifth k step is tap 8 alone)
  const int o1a = (t4 / 3) * kFXP + t4 % 3, o1b = ((t4 + 4) / 3) * kFXP + (t4 + 4) % 3;
  constexpr int o8 = 2 * kFXP + 2;
  const int mj = lane >> 3, pr = (lane & 7) + (mj & 1) * 8, odd = mj >> 1;
  int o2[KP2 / 16];
#pragma unroll
  for (int ks = 0; ks < KP2 / 16; ++ks) {
    const int tap = 2 * ks + odd;
    o2[ks] = tap < 9 ? (tap / 3) * kF1W + tap % 3 : 2 * kF1W + 2;  // x2 load: upper lanes unused
  }
  uint32_t* tab1 = reinterpret_cast<uint32_t*>(fsm + kFSmemA + kFSmemB);
  uint16_t* tab2 = reinterpret_cast<uint16_t*>(tab1 + kFTab1);
  for (int i = tid; i < kFTab1; i += kFThreads) {
    const int p0 = (i / 8) * 16 + i % 8, p1 = p0 + 8;
    // region pixel (ry, rx) reads the halo from (ry, rx + 1): the halo starts a column earlier
    tab1[i] = static_cast<uint32_t>(p0 / kF1W * kFXP + p0 % kF1W + 1) |
              (static_cast<uint32_t>(p1 / kF1W * kFXP + p1 % kF1W + 1) << 16);
  }
  for (int i = tid; i < kFTab2; i += kFThreads) {
    const int pa = min(i, kF2N - 1);
    tab2[i] = static_cast<uint16_t>(pa / kF2W * kF1W + pa % kF2W);
  }

  const int tx_n = (W + kFT - 1) / kFT, ntiles = tx_n * ((H + kFT - 1) / kFT);
  // x halo chunks (4 pixels of one row, 8 bytes of compact f0): a thread
  // fetches chunks tid and tid + kFThreads of a tile into registers one tile
  // ahead, so the loads fly while the previous tile computes.  W % 16 == 0,
  // so a chunk lies wholly inside or wholly outside the image.
  uint2 hv[2];
  bool hin[2];
  auto fetch = [&](int t) {
    const int fy0 = (t / tx_n) * kFT, fx0 = (t % tx_n) * kFT;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int ch = tid + j * kFThreads, row = ch / (kFXC / 4), k = ch - row * (kFXC / 4);
      const int gy = fy0 - 3 + row, gx = fx0 - 4 + 4 * k;
      hin[j] = ch < kFXChunks && in_image(gy, gx, H, W);
      hv[j] = make_uint2(0u, 0u);
      if (hin[j]) {
        const long long e = img + static_cast<long long>(gy) * W + gx;
        if constexpr (CSTR == 1) {
          hv[j] = *reinterpret_cast<const uint2*>(a.x + e);
        } else {
          const uint16_t* x16 = reinterpret_cast<const uint16_t*>(a.x);
          hv[j] = make_uint2(x16[e * CSTR] | (static_cast<uint32_t>(x16[(e + 1) * CSTR]) << 16),
                             x16[(e + 2) * CSTR] | (static_cast<uint32_t>(x16[(e + 3) * CSTR]) << 16));
        }
      }
    }
  };
  double acc = 0.0;
  if (blockIdx.x < ntiles) fetch(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int y0 = (tile / tx_n) * kFT, x0 = (tile % tx_n) * kFT;
    // the whole halo lies inside the image: no region pixel is padding
    const bool inner = y0 >= 3 && x0 >= 3 && y0 + kFT + 3 <= H && x0 + kFT + 3 <= W;
    __syncthreads();  // the tables are built; the previous tile's z is read
#pragma unroll
    for (int j = 0; j < 2; ++j) {  // (f0, f1) pairs, zero outside the image
      const int ch = tid + j * kFThreads, row = ch / (kFXC / 4);
      if (ch < kFXChunks) {
        const uint32_t m = hin[j] ? c1hi : 0u;
        reinterpret_cast<uint4*>(xs + row * kFXP)[ch - row * (kFXC / 4)] =
            make_uint4(m | (hv[j].x & 0xFFFFu), m | (hv[j].x >> 16), m | (hv[j].y & 0xFFFFu), m | (hv[j].y >> 16));
      }
    }
    if (tile + gridDim.x < ntiles) fetch(tile + gridDim.x);
    __syncthreads();
    // layer 1: rows g, g + 8 of fragment f are region pixels f * 16 + g (+ 8);
    // a warp takes fragments f and f + 8 together (two independent chains)
    for (int f = warp; f < kFFrag1; f += 2 * (kFThreads / 32)) {
      const int fb = min(f + kFThreads / 32, kFFrag1 - 1);
      const uint32_t qa = tab1[f * 8 + g], qb = tab1[fb * 8 + g];
      const uint32_t *xa0 = xs + (qa & 0xFFFFu), *xa1 = xs + (qa >> 16);
      const uint32_t *xb0 = xs + (qb & 0xFFFFu), *xb1 = xs + (qb >> 16);
      float ca[4] = {b1a, b1b, b1a, b1b}, cb[4] = {b1a, b1b, b1a, b1b};
      mma_bf16_16816(ca, xa0[o1a], xa1[o1a], xa0[o1b], xa1[o1b], l1b0, l1b1);
      mma_bf16_16816(cb, xb0[o1a], xb1[o1a], xb0[o1b], xb1[o1b], l1b0, l1b1);
      mma_bf16_16816(ca, t4 == 0 ? xa0[o8] : 0u, t4 == 0 ? xa1[o8] : 0u, 0u, 0u, l1b2, 0u);
      mma_bf16_16816(cb, t4 == 0 ? xb0[o8] : 0u, t4 == 0 ? xb1[o8] : 0u, 0u, 0u, l1b2, 0u);
      const int nf = f + kFThreads / 32 < kFFrag1 ? 2 : 1;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (u >= nf) break;
        const float* cc = u ? cb : ca;
        const uint32_t w0 = relu_bf16x2(cc[0], cc[1]), w1 = relu_bf16x2(cc[2], cc[3]);
        const int p0 = (u ? fb : f) * 16 + g;
        h1w[p0 * 4 + t4] = w0;
        h1w[(p0 + 8) * 4 + t4] = w1;
        if constexpr (TRAIN) {  // the tile's own 32 x 32 pixels
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int pp = p0 + 8 * h, ry = pp / kF1W, rx = pp - ry * kF1W;
            const int gy = y0 - 2 + ry, gx = x0 - 2 + rx;
            if (ry >= 2 && ry < kFT + 2 && rx >= 2 && rx < kFT + 2 && in_image(gy, gx, H, W))
              reinterpret_cast<uint32_t*>(a.h1 + (img + static_cast<long long>(gy) * W + gx) * kHid)[t4] =
                  h ? w1 : w0;
          }
        }
      }
    }
    if (!inner) {  // region pixels outside the image are the zero padding
      __syncthreads();
      for (int i = tid; i < kF1N; i += kFThreads) {
        const int ry = i / kF1W;
        if (!in_image(y0 - 2 + ry, x0 - 2 + (i - ry * kF1W), H, W)) h1[i] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    __syncthreads();
    // layer 2 and the per-pixel tap products of layer 3, fragments f and
    // f + 8 together
    for (int f = warp; f < kFFrag2; f += 2 * (kFThreads / 32)) {
      const int fb = min(f + kFThreads / 32, kFFrag2 - 1);
      const uint4* ha = h1 + tab2[f * 16 + pr];
      const uint4* hb = h1 + tab2[fb * 16 + pr];
      float ca[4] = {b2a, b2b, b2a, b2b}, cb[4] = {b2a, b2b, b2a, b2b};
#pragma unroll
      for (int ks = 0; ks < KP2 / 16 - 1; ++ks) {
        uint32_t a0, a1, a2, a3, b0, b1, b2, b3v;
        ldmatrix_x4(smem_u32(ha + o2[ks]), a0, a1, a2, a3);
        ldmatrix_x4(smem_u32(hb + o2[ks]), b0, b1, b2, b3v);
        mma_bf16_16816(ca, a0, a1, a2, a3, bq[ks][0], bq[ks][1]);
        mma_bf16_16816(cb, b0, b1, b2, b3v, bq[ks][0], bq[ks][1]);
      }
      {  // tap 8 (k 64-71): pixels 0-7 and 8-15 of the fragment
        uint32_t a0, a1, b0, b1;
        ldmatrix_x2(smem_u32(ha + o2[KP2 / 16 - 1]), a0, a1);
        ldmatrix_x2(smem_u32(hb + o2[KP2 / 16 - 1]), b0, b1);
        mma_bf16_1688(ca, a0, a1, bq[KP2 / 16 - 1][0]);
        mma_bf16_1688(cb, b0, b1, bq[KP2 / 16 - 1][0]);
      }
      const int nf = f + kFThreads / 32 < kFFrag2 ? 2 : 1;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (u >= nf) break;
        const float* cc = u ? cb : ca;
        const uint32_t u0 = relu_bf16x2(cc[0], cc[1]), u1 = relu_bf16x2(cc[2], cc[3]);
        const int q0 = (u ? fb : f) * 16 + g;
        if constexpr (TRAIN) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int q = q0 + 8 * h, sy = q / kF2W, sx = q - sy * kF2W;
            const int gy = y0 - 1 + sy, gx = x0 - 1 + sx;
            if (q < kF2N && sy >= 1 && sy <= kFT && sx >= 1 && sx <= kFT && in_image(gy, gx, H, W))
              reinterpret_cast<uint32_t*>(a.h2 + (img + static_cast<long long>(gy) * W + gx) * kHid)[t4] =
                  h ? u1 : u0;
          }
        }
        // the accumulator fragment (rows g, g + 8; channels 2 t4, 2 t4 + 1)
        // is the A fragment of m16n8k8: z for taps 0-7, then tap 8
        float za[4] = {0.f, 0.f, 0.f, 0.f}, zb[4] = {0.f, 0.f, 0.f, 0.f};
        mma_bf16_1688(za, u0, u1, bz0);
        mma_bf16_1688(zb, u0, u1, bz1);
        if (q0 < kF2N) {
          z[(2 * t4) * kF2N + q0] = za[0];
          z[(2 * t4 + 1) * kF2N + q0] = za[1];
          if (t4 == 0) z[8 * kF2N + q0] = zb[0];
        }
        if (q0 + 8 < kF2N) {
          z[(2 * t4) * kF2N + q0 + 8] = za[2];
          z[(2 * t4 + 1) * kF2N + q0 + 8] = za[3];
          if (t4 == 0) z[8 * kF2N + q0 + 8] = zb[2];
        }
      }
    }
    __syncthreads();
    if (!inner) {  // h2 outside the image is zero padding: so are its tap products
      for (int i = tid; i < kF2N; i += kFThreads) {
        const int sy = i / kF2W;
        if (!in_image(y0 - 1 + sy, x0 - 1 + (i - sy * kF2W), H, W))
#pragma unroll
          for (int tap = 0; tap < 9; ++tap) z[tap * kF2N + i] = 0.f;
      }
      __syncthreads();
    }
    {  // layer 3: out = sum over the taps (in order) + b3
      const int col = tid % kFT, r0 = (tid / kFT) * kFStrip;
      float o[kFStrip];
#pragma unroll
      for (int pp = 0; pp < kFStrip; ++pp) {
        const int qb = (r0 + pp) * kF2W + col;
        float sacc = z[qb];
#pragma unroll
        for (int tap = 1; tap < 9; ++tap) sacc += z[tap * kF2N + qb + (tap / 3) * kF2W + tap % 3];
        o[pp] = sacc + b3;
      }
      if constexpr (TRAIN) {
        const int gx = x0 + col;
#pragma unroll
        for (int pp = 0; pp < kFStrip; ++pp) {
          const int gy = y0 + r0 + pp;
          if (gy < H && gx < W) a.out[img + static_cast<long long>(gy) * W + gx] = o[pp];
        }
      } else {
        prior_strip(o, base, fl, a.gamma + img, H, W, y0 + r0, x0 + col, acc);
      }
    }
  }
  if constexpr (!TRAIN) {
    const double sum = block_sum(acc, red);
    if (tid == 0)
      for (int k = blockIdx.x; k < a.nslots; k += gridDim.x)
        a.upart[(static_cast<long long>(b) * kMaxTilesPerScene + k) * kPartSlots] = k == blockIdx.x ? sum : 0.0;
  }
}

}  // namespace cnn
}  // namespace fbme

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

using namespace fbme;

size_t a256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

constexpr int kWgradBlocks = 296;

struct CnnLayout {
  size_t packed, x8, h1, h2, out, dout8, dh2, dh1, partial, lpart, fpart, grad, total;
};

CnnLayout cnn_layout(long long B, long long H, long long W) {
  using namespace cnn;
  CnnLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = a256(off + bytes);
    return o;
  };
  const size_t P = B * H * W;
  L.packed = take(64 * 1024);
  L.x8 = take(P * kInP * 2);
  L.h1 = take(P * kHid * 2);
  L.h2 = take(P * kHid * 2);
  L.out = take(P * 4);
  L.dout8 = take(P * 8 * 4);
  L.dh2 = take(P * kHid * 4);
  L.dh1 = take(P * kHid * 4);
  L.partial = take(static_cast<size_t>(kWgradBlocks) * (9 * kHid * kHid + kHid) * 4);
  L.lpart = take(1024 * 8);
  L.fpart = take(B * 128 * 8);
  L.grad = take(kNParams * 4);
  L.total = off;
  return L;
}

cnn::Packed packed_at(uint8_t* w) {
  using namespace cnn;
  Packed P;
  uint8_t* p = w;
  auto take = [&](size_t bytes) {
    uint8_t* r = p;
    p += a256(bytes);
    return r;
  };
  P.wb3 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kKb3 * 2));
  P.wb2 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kK2 * 2));
  return P;
}

}  // namespace

namespace fbme {

int cnn_param_count() { return cnn::kNParams; }

size_t cnn_workspace_bytes(long long B, long long H, long long W) { return cnn_layout(B, H, W).total; }

const char* cnn_check(long long B, long long H, long long W) {
  if (B < 1 || H < 1 || W < 1) return "batch and grid must be positive";
  if (H % cnn::kTileH != 0 || W % cnn::kTileW != 0)
    return "the warm-start network needs N1 % 8 == 0 and N2 % 16 == 0";
  return nullptr;
}

namespace {
// Blocks (and FP64 partials) per scene of a feature pass: a block takes
// 4096 pixels or more, 16 a thread, so its loads overlap.
int feature_parts(int H, int W) {
  return static_cast<int>(std::min<long long>(16, (static_cast<long long>(H) * W + 4095) / 4096));
}
// Passes 0 and 1 (the energy mean, f0 and its partial sums); pass 2 stores
// the f1 channel, which only the backward pass reads from the workspace.
// The feature statistics' first pass from a known sum |bp|^2 per scene (the
// initialisation's sum of the backprojection power): partial 0 holds it,
// the other partials of the pass zero.
__global__ void seed_feature_sum_kernel(const float* ebp, int B, int parts, double* part) {
  const int b = blockIdx.x, k = threadIdx.x;
  if (b < B && k < parts) part[b * 128 + k] = k == 0 ? static_cast<double>(ebp[b]) : 0.0;
}

void features_passes(const float2* bp, int B, int H, int W, void* ws, int passes, cudaStream_t st,
                     bool compact = false, int first = 0) {
  using namespace cnn;
  const CnnLayout L = cnn_layout(B, H, W);
  uint8_t* w = static_cast<uint8_t*>(ws);
  auto* x8 = reinterpret_cast<__nv_bfloat16*>(w + L.x8);
  auto* fpart = reinterpret_cast<double*>(w + L.fpart);
  for (int pass = first; pass < passes; ++pass)
    features_kernel<<<dim3(feature_parts(H, W), B), 256, 0, st>>>(pass, bp, B, static_cast<long long>(H) * W,
                                                                  x8, fpart, compact);
}
}  // namespace

void cnn_features(const float2* bp, int B, int H, int W, void* ws, cudaStream_t st) {
  features_passes(bp, B, H, W, ws, 3, st);
}

// Forward pass from the features in the workspace; the output [B][H][W]
// stays in the workspace (for cnn_backward) and is copied to `out` if given.
void cnn_forward(const float* params, int B, int H, int W, void* ws, float* out, cudaStream_t st) {
  using namespace cnn;
  const CnnLayout L = cnn_layout(B, H, W);
  uint8_t* w = static_cast<uint8_t*>(ws);
  const Packed P = packed_at(w + L.packed);  // the backward pass's operand matrices
  pack_kernel<<<(kHid * kK2 + 255) / 256, 256, 0, st>>>(params, P);
  float* wout = reinterpret_cast<float*>(w + L.out);  // kept for cnn_backward
  NetArgs na{};
  na.x = reinterpret_cast<const __nv_bfloat16*>(w + L.x8);
  na.fpart = reinterpret_cast<const double*>(w + L.fpart);
  na.nparts = feature_parts(H, W);
  na.params = params;
  na.H = H;
  na.W = W;
  na.h1 = reinterpret_cast<__nv_bfloat16*>(w + L.h1);
  na.h2 = reinterpret_cast<__nv_bfloat16*>(w + L.h2);
  na.out = wout;
  const int ntiles = ((H + kFT - 1) / kFT) * ((W + kFT - 1) / kFT);
  net_tile_kernel<true, kInP><<<dim3(ntiles, B), kFThreads, kFSmem, st>>>(na);
  if (out && out != wout)
    cudaMemcpyAsync(out, wout, static_cast<size_t>(B) * H * W * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

// Loss and gradient after cnn_forward (same workspace): grad[kNParams], and
// the loss written to *loss_out (device FP64) as the sum of block partials.
void cnn_backward(const float* target, int B, int H, int W, void* ws, float* grad, double* loss_out,
                  cudaStream_t st) {
  using namespace cnn;
  const CnnLayout L = cnn_layout(B, H, W);
  uint8_t* w = static_cast<uint8_t*>(ws);
  const Packed P = packed_at(w + L.packed);
  const long long n = static_cast<long long>(B) * H * W;
  auto* x8 = reinterpret_cast<const __nv_bfloat16*>(w + L.x8);
  auto* h1 = reinterpret_cast<const __nv_bfloat16*>(w + L.h1);
  auto* h2 = reinterpret_cast<const __nv_bfloat16*>(w + L.h2);
  auto* out = reinterpret_cast<const float*>(w + L.out);
  auto* dout8 = reinterpret_cast<float*>(w + L.dout8);
  auto* dh2 = reinterpret_cast<float*>(w + L.dh2);
  auto* dh1 = reinterpret_cast<float*>(w + L.dh1);
  auto* partial = reinterpret_cast<float*>(w + L.partial);
  auto* lpart = reinterpret_cast<double*>(w + L.lpart);
  loss_kernel<<<1024, 256, 0, st>>>(out, target, n, dout8, lpart);
  const dim3 grid(W / kTileW, H / kTileH, B);
  // layer 3
  wgrad_kernel<__nv_bfloat16, kHid, 8><<<kWgradBlocks, 256, 0, st>>>(h2, dout8, nullptr, B, H, W, partial);
  grad_reduce_kernel<<<(9 * kHid * 8 + 8 + 255) / 256, 256, 0, st>>>(partial, kWgradBlocks, kHid, kHid, 8, 1,
                                                                       kOffW3, kOffB3, grad);
  conv3x3_kernel<float, 8, kHid, kOutF32All><<<grid, kConvThreads, 0, st>>>(dout8, nullptr, P.wb3, nullptr,
                                                                            dh2, H, W);
  // layer 2 (d a2 = d h2 masked by h2 > 0)
  wgrad_kernel<__nv_bfloat16, kHid, kHid><<<kWgradBlocks, 256, 0, st>>>(h1, dh2, h2, B, H, W, partial);
  grad_reduce_kernel<<<(9 * kHid * kHid + kHid + 255) / 256, 256, 0, st>>>(
      partial, kWgradBlocks, kHid, kHid, kHid, kHid, kOffW2, kOffB2, grad);
  conv3x3_kernel<float, kHid, kHid, kOutF32All><<<grid, kConvThreads, 0, st>>>(dh2, h2, P.wb2, nullptr, dh1,
                                                                               H, W);
  // layer 1 (d a1 = d h1 masked by h1 > 0)
  wgrad_kernel<__nv_bfloat16, kInP, kHid><<<kWgradBlocks, 256, 0, st>>>(x8, dh1, h1, B, H, W, partial);
  grad_reduce_kernel<<<(9 * kInP * kHid + kHid + 255) / 256, 256, 0, st>>>(
      partial, kWgradBlocks, kInP, kIn, kHid, kHid, kOffW1, kOffB1, grad);
  if (loss_out) loss_sum_kernel<<<1, 1, 0, st>>>(lpart, 1024, 1.0 / static_cast<double>(n), loss_out);
}

void cnn_adam(float* params, const float* grad, float* m, float* v, int step, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, static_cast<float>(step));
  const float c2 = 1.f - powf(b2, static_cast<float>(step));
  cnn::adam_kernel<<<(cnn::kNParams + 255) / 256, 256, 0, st>>>(params, grad, m, v, cnn::kNParams, lr, b1, b2,
                                                                 1e-8f, c1, c2);
}

// Warm start inside a plan: features of A^H y, then the fused network +
// prior (prior0 and its partial sums in `nblocks` slots per scene); the
// caller then re-runs the scalar initialisation.
void cnn_warm_prior(const float* params, const float2* bp, int B, int H, int W, void* ws,
                    const float* data_power, const float* floor_, float* gamma, double* upart,
                    int nblocks, cudaStream_t st, const float* ebp) {
  using namespace cnn;
  const CnnLayout L = cnn_layout(B, H, W);
  uint8_t* w = static_cast<uint8_t*>(ws);
  auto* fpart = reinterpret_cast<double*>(w + L.fpart);
  // f0 alone, one BF16 per pixel (the network takes f1 from the partials);
  // with the backprojection power `ebp` the statistics pass is not repeated
  if (ebp) {
    seed_feature_sum_kernel<<<B, 64, 0, st>>>(ebp, B, feature_parts(H, W), fpart);
    features_passes(bp, B, H, W, ws, 2, st, true, 1);
  } else {
    features_passes(bp, B, H, W, ws, 2, st, true);
  }
  NetArgs na{};
  na.x = reinterpret_cast<const __nv_bfloat16*>(w + L.x8);
  na.fpart = fpart;
  na.nparts = feature_parts(H, W);
  na.params = params;
  na.H = H;
  na.W = W;
  na.data_power = data_power;
  na.floor_ = floor_;
  na.gamma = gamma;
  na.upart = upart;
  na.nslots = nblocks;
  net_tile_kernel<false, 1><<<dim3(warm_ctas(H, W, nblocks), B), kFThreads, kFSmem, st>>>(na);
}

void warm_prior_from_map(const float* map, int B, int H, int W, const float* data_power, const float* floor_,
                         float* gamma, double* upart, int nblocks, cudaStream_t st) {
  using namespace cnn;
  warm_map_kernel<<<dim3(warm_ctas(H, W, nblocks), B), kFThreads, 0, st>>>(map, H, W, data_power, floor_, gamma,
                                                                          upart, nblocks);
}

cudaError_t set_cnn_attributes() {
  cudaError_t e = cudaFuncSetAttribute(cnn::net_tile_kernel<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(cnn::kFSmem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cnn::net_tile_kernel<true, cnn::kInP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(cnn::kFSmem));
  return e;
}

}  // namespace fbme

// ---------------------------------------------------------------------------
// C ABI of the network (training and inference stages)
// ---------------------------------------------------------------------------
namespace {
int cnn_args(int B, int H, int W, const void* ws) {
  if (const char* why = fbme::cnn_check(B, H, W)) return fbme::api_fail(FBME_ERR_INVALID, why);
  if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u) != 0)
    return fbme::api_fail(FBME_ERR_WORKSPACE, "workspace must be a 256-byte aligned device pointer");
  return FBME_OK;
}
int cnn_launch_status(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fbme::api_fail(FBME_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return FBME_OK;
}
}  // namespace

extern "C" {

int32_t fbme_cnn_param_count(void) { return fbme::cnn_param_count(); }

size_t fbme_cnn_workspace_bytes(int32_t batch, int32_t n1, int32_t n2) {
  if (fbme::cnn_check(batch, n1, n2)) return 0;
  return fbme::cnn_workspace_bytes(batch, n1, n2);
}

int fbme_cnn_features(const void* backprojection, int32_t batch, int32_t n1, int32_t n2, void* workspace,
                      fbme_stream_t stream) {
  if (!backprojection) return fbme::api_fail(FBME_ERR_INVALID, "NULL argument");
  int rc = cnn_args(batch, n1, n2, workspace);
  if (rc != FBME_OK) return rc;
  fbme::cnn_features(static_cast<const float2*>(backprojection), batch, n1, n2, workspace,
                     reinterpret_cast<cudaStream_t>(stream));
  return cnn_launch_status("fbme_cnn_features");
}

int fbme_cnn_forward(const float* params, int32_t batch, int32_t n1, int32_t n2, void* workspace, float* out,
                     fbme_stream_t stream) {
  if (!params) return fbme::api_fail(FBME_ERR_INVALID, "NULL argument");
  int rc = cnn_args(batch, n1, n2, workspace);
  if (rc != FBME_OK) return rc;
  fbme::cnn_forward(params, batch, n1, n2, workspace, out, reinterpret_cast<cudaStream_t>(stream));
  return cnn_launch_status("fbme_cnn_forward");
}

int fbme_cnn_backward(const float* target, int32_t batch, int32_t n1, int32_t n2, void* workspace, float* grad,
                      double* loss, fbme_stream_t stream) {
  if (!target || !grad) return fbme::api_fail(FBME_ERR_INVALID, "NULL argument");
  int rc = cnn_args(batch, n1, n2, workspace);
  if (rc != FBME_OK) return rc;
  fbme::cnn_backward(target, batch, n1, n2, workspace, grad, loss, reinterpret_cast<cudaStream_t>(stream));
  return cnn_launch_status("fbme_cnn_backward");
}

int fbme_cnn_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                  fbme_stream_t stream) {
  if (!params || !grad || !m || !v || step < 1) return fbme::api_fail(FBME_ERR_INVALID, "bad argument");
  fbme::cnn_adam(params, grad, m, v, step, lr, reinterpret_cast<cudaStream_t>(stream));
  return cnn_launch_status("fbme_cnn_adam");
}

}  // extern "C"
