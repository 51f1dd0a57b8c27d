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
// The 8-to-8-channel convolutions (layer 2 forward, the input gradients)
// run as implicit GEMMs on the tensor cores (mma.sync m16n8k16, BF16
// operands, FP32 accumulation): M = 16 pixels of one tile row, N = 8 output
// channels, K = (tap, input channel) with the channel fastest, so an operand
// pair is one 32-bit load from the NHWC tile in shared memory.  Layers 1
// (2 inputs) and 3 (1 output) run on the CUDA cores: padded to MMA shapes
// they would waste most of the work.  The gradient with respect to a layer input is the same
// convolution with flipped, transposed weights; the weight gradient is a
// reduction over pixels on the CUDA cores with fixed-order block partials.
// Parameters are an FP32 master vector; every use packs them into the BF16
// matrices the kernels read.
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

constexpr int kK1 = kpad(kInP);   // 80
constexpr int kK2 = kpad(kHid);   // 144
constexpr int kKb3 = kpad(8);     // 80: layer-3 backward, input = 8 padded gradient channels

// BF16 operand matrices [Cout][K] and padded biases.
struct Packed {
  __nv_bfloat16* wt1;  // [16][80]
  __nv_bfloat16* wt2;  // [16][144]
  __nv_bfloat16* wt3;  // [8][144]
  __nv_bfloat16* wb3;  // [16][80]   d h2 = conv(d out, W3 flipped)
  __nv_bfloat16* wb2;  // [16][144]  d h1 = conv(d a2, W2 flipped)
  float *b1, *b2, *b3;  // [kHid], [kHid], [8]
  float* w1f;  // [9][2][kHid]  layer 1, BF16-rounded, for the CUDA-core forward
  float* w3f;  // [9][kHid]     layer 3, BF16-rounded
};

__global__ void pack_kernel(const float* p, Packed P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // forward layer 1: k = tap * 8 + ci
  if (i < kHid * kK1) {
    const int co = i / kK1, k = i % kK1, tap = k / kInP, ci = k % kInP;
    const float v = (k < 9 * kInP && ci < kIn) ? p[kOffW1 + (tap * kIn + ci) * kHid + co] : 0.f;
    P.wt1[i] = __float2bfloat16_rn(v);
  }
  if (i < kHid * kK2) {
    const int co = i / kK2, k = i % kK2, tap = k / kHid, ci = k % kHid;
    P.wt2[i] = __float2bfloat16_rn(p[kOffW2 + (tap * kHid + ci) * kHid + co]);
    // backward of layer 2: out channel = ci of W2, in channel = co of W2, taps flipped
    const int cin2 = co, cout2 = ci;  // rename: row = input channel of the forward layer
    P.wb2[i] = __float2bfloat16_rn(p[kOffW2 + ((8 - tap) * kHid + cin2) * kHid + cout2]);
  }
  if (i < 8 * kK2) {
    const int co = i / kK2, k = i % kK2, tap = k / kHid, ci = k % kHid;
    P.wt3[i] = __float2bfloat16_rn(co == 0 ? p[kOffW3 + tap * kHid + ci] : 0.f);
  }
  if (i < kHid * kKb3) {
    const int ci = i / kKb3, k = i % kKb3, tap = k / 8, co = k % 8;
    const float v = (k < 72 && co == 0) ? p[kOffW3 + (8 - tap) * kHid + ci] : 0.f;
    P.wb3[i] = __float2bfloat16_rn(v);
  }
  if (i < kHid) {
    P.b1[i] = p[kOffB1 + i];
    P.b2[i] = p[kOffB2 + i];
  }
  if (i < 9 * kIn * kHid) P.w1f[i] = __bfloat162float(__float2bfloat16_rn(p[kOffW1 + i]));
  if (i < 9 * kHid) P.w3f[i] = __bfloat162float(__float2bfloat16_rn(p[kOffW3 + i]));
  if (i < 8) P.b3[i] = i == 0 ? p[kOffB3] : 0.f;
}

FBME_DEV uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

FBME_DEV void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                             uint32_t b0, uint32_t b1) {
  asm volatile(
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

// Layer 2 forward (8 -> 8 channels, relu, BF16 NHWC output) on a 16 x 16
// pixel tile: 4 warps x 4 rows of 16 pixels.  An A fragment is one
// ldmatrix.x4 from the halo tile -- a matrix row is one pixel's 8 channels
// at one tap (16 bytes), so the four 8x8 matrices are pixels 0-7 / 8-15 at
// taps 2ks and 2ks+1 -- and the weight fragments and the bias stay in
// registers.  The MMA operands and their order are those of
// conv3x3_kernel<bf16, 8, 8, kOutReluBf16>, so the output is the same bit
// for bit, with a quarter of its shared-memory loads and half its halo
// overhead per pixel.
constexpr int kF8Rows = 16, kF8Cols = 16;
FBME_DEV void ldmatrix_x4(uint32_t addr, uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
               : "r"(addr));
}

__global__ void __launch_bounds__(128) conv3x3_fwd8_kernel(const __nv_bfloat16* x, const __nv_bfloat16* wt,
                                                          const float* bias, __nv_bfloat16* out, int H, int W) {
  constexpr int KP = kpad(8);
  constexpr int HW = kF8Rows + 2, WW = kF8Cols + 2, NP = HW * WW;
  __shared__ uint4 xs[NP + 1];  // halo tile, one pixel (8 BF16) each, then a zero pixel for padded taps
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int x0 = blockIdx.x * kF8Cols, y0 = blockIdx.y * kF8Rows, b = blockIdx.z;
  const long long img = static_cast<long long>(b) * H * W;
  constexpr int IT = (NP + 127) / 128;
  uint4 v[IT];
#pragma unroll
  for (int j = 0; j < IT; ++j) {
    const int i = tid + j * 128;
    const int gy = y0 - 1 + i / WW, gx = x0 - 1 + i % WW;
    v[j] = make_uint4(0u, 0u, 0u, 0u);
    if (i < NP && gy >= 0 && gy < H && gx >= 0 && gx < W)
      v[j] = *reinterpret_cast<const uint4*>(x + (img + static_cast<long long>(gy) * W + gx) * 8);
  }
  const uint32_t* wt32 = reinterpret_cast<const uint32_t*>(wt);
  uint32_t bq[KP / 16][2];
#pragma unroll
  for (int ks = 0; ks < KP / 16; ++ks) {
    bq[ks][0] = wt32[(g * KP + ks * 16 + t * 2) / 2];
    bq[ks][1] = wt32[(g * KP + ks * 16 + t * 2 + 8) / 2];
  }
  const float bias0 = bias[2 * t], bias1 = bias[2 * t + 1];
#pragma unroll
  for (int j = 0; j < IT; ++j) {
    const int i = tid + j * 128;
    if (i < NP) xs[i] = v[j];
  }
  if (tid == 0) xs[NP] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  // ldmatrix rows: lanes 8m..8m+7 address matrix m = (pixel half m&1, tap 2ks + (m>>1))
  const int mj = lane >> 3, pr = (lane & 7) + (mj & 1) * 8;
  float acc[4][4];
#pragma unroll
  for (int mf = 0; mf < 4; ++mf)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[mf][j] = 0.f;
#pragma unroll
  for (int ks = 0; ks < KP / 16; ++ks) {
    const int tap = 2 * ks + (mj >> 1);
#pragma unroll
    for (int mf = 0; mf < 4; ++mf) {
      const int yy = warp * 4 + mf;
      const int pix = tap < 9 ? (yy + tap / 3) * WW + pr + tap % 3 : NP;
      uint32_t a0, a1, a2, a3;
      ldmatrix_x4(smem_u32(&xs[pix]), a0, a1, a2, a3);
      mma_bf16_16816(acc[mf], a0, a1, a2, a3, bq[ks][0], bq[ks][1]);
    }
  }
#pragma unroll
  for (int mf = 0; mf < 4; ++mf) {
    const int gy = y0 + warp * 4 + mf;
    if (gy >= H) continue;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int gx = x0 + g + half * 8;
      if (gx >= W) continue;
      const long long pix = img + static_cast<long long>(gy) * W + gx;
      const float v0 = acc[mf][half * 2] + bias0, v1 = acc[mf][half * 2 + 1] + bias1;
      reinterpret_cast<uint32_t*>(out + pix * 8 + 2 * t)[0] = pack_bf16x2(fmaxf(v0, 0.f), fmaxf(v1, 0.f));
    }
  }
}

// Layers with few channels on the CUDA cores: 3x3 convolution, zero
// padding 1, from CIN channels of an NHWC BF16 input (stride CSTR) to COUT
// outputs over a 16 x 32 tile; each of the 128 threads computes 4 pixels
// of one column, so every input value loaded from shared memory serves up
// to 3 taps of 4 pixels and every weight vector 4 pixels.  The tile holds
// channel pairs, and the multiply-adds run on the paired FP32 FMA over
// pairs of output channels (layer 1) or input channels (layer 3): the
// kernel is bound by issued instructions, which this halves.  BF16-rounded
// weights w[tap][ci][co], FP32 accumulation.  RELU_BF16: relu, BF16 NHWC
// output with COUT channels; else FP32 channel 0.  With f1part (layer 1),
// input channel 1 is not read: it is the scene constant BF16(sum of the
// nparts feature partials f1part[b * 128 + 64 + k] / N), the value the
// third feature pass stores.
constexpr int kSmallTW = 16, kSmallTH = 32, kSmallThreads = 128, kSmallRows = 4;
template <int CIN, int CSTR, int COUT, bool RELU_BF16>
__global__ void __launch_bounds__(kSmallThreads)
conv_small_kernel(const __nv_bfloat16* x, const float* w, const float* bias, void* out, int H, int W,
                  const double* f1part = nullptr, int nparts = 0) {
  static_assert(CIN == 2 || CIN == 8, "input channels: one 32-bit or 128-bit load");
  static_assert(COUT == 8 || COUT == 1, "output channels");
  constexpr int TW = kSmallTW + 2, TH = kSmallTH + 2, NP = TW * TH, R = kSmallRows;
  constexpr int NW = 9 * CIN * COUT;
  __shared__ float2 xs2[(CIN / 2) * NP];  // channel pairs, pair-major: lanes read consecutive pairs
  __shared__ __align__(16) float ws[NW + 8];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kSmallTW, y0 = blockIdx.y * kSmallTH, b = blockIdx.z;
  const long long img = static_cast<long long>(b) * H * W;
  float c1 = 0.f;
  if (CIN == 2 && f1part) {
    double f1 = 0.0;
    for (int k = 0; k < nparts; ++k) f1 += f1part[b * 128 + 64 + k];
    c1 = __bfloat162float(__float2bfloat16_rn(static_cast<float>(f1 / (static_cast<double>(H) * W))));
  }
  // All of a thread's global loads are issued before any is stored.
  constexpr int IT = (NP + kSmallThreads - 1) / kSmallThreads;
  // CSTR == 1: channel 0 alone, one BF16 per pixel (channel 1 from f1part)
  using LoadT = typename std::conditional<CIN == 8, uint4,
                                          typename std::conditional<CSTR == 1, uint16_t, uint32_t>::type>::type;
  LoadT v[IT];
  bool in[IT];
#pragma unroll
  for (int j = 0; j < IT; ++j) {
    const int pix = tid + j * kSmallThreads;
    const int gy = y0 - 1 + pix / TW, gx = x0 - 1 + pix % TW;
    in[j] = pix < NP && gy >= 0 && gy < H && gx >= 0 && gx < W;
    v[j] = LoadT{};
    if (in[j]) v[j] = *reinterpret_cast<const LoadT*>(x + (img + static_cast<long long>(gy) * W + gx) * CSTR);
  }
#pragma unroll
  for (int j = 0; j < IT; ++j) {
    const int pix = tid + j * kSmallThreads;
    if (pix >= NP) break;
    if constexpr (CIN == 8) {
      const uint32_t u[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        xs2[k * NP + pix] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u[k]));
    } else if constexpr (CSTR == 1) {
      const float f0 = __bfloat162float(__ushort_as_bfloat16(v[j]));
      xs2[pix] = make_float2(f0, in[j] ? c1 : 0.f);
    } else {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v[j]));
      xs2[pix] = make_float2(f.x, f1part ? (in[j] ? c1 : 0.f) : f.y);
    }
  }
  for (int i = tid; i < NW; i += kSmallThreads) ws[i] = w[i];
  if (tid < COUT) ws[NW + tid] = bias[tid];
  __syncthreads();
  const int px = tid % kSmallTW, r0 = (tid / kSmallTW) * R;
  // COUT == 8: acc2[p][k] holds output channels (2k, 2k+1); COUT == 1:
  // acc2[p][0] holds the sums over the even and the odd input channels
  constexpr int NA = COUT == 8 ? 4 : 1;
  float2 acc2[R][NA];
#pragma unroll
  for (int p = 0; p < R; ++p)
#pragma unroll
    for (int k = 0; k < NA; ++k) acc2[p][k] = make_float2(0.f, 0.f);
#pragma unroll
  for (int cp = 0; cp < CIN / 2; ++cp) {
    float2 xw[R + 2][3];
#pragma unroll
    for (int r = 0; r < R + 2; ++r)
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) xw[r][dx] = xs2[cp * NP + (r0 + r) * TW + px + dx];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      if constexpr (COUT == 8) {
        const float4* wp = reinterpret_cast<const float4*>(ws + (tap * CIN + 2 * cp) * 8);
        const float4 a0 = wp[0], a1 = wp[1], b0 = wp[2], b1 = wp[3];  // channels 2cp and 2cp + 1
        const float2 wa[4] = {make_float2(a0.x, a0.y), make_float2(a0.z, a0.w), make_float2(a1.x, a1.y),
                              make_float2(a1.z, a1.w)};
        const float2 wb[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w), make_float2(b1.x, b1.y),
                              make_float2(b1.z, b1.w)};
#pragma unroll
        for (int p = 0; p < R; ++p) {
          const float2 xv = xw[p + tap / 3][tap % 3];
          const float2 xa = make_float2(xv.x, xv.x), xb = make_float2(xv.y, xv.y);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            acc2[p][k] = __ffma2_rn(xa, wa[k], acc2[p][k]);
            acc2[p][k] = __ffma2_rn(xb, wb[k], acc2[p][k]);
          }
        }
      } else {
        const float2 wv = *reinterpret_cast<const float2*>(ws + tap * CIN + 2 * cp);
#pragma unroll
        for (int p = 0; p < R; ++p) acc2[p][0] = __ffma2_rn(xw[p + tap / 3][tap % 3], wv, acc2[p][0]);
      }
    }
  }
  const int gx = x0 + px;
  if (gx >= W) return;
#pragma unroll
  for (int p = 0; p < R; ++p) {
    const int gy = y0 + r0 + p;
    if (gy >= H) break;
    const long long pix = img + static_cast<long long>(gy) * W + gx;
    if constexpr (RELU_BF16) {
      static_assert(!RELU_BF16 || COUT == 8, "one 128-bit store per pixel");
      uint32_t o[4];
#pragma unroll
      for (int k = 0; k < 4; ++k)
        o[k] = pack_bf16x2(fmaxf(acc2[p][k].x + ws[NW + 2 * k], 0.f), fmaxf(acc2[p][k].y + ws[NW + 2 * k + 1], 0.f));
      *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(out) + pix * COUT) = make_uint4(o[0], o[1], o[2], o[3]);
    } else {
      static_cast<float*>(out)[pix] = (acc2[p][0].x + acc2[p][0].y) + ws[NW];
    }
  }
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
  if (pass >= 1) {
    for (int k = 0; k < gridDim.x; ++k) mean += part[b * 128 + k];
    mean = fmax(mean / static_cast<double>(N), 1e-30);
  }
  if (pass == 2) {
    for (int k = 0; k < gridDim.x; ++k) f1 += part[b * 128 + 64 + k];
    f1 /= static_cast<double>(N);
  }
  if (pass == 1 && compact && (N & 3) == 0) {
    // four pixels a step: two 16-byte loads, one 8-byte store of BF16 f0
    const float4* src = reinterpret_cast<const float4*>(bp + b * N);
    uint2* dst = reinterpret_cast<uint2*>(x8 + b * N);
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

// prior0 = max(data_power / N * exp(out), floor) and its per-block sums
// (slot 0 of the UAMP partial array, as the plain initialisation writes).
__global__ void __launch_bounds__(256) warm_prior_kernel(const float* out, long long N,
                                                         const float* data_power, const float* floor_,
                                                         float* gamma, double* upart) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const float base = data_power[b] / static_cast<float>(N), fl = floor_[b];
  double acc = 0.0;
  for (long long n = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float o = fminf(fmaxf(out[b * N + n], -40.f), 40.f);
    const float gm = fmaxf(base * expf(o), fl);
    gamma[b * N + n] = gm;
    acc += gm;
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0)
    upart[(static_cast<long long>(b) * kMaxTilesPerScene + blockIdx.x) * kPartSlots] = s;
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
  P.wt1 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kK1 * 2));
  P.wt2 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kK2 * 2));
  P.wt3 = reinterpret_cast<__nv_bfloat16*>(take(8 * kK2 * 2));
  P.wb3 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kKb3 * 2));
  P.wb2 = reinterpret_cast<__nv_bfloat16*>(take(kHid * kK2 * 2));
  P.b1 = reinterpret_cast<float*>(take(kHid * 4));
  P.b2 = reinterpret_cast<float*>(take(kHid * 4));
  P.b3 = reinterpret_cast<float*>(take(8 * 4));
  P.w1f = reinterpret_cast<float*>(take(9 * kIn * kHid * 4));
  P.w3f = reinterpret_cast<float*>(take(9 * kHid * 4));
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
int feature_parts(int H, int W) {
  return static_cast<int>(std::min<long long>(64, (static_cast<long long>(H) * W + 255) / 256));
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
void cnn_forward(const float* params, int B, int H, int W, void* ws, float* out, cudaStream_t st,
                 bool compact) {
  using namespace cnn;
  const CnnLayout L = cnn_layout(B, H, W);
  uint8_t* w = static_cast<uint8_t*>(ws);
  const Packed P = packed_at(w + L.packed);
  pack_kernel<<<(kHid * kK2 + 255) / 256, 256, 0, st>>>(params, P);
  const dim3 grid(W / kTileW, H / kTileH, B);
  auto* x8 = reinterpret_cast<const __nv_bfloat16*>(w + L.x8);
  auto* h1 = reinterpret_cast<__nv_bfloat16*>(w + L.h1);
  auto* h2 = reinterpret_cast<__nv_bfloat16*>(w + L.h2);
  const dim3 grid_small((W + kSmallTW - 1) / kSmallTW, (H + kSmallTH - 1) / kSmallTH, B);
  if (compact)
    conv_small_kernel<kIn, 1, kHid, true><<<grid_small, kSmallThreads, 0, st>>>(
        x8, P.w1f, P.b1, h1, H, W, reinterpret_cast<const double*>(w + L.fpart), feature_parts(H, W));
  else
    conv_small_kernel<kIn, kInP, kHid, true><<<grid_small, kSmallThreads, 0, st>>>(
        x8, P.w1f, P.b1, h1, H, W, reinterpret_cast<const double*>(w + L.fpart), feature_parts(H, W));
  static_assert(kHid == 8, "conv3x3_fwd8_kernel is the 8 -> 8 layer");
  conv3x3_fwd8_kernel<<<dim3((W + kF8Cols - 1) / kF8Cols, (H + kF8Rows - 1) / kF8Rows, B), 128, 0, st>>>(
      h1, P.wt2, P.b2, h2, H, W);
  float* wout = reinterpret_cast<float*>(w + L.out);  // kept for cnn_backward
  conv_small_kernel<kHid, kHid, 1, false><<<grid_small, kSmallThreads, 0, st>>>(h2, P.w3f, P.b3, wout, H, W);
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

// Warm start inside a plan: features of A^H y, forward, prior0 and its
// block sums; the caller then re-runs the scalar initialisation.
void cnn_warm_prior(const float* params, const float2* bp, int B, int H, int W, void* ws,
                    const float* data_power, const float* floor_, float* gamma, double* upart,
                    int nblocks, cudaStream_t st, const float* ebp) {
  using namespace cnn;
  // f0 alone, one BF16 per pixel (the first layer takes f1 from the partials);
  // with the backprojection power `ebp` the statistics pass is not repeated
  if (ebp) {
    const CnnLayout L = cnn_layout(B, H, W);
    seed_feature_sum_kernel<<<B, 64, 0, st>>>(ebp, B, feature_parts(H, W),
                                             reinterpret_cast<double*>(static_cast<uint8_t*>(ws) + L.fpart));
    features_passes(bp, B, H, W, ws, 2, st, true, 1);
  } else {
    features_passes(bp, B, H, W, ws, 2, st, true);
  }
  const CnnLayout L = cnn_layout(B, H, W);
  float* out = reinterpret_cast<float*>(static_cast<uint8_t*>(ws) + L.out);
  cnn_forward(params, B, H, W, ws, out, st, true);
  warm_prior_kernel<<<dim3(nblocks, B), 256, 0, st>>>(out, static_cast<long long>(H) * W, data_power,
                                                      floor_, gamma, upart);
}

void warm_prior_from_map(const float* map, int B, long long N, const float* data_power, const float* floor_,
                         float* gamma, double* upart, int nblocks, cudaStream_t st) {
  using namespace cnn;
  warm_prior_kernel<<<dim3(nblocks, B), 256, 0, st>>>(map, N, data_power, floor_, gamma, upart);
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
