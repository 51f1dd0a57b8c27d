// Observation masks (non-rectangular sampling) for the plan path.
//
// Replaces the observed-sample restriction of PrefixFourierOperator
// (torch_sbl/operators.py:57-75 observed_indices, 473-496 restrict /
// expand) as the plan uses it: data keep the M1 x M2 block layout with
// unobserved samples held at zero, which makes A^H of a zero-filled block
// the masked adjoint and leaves the stage kernels unchanged.  The data-
// space kernels mask their outputs (the message update, the residual sum),
// scalar updates count the observed samples, and the active-set Gram
// A_S^H A_S becomes a 2-D table:
//
//   G(d1, d2) = sum over observed (m1, m2) of exp(+2 pi i (m1 d1 / N1 + m2 d2 / N2))
//
// (for the full block it factors into the two Dirichlet kernels), built
// here in FP64 from integer phases, in two passes over the axes.
#include <math.h>

#include "common.cuh"
#include "kernels.cuh"

namespace fbme {

namespace {

// Mask bytes normalised to 0 / 1 and the number of observed samples.
__global__ void __launch_bounds__(1024) mask_copy_count_kernel(const uint8_t* in, long long m, uint8_t* out,
                                                               unsigned long long* count) {
  __shared__ unsigned long long part[32];
  unsigned long long c = 0;
  for (long long i = threadIdx.x; i < m; i += blockDim.x) {
    const uint8_t v = in[i] ? 1 : 0;
    out[i] = v;
    c += v;
  }
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += part[w];
    *count = t;
  }
}

// exp(+2 pi i k / L) from the integer phase k mod L, in FP64.
FBME_DEV double2 twiddle64(long long k, int L) {
  double s, c;
  sincospi(2.0 * static_cast<double>(k % L) / static_cast<double>(L), &s, &c);
  return make_double2(c, s);
}

// Pass 1: R[m1][d2] = sum_{m2} mask[m1][m2] exp(+2 pi i m2 d2 / N2).
__global__ void __launch_bounds__(256) gram_pass1_kernel(const uint8_t* mask, int m1n, int m2n, int n2,
                                                         double2* r) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<long long>(m1n) * n2) return;
  const int a = static_cast<int>(i / n2), d2 = static_cast<int>(i % n2);
  double re = 0.0, im = 0.0;
  for (int b = 0; b < m2n; ++b) {
    if (!mask[static_cast<long long>(a) * m2n + b]) continue;
    const double2 w = twiddle64(static_cast<long long>(b) * d2, n2);
    re += w.x;
    im += w.y;
  }
  r[i] = make_double2(re, im);
}

// Pass 2: G[d1][d2] = sum_{m1} R[m1][d2] exp(+2 pi i m1 d1 / N1).
__global__ void __launch_bounds__(256) gram_pass2_kernel(const double2* r, int m1n, int n1, int n2, float2* g) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<long long>(n1) * n2) return;
  const int d1 = static_cast<int>(i / n2), d2 = static_cast<int>(i % n2);
  double re = 0.0, im = 0.0;
  for (int a = 0; a < m1n; ++a) {
    const double2 v = r[static_cast<long long>(a) * n2 + d2];
    const double2 w = twiddle64(static_cast<long long>(a) * d1, n1);
    re += v.x * w.x - v.y * w.y;
    im += v.x * w.y + v.y * w.x;
  }
  g[i] = make_float2(static_cast<float>(re), static_cast<float>(im));
}

// Masked copy of the caller's data: out[b][m] = mask[m] ? y[b][m] : 0.
__global__ void __launch_bounds__(256) mask_data_kernel(const float2* y, const uint8_t* mask, long long m,
                                                        float2* out) {
  const long long scene = blockIdx.y;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    out[scene * m + i] = mask[i] ? y[scene * m + i] : make_float2(0.f, 0.f);
}

}  // namespace

size_t mask_gram_scratch_bytes(const BatchShape& s) {
  return static_cast<size_t>(s.m1) * s.n2 * sizeof(double2) + 256;
}

cudaError_t mask_setup(const BatchShape& s, const uint8_t* mask_in, uint8_t* mask, float2* gram, void* scratch,
                       long long* observed, cudaStream_t st) {
  const long long m = s.m();
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(scratch);
  double2* r = reinterpret_cast<double2*>(static_cast<uint8_t*>(scratch) + 256);
  mask_copy_count_kernel<<<1, 1024, 0, st>>>(mask_in, m, mask, cnt);
  const long long n1r = static_cast<long long>(s.m1) * s.n2, nn = s.n();
  gram_pass1_kernel<<<static_cast<unsigned>((n1r + 255) / 256), 256, 0, st>>>(mask, s.m1, s.m2, s.n2, r);
  gram_pass2_kernel<<<static_cast<unsigned>((nn + 255) / 256), 256, 0, st>>>(r, s.m1, s.n1, s.n2, gram);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  unsigned long long h = 0;
  e = cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  *observed = static_cast<long long>(h);
  return e;
}

void mask_data(const BatchShape& s, const float2* y, const uint8_t* mask, float2* out, cudaStream_t st) {
  const long long m = s.m();
  const long long blocks = (m + 255) / 256;
  mask_data_kernel<<<dim3(static_cast<unsigned>(blocks < 256 ? blocks : 256), s.B), 256, 0, st>>>(y, mask, m, out);
}

}  // namespace fbme
