// Unfused variational ARD prior update of the UAMP path.
//
// Replaces uamp_prior_update / _uamp_prior_kernel
// (torch_sbl/triton_kernels.py:670-735, 196-235), the prior update that
// torch_sbl/solver.py:1605-1625 takes when the UAMP posterior did not
// already damp the prior (the plans fold the same arithmetic into the
// denoiser; this entry keeps the stand-alone form):
//
//   m2      = re(mu)^2 + im(mu)^2 + v
//   cand    = clamp((m2 + hyper_rate) / (1 + hyper_shape), floor, maximum)
//   gamma'  = max(damping * gamma + (1 - damping) * cand, floor)
//
// Every operation is rounded on its own (no contraction into FMAs), in the
// order written, so the result equals the same expression evaluated one
// float32 operation at a time.  Memory-bound: 20 bytes read and 4 written
// per coefficient, 16-byte accesses where the rows allow them.
#include "common.cuh"
#include "kernels.cuh"

namespace fbme {

namespace {

constexpr int kPriorThreads = 256;
constexpr int kPriorPerThread = 4;

struct PriorArgs {
  const float2* mean;
  const float* var;
  const float* old_prior;
  const float* floor_;
  float* out;
  long long n;
  float hyper_shape, hyper_rate, damping, maximum;
};

FBME_DEV float prior_one(const PriorArgs& a, float2 m, float v, float g, float fl) {
  const float m2 = __fadd_rn(__fadd_rn(__fmul_rn(m.x, m.x), __fmul_rn(m.y, m.y)), v);
  float cand = __fdiv_rn(__fadd_rn(m2, a.hyper_rate), __fadd_rn(1.0f, a.hyper_shape));
  cand = fmaxf(fl, fminf(a.maximum, cand));
  const float upd = __fadd_rn(__fmul_rn(a.damping, g), __fmul_rn(__fsub_rn(1.0f, a.damping), cand));
  return fmaxf(upd, fl);
}

// blockIdx.y = scene; each thread handles kPriorPerThread consecutive
// coefficients (one float4 of v / gamma, two of mean) when the scene's row
// is 16-byte aligned, else element by element.
__global__ void __launch_bounds__(kPriorThreads) prior_update_kernel(const PriorArgs a, int vec) {
  const long long scene = blockIdx.y;
  const long long i0 = (static_cast<long long>(blockIdx.x) * kPriorThreads + threadIdx.x) * kPriorPerThread;
  if (i0 >= a.n) return;
  const long long base = scene * a.n;
  const float fl = a.floor_[scene];
  if (vec && i0 + kPriorPerThread <= a.n) {
    const float4 m01 = *reinterpret_cast<const float4*>(a.mean + base + i0);
    const float4 m23 = *reinterpret_cast<const float4*>(a.mean + base + i0 + 2);
    const float4 v = *reinterpret_cast<const float4*>(a.var + base + i0);
    const float4 g = *reinterpret_cast<const float4*>(a.old_prior + base + i0);
    float4 r;
    r.x = prior_one(a, make_float2(m01.x, m01.y), v.x, g.x, fl);
    r.y = prior_one(a, make_float2(m01.z, m01.w), v.y, g.y, fl);
    r.z = prior_one(a, make_float2(m23.x, m23.y), v.z, g.z, fl);
    r.w = prior_one(a, make_float2(m23.z, m23.w), v.w, g.w, fl);
    *reinterpret_cast<float4*>(a.out + base + i0) = r;
    return;
  }
  for (long long i = i0; i < i0 + kPriorPerThread && i < a.n; ++i)
    a.out[base + i] = prior_one(a, a.mean[base + i], a.var[base + i], a.old_prior[base + i], fl);
}

}  // namespace

void uamp_prior_update(const float2* mean, const float* var, const float* old_prior, const float* floor_,
                       int batch, long long n, float hyper_shape, float hyper_rate, float damping,
                       float maximum, float* out, cudaStream_t st) {
  PriorArgs a{mean, var, old_prior, floor_, out, n, hyper_shape, hyper_rate, damping, maximum};
  const auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  const int vec = (n % kPriorPerThread == 0) && aligned(mean) && aligned(var) && aligned(old_prior) &&
                  aligned(out);
  const long long per_block = static_cast<long long>(kPriorThreads) * kPriorPerThread;
  const unsigned gx = static_cast<unsigned>((n + per_block - 1) / per_block);
  prior_update_kernel<<<dim3(gx, batch), kPriorThreads, 0, st>>>(a, vec);
}

}  // namespace fbme
