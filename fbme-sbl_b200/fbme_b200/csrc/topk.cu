// Per-scene top-K selection over order-preserving 32-bit float keys.
//
// Replaces torch.topk(score, K) at torch_sbl/solver.py:1931 (active set)
// and 4410 (residual-exchange additions).  Two launches:
//   topk_blocks_kernel  each CTA reduces an 8192-key slice of one scene to
//                       its k best: the keys at or above the k-th largest
//                       thread maximum, ranked by counting (radix select
//                       over all register-held keys as the fallback);
//   topk_merge_kernel   one CTA per scene sorts the candidates as 64-bit
//                       (key, ~index) words and keeps the k first, so the
//                       result is the exact top-k, largest first, ties by
//                       lower index.
#include "kernels.cuh"
#include "topk.cuh"

namespace fbme {

constexpr int kTopkBlockThreads = 512;
constexpr int kTopkKpt = 16;
constexpr int kTopkSlice = kTopkBlockThreads * kTopkKpt;  // 8192 keys per CTA
constexpr int kMergeMax = 2048;
FBME_DEV int topk_slices_dev(long long n) { return static_cast<int>((n + kTopkSlice - 1) / kTopkSlice); }

// FROM_SCORES: `in` holds float scores (converted to keys); else keys.
// The slice's k best lie among its keys at or above the k-th largest
// thread maximum (radix bound), typically a few dozen of the 8192.
template <bool FROM_SCORES>
FBME_DEV void topk_blocks_body(const void* in, long long n, int k, uint32_t* cand_key, int* cand_idx, int scene,
                               int blk, int nblk) {
  __shared__ TopkPrunedShared S;
  const uint32_t* kp = static_cast<const uint32_t*>(in) + scene * n;
  const float* sp = static_cast<const float*>(in) + scene * n;
  const long long base = static_cast<long long>(blk) * kTopkSlice + threadIdx.x;
  uint32_t key[kTopkKpt];
  uint32_t valid = 0u;
#pragma unroll
  for (int i = 0; i < kTopkKpt; ++i) {
    const long long e = base + static_cast<long long>(i) * kTopkBlockThreads;
    key[i] = 0u;
    if (e < n) {
      valid |= 1u << i;
      key[i] = FROM_SCORES ? float_key_t(sp[e]) : kp[e];
    }
  }
  const size_t off = (static_cast<size_t>(scene) * nblk + blk) * k;
  block_topk_pruned<kTopkKpt, false, TopkBound::kRadix>(
      key, valid, [&](int i) { return static_cast<int>(base + static_cast<long long>(i) * kTopkBlockThreads); }, k,
      S, cand_key + off, cand_idx + off);
}

template <bool FROM_SCORES>
__global__ void __launch_bounds__(kTopkBlockThreads, 2)
topk_blocks_kernel(const void* in, long long n, int k, uint32_t* cand_key, int* cand_idx) {
  topk_blocks_body<FROM_SCORES>(in, n, k, cand_key, cand_idx, blockIdx.y, blockIdx.x, gridDim.x);
}

// Several shape buckets' slices in one launch (blockIdx.z: the bucket;
// blocks past a bucket's own slices or scenes return).
__global__ void __launch_bounds__(kTopkBlockThreads, 2) topk_blocks_multi_kernel(const TopkJobs J) {
  const TopkJob& j = J.j[blockIdx.z];
  const int nblk = topk_slices_dev(j.n);
  if (static_cast<int>(blockIdx.x) >= nblk || static_cast<int>(blockIdx.y) >= j.B) return;
  topk_blocks_body<false>(j.keys, j.n, j.k, j.cand_key, j.cand_idx, blockIdx.y, blockIdx.x, nblk);
}

template <typename Idx>
FBME_DEV void topk_merge_body(const uint32_t* cand_key, const int* cand_idx, int ncand, int k, Idx* out_idx,
                              float* out_val, int scene) {
  __shared__ unsigned long long s[kMergeMax];
  int np = 1;
  while (np < ncand) np <<= 1;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    unsigned long long w = 0ull;
    if (i < ncand) {
      const size_t e = static_cast<size_t>(scene) * ncand + i;
      w = (static_cast<unsigned long long>(cand_key[e]) << 32) |
          static_cast<unsigned long long>(0xFFFFFFFFu - static_cast<uint32_t>(cand_idx[e]));
    }
    s[i] = w;
  }
  __syncthreads();
  // bitonic sort, descending
  for (int size = 2; size <= np; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < np; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool desc = (i & size) == 0;
          const unsigned long long a = s[i], b = s[j];
          if (desc ? (a < b) : (a > b)) {
            s[i] = b;
            s[j] = a;
          }
        }
      }
      __syncthreads();
    }
  if (threadIdx.x < k) {
    const unsigned long long w = s[threadIdx.x];
    out_idx[scene * k + threadIdx.x] = static_cast<Idx>(0xFFFFFFFFu - static_cast<uint32_t>(w));
    out_val[scene * k + threadIdx.x] = key_to_float(static_cast<uint32_t>(w >> 32));
  }
}

template <typename Idx>
__global__ void __launch_bounds__(1024)
topk_merge_kernel(const uint32_t* cand_key, const int* cand_idx, int ncand, int k, Idx* out_idx,
                  float* out_val) {
  topk_merge_body<Idx>(cand_key, cand_idx, ncand, k, out_idx, out_val, blockIdx.x);
}

__global__ void __launch_bounds__(1024) topk_merge_multi_kernel(const TopkMergeJobs J) {
  const TopkMergeJob& j = J.j[blockIdx.z];
  if (static_cast<int>(blockIdx.x) >= j.B) return;
  topk_merge_body<int>(j.cand_key, j.cand_idx, j.ncand, j.k, j.out_idx, j.out_val, blockIdx.x);
}

int topk_slices(long long n) { return static_cast<int>((n + kTopkSlice - 1) / kTopkSlice); }

void launch_topk_blocks_multi(const TopkJobs& J, int max_slices, int max_b, cudaStream_t st) {
  topk_blocks_multi_kernel<<<dim3(max_slices, max_b, J.n), kTopkBlockThreads, 0, st>>>(J);
}
void launch_topk_merge_multi(const TopkMergeJobs& J, int max_b, cudaStream_t st) {
  topk_merge_multi_kernel<<<dim3(max_b, 1, J.n), 1024, 0, st>>>(J);
}

void launch_topk_blocks(const uint32_t* keys, long long n, int k, int B, uint32_t* cand_key, int* cand_idx,
                        cudaStream_t st) {
  topk_blocks_kernel<false>
      <<<dim3(topk_slices(n), B), kTopkBlockThreads, 0, st>>>(keys, n, k, cand_key, cand_idx);
}

void launch_topk(const uint32_t* keys, long long n, int k, int B, uint32_t* cand_key, int* cand_idx,
                 int* out_idx, float* out_val, cudaStream_t st) {
  launch_topk_blocks(keys, n, k, B, cand_key, cand_idx, st);
  topk_merge_kernel<int><<<B, 1024, 0, st>>>(cand_key, cand_idx, topk_slices(n) * k, k, out_idx, out_val);
}

void launch_topk_merge(const uint32_t* cand_key, const int* cand_idx, int ncand, int k, int B,
                       int* out_idx, float* out_val, cudaStream_t st) {
  topk_merge_kernel<int><<<B, 1024, 0, st>>>(cand_key, cand_idx, ncand, k, out_idx, out_val);
}

// Candidate scratch of the score top-k: per row, one k-list per 8192-score slice.
size_t topk_scratch_bytes(long long n, int k, int batch) {
  return static_cast<size_t>(batch) * topk_slices(n) * k * (sizeof(uint32_t) + sizeof(int));
}

const char* topk_check(long long n, int k, int batch) {
  if (n < 1 || batch < 1) return "n and batch must be positive";
  if (batch > 65535) return "batch above 65535 (rows run on gridDim.y)";
  if (k < 1 || k > 32) return "k must be in [1, 32]";
  if (k > n) return "k exceeds n";
  if (n > (1LL << 31) - 1) return "n above 2^31 - 1";
  if (static_cast<long long>(topk_slices(n)) * k > kMergeMax)
    return "n too large for the candidate merge (ceil(n/8192)*k must be <= 2048)";
  return nullptr;
}

// Top-k of float scores with candidates in `scratch` (topk_scratch_bytes).
void topk_scores(const float* scores, long long n, int k, int batch, void* scratch,
                 int64_t* indices, float* values, cudaStream_t st) {
  const int nblk = topk_slices(n);
  uint32_t* ck = static_cast<uint32_t*>(scratch);
  int* ci = reinterpret_cast<int*>(ck + static_cast<size_t>(batch) * nblk * k);
  topk_blocks_kernel<true><<<dim3(nblk, batch), kTopkBlockThreads, 0, st>>>(scores, n, k, ck, ci);
  topk_merge_kernel<int64_t><<<batch, 1024, 0, st>>>(ck, ci, nblk * k, k, indices, values);
}

}  // namespace fbme

// ---------------------------------------------------------------------------
// Allocation-free top-k (C ABI fbme_topk_static).
//
// For callers that cannot allocate device memory when they need a top-k:
// code that runs while another component captures a CUDA graph (allocation
// is not allowed during global-mode stream capture), real-time hosts that
// freeze their memory budget after start-up, and FFI hosts that only receive
// device pointers from another framework.  The candidate scratch lives in a
// library-owned, file-scope device array instead of a caller workspace.
// ---------------------------------------------------------------------------
#include <cuda.h>

#include <mutex>
#include <string>

namespace {

constexpr size_t kStaticScratchBytes = FBME_TOPK_STATIC_SCRATCH_BYTES;
// Held by every GPU that loads this library until the process exits.  All
// calls share it; its contents persist from the last call.
__device__ __align__(256) unsigned char g_topk_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
// Per device: the array's device address and the unique ID of the context
// it was looked up in.  cudaDeviceReset destroys the context and a later
// call runs in a new one (new ID), so the address is looked up again then.
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};
thread_local std::string g_static_error;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique ID of the calling thread's current context (0 when it cannot be
// read).  The driver functions come through the runtime's entry-point
// query, so the library needs no link against libcuda.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// Device address of g_topk_scratch on the current device, looked up with
// that device current: once per device, and again whenever the device's
// context has changed since (after cudaDeviceReset).  In host code the
// array's name is only a host-side stand-in, never a device address.
int static_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    g_static_error = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return FBME_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    g_static_error = "device ordinal outside the static scratch table";
    return FBME_ERR_UNSUPPORTED;
  }
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_topk_scratch);
    if (e != cudaSuccess || !p) {
      g_static_error = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return FBME_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return FBME_OK;
}

}  // namespace

extern "C" int fbme_topk_static(const float* scores, int64_t n, int32_t k, int32_t batch,
                                int64_t* indices, float* values, fbme_stream_t stream) {
  if (!scores || !indices || !values) {
    g_static_error = "NULL argument";
    return FBME_ERR_INVALID;
  }
  if (const char* why = fbme::topk_check(n, k, batch)) {
    g_static_error = why;
    return FBME_ERR_INVALID;
  }
  const size_t need = fbme::topk_scratch_bytes(n, k, batch);
  if (need > kStaticScratchBytes) {
    g_static_error = "fbme_topk_static: batch * ceil(n/8192) * k * 8 bytes exceeds the " +
                     std::to_string(kStaticScratchBytes) + "-byte static scratch";
    return FBME_ERR_INVALID;
  }
  // An error left pending by an earlier, unrelated launch is reported as
  // such, before anything is launched, so it is not taken for this call's.
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    g_static_error = std::string("fbme_topk_static: error pending from an earlier call: ") +
                     cudaGetErrorString(pending);
    return FBME_ERR_CUDA;
  }
  void* scratch = nullptr;
  const int rc = static_scratch(&scratch);
  if (rc != FBME_OK) return rc;
  // Every candidate slot is written before it is read: nothing to clear.
  fbme::topk_scores(scores, n, k, batch, scratch, indices, values,
                    reinterpret_cast<cudaStream_t>(stream));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_static_error = std::string("fbme_topk_static: ") + cudaGetErrorString(e);
    return FBME_ERR_CUDA;
  }
  return FBME_OK;
}

extern "C" const char* fbme_topk_static_error(void) { return g_static_error.c_str(); }
