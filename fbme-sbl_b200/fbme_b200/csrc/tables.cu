// Constant tables of a plan: pre-swizzled split-BF16 DFT twiddle blocks and
// the Dirichlet kernels used by the reduced (active-set) posterior.
#include "common.cuh"
#include "kernels.cuh"

namespace fbme {

// Twiddle block layout for one axis length L and sign s:
//   block (ct, kc, p) = real columns [ct*NT, ct*NT+NT) x real K [kc*64, kc*64+64)
//   of part p of E, stored K-major with the 128-byte swizzle, NT*128 bytes.
// E[2k+a][2c+b] = [[Re w, Im w], [-Im w, Re w]][a][b], w = exp(s*2*pi*i*k*c/L),
// with k*c reduced modulo L in integers before the FP64 sin/cos, and zero
// for k >= L or c >= L.  Parts: hi = bf16(E), then bf16 of the remainders.
__global__ void twiddle_table_kernel(uint8_t* dst, int L, int sign, int n_tile, int col_tiles,
                                     int kchunks, int parts) {
  const long long total = static_cast<long long>(col_tiles) * kchunks * n_tile * 64;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int klocal = static_cast<int>(e % 64);
    const int row = static_cast<int>((e / 64) % n_tile);
    const long long blk = e / (64LL * n_tile);  // = ct * kchunks + kc
    const int kc = static_cast<int>(blk % kchunks);
    const int ct = static_cast<int>(blk / kchunks);
    const int cr = ct * n_tile + row, kr = kc * 64 + klocal;
    const int c = cr >> 1, b = cr & 1, k = kr >> 1, a = kr & 1;
    double val = 0.0;
    if (k < L && c < L) {
      const long long r = (static_cast<long long>(k) * c) % L;
      double sn, cs;
      sincospi(2.0 * static_cast<double>(r) / static_cast<double>(L), &sn, &cs);
      const double im = sign * sn;
      val = (a == 0) ? (b == 0 ? cs : im) : (b == 0 ? -im : cs);
    }
    uint8_t* base = dst + blk * static_cast<long long>(parts) * n_tile * 128;
    const uint32_t off = sw128_offset(row, klocal);
    double rem = val;
    for (int p = 0; p < parts; ++p) {
      const __nv_bfloat16 h = __double2bfloat16(rem);
      rem -= static_cast<double>(__bfloat162float(h));
      *reinterpret_cast<__nv_bfloat16*>(base + p * n_tile * 128 + off) = h;
    }
  }
}

// D[d] = sum_{m<M} exp(+2*pi*i*m*d/L) for d in [0, L): the Gram entries of
// prefix Fourier atoms, G[k][l] = D1[(n1k-n1l) mod N1] * D2[(n2k-n2l) mod N2].
// Summed in FP64 with integer phase reduction.
__global__ void dirichlet_kernel(float2* dst, int M, int L) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < L; d += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int m = 0; m < M; ++m) {
      const long long r = (static_cast<long long>(m) * d) % L;
      double sn, cs;
      sincospi(2.0 * static_cast<double>(r) / static_cast<double>(L), &sn, &cs);
      re += cs;
      im += sn;
    }
    dst[d] = make_float2(static_cast<float>(re), static_cast<float>(im));
  }
}

void launch_twiddle_table(uint8_t* dst, int L, int sign, int n_tile, int col_tiles, int kchunks,
                          int parts, cudaStream_t st) {
  twiddle_table_kernel<<<296, 256, 0, st>>>(dst, L, sign, n_tile, col_tiles, kchunks, parts);
}

void launch_dirichlet(float2* dst, int M, int L, cudaStream_t st) {
  dirichlet_kernel<<<(L + 127) / 128, 128, 0, st>>>(dst, M, L);
}

}  // namespace fbme
