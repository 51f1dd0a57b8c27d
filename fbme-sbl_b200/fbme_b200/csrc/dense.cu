// mode="dense": the exact posterior through the M x M data covariance
// (torch_sbl/solver.py:2962-2990 with 3025-3035; operators.py:282-297 and
// 418-442), per scene, in FP64 on the device:
//
//   lags      L(d) = sum_n gamma_n exp(-2 pi i d.n / N) for the sample lags
//             d in (-(M1-1)..M1-1) x (-(M2-1)..M2-1), separable (two passes)
//   Q         Q[i][j] = L(m_i - m_j) + noise delta_ij, plus the deterministic
//             loading of the CUDA Cholesky branch (m * eps64 * mean|diag|)
//   Cholesky  blocked right-looking, 32-column panels (one CTA per scene)
//             and 64 x 64 tiles of the trailing update (the whole GPU)
//   L^-1      blocked forward substitution on the identity, same split
//   Q^-1      = L^-H L^-1 (lower tiles, over the rows below each tile)
//   Q^-1 y, the lag sums of Q^-1 and the data diagonal
//             diag(A^H Q^-1 A) = Re N ifft2(lag sums); A^H Q^-1 y; the
//             residual energy from the identity y - A mean = (noise +
//             loading) Q^-1 y
//
// The reference's FP32 run loses the posterior variance gamma - gamma^2 dd to
// cancellation (its FP32 and FP64 runs differ by 50-230 times the norm on the
// C1 scenes); FP64 here keeps it, and matches the reference's FP64 run.
// Matrices are column-major ([j * M + i]) with the lower triangle in use.
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "stage.cuh"

namespace fbme {

namespace {

// The deterministic Cholesky loading m * eps * mean|diag| of the CUDA branch
// (solver.py:2907-2920) takes eps of the arithmetic's precision: FP64 here,
// as the reference's complex128 path does.
constexpr double kEps64 = 2.220446049250313e-16;
constexpr int kPanel = 32;   // Cholesky / inverse panel width
constexpr int kTile = 64;    // output tile of the update kernels
constexpr int kDk = 16;      // depth chunk of the update kernels

__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// exp(-2 pi i k / L), k < L, FP64
__global__ void dense_twiddle_kernel(double2* tw, int L) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L) return;
  double s, c;
  sincospi(-2.0 * static_cast<double>(k) / static_cast<double>(L), &s, &c);
  tw[k] = make_double2(c, s);
}

// w^(sign * e) from the table of w = exp(-2 pi i / L), e any integer
__device__ __forceinline__ double2 twid(const double2* tw, int L, long long e, int sign) {
  long long r = e % L;
  if (r < 0) r += L;
  const double2 w = tw[r];
  return sign < 0 ? w : make_double2(w.x, -w.y);
}

// Lag pass 1: T[b][n1][e2] = sum_n2 gamma[b][n1][n2] w2^(d2 n2), d2 = e2 - (M2 - 1)
__global__ void dense_lag1_kernel(const float* gamma, int B, int n1, int n2, int m2, const double2* tw2,
                                  double2* T) {
  const int W2 = 2 * m2 - 1;
  const long long total = static_cast<long long>(B) * n1 * W2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int e2 = static_cast<int>(t % W2);
    const long long r = t / W2;  // b * n1 + row
    const int d2 = e2 - (m2 - 1);
    const float* g = gamma + r * n2;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < n2; ++k) {
      const double2 w = twid(tw2, n2, static_cast<long long>(d2) * k, -1);
      const double v = g[k];
      acc.x += v * w.x;
      acc.y += v * w.y;
    }
    T[t] = acc;
  }
}

// Lag pass 2: lag[b][e1][e2] = sum_n1 w1^(d1 n1) T[b][n1][e2], d1 = e1 - (M1 - 1)
__global__ void dense_lag2_kernel(const double2* T, int B, int n1, int m1, int m2, const double2* tw1,
                                  double2* lag) {
  const int W1 = 2 * m1 - 1, W2 = 2 * m2 - 1;
  const long long total = static_cast<long long>(B) * W1 * W2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int e2 = static_cast<int>(t % W2);
    const long long r = t / W2;
    const int e1 = static_cast<int>(r % W1);
    const int b = static_cast<int>(r / W1);
    const int d1 = e1 - (m1 - 1);
    const double2* tb = T + static_cast<long long>(b) * n1 * W2 + e2;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < n1; ++k) acc = zadd(acc, zmul(twid(tw1, n1, static_cast<long long>(d1) * k, -1), tb[k * W2]));
    lag[t] = acc;
  }
}

// Q (lower triangle, column-major) from the lags, noise and loading.
__global__ void dense_build_q_kernel(const double2* lag, int B, int m1, int m2, const float* noise, float jitter,
                                     double2* Q) {
  const int M = m1 * m2, W1 = 2 * m1 - 1, W2 = 2 * m2 - 1;
  const long long MM = static_cast<long long>(M) * M;
  const long long total = static_cast<long long>(B) * MM;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int b = static_cast<int>(t / MM);
    const long long r = t - b * MM;
    const int j = static_cast<int>(r / M), i = static_cast<int>(r - static_cast<long long>(j) * M);
    if (i < j) continue;
    const int i1 = i / m2, i2 = i - (i / m2) * m2, j1 = j / m2, j2 = j - (j / m2) * m2;
    const double2* lb = lag + static_cast<long long>(b) * W1 * W2;
    double2 q = lb[(i1 - j1 + m1 - 1) * W2 + (i2 - j2 + m2 - 1)];
    if (i == j) {
      // every diagonal entry is L(0) + noise: the loading is m eps64 (L(0) + noise)
      const double dg = lb[(m1 - 1) * W2 + (m2 - 1)].x + noise[b];
      q = make_double2(dg + static_cast<double>(jitter) * kEps64 * fabs(dg), 0.0);
    }
    Q[t] = q;
  }
}


// The diagonal block [k, k + 32) of the Cholesky factor, in shared memory:
// one warp per scene, lane i owning row i of the block.
__global__ void __launch_bounds__(32) dense_diag_chol_kernel(double2* Q, int M, int k, int* status) {
  __shared__ double2 D[kPanel][kPanel + 1];
  double2* A = Q + static_cast<long long>(blockIdx.x) * M * M;
  const int nb = M - k < kPanel ? M - k : kPanel, lane = threadIdx.x;
  for (int c = 0; c < nb; ++c)
    if (lane < nb && lane >= c) D[lane][c] = A[static_cast<long long>(k + c) * M + k + lane];
  __syncwarp();
  for (int c = 0; c < nb; ++c) {
    double d = D[c][c].x;
    if (!(d > 0.0)) {
      if (lane == 0 && status)
        atomicOr(status + blockIdx.x, isfinite(d) ? FBME_STATUS_CHOLESKY : FBME_STATUS_NONFINITE);
      d = 2.2250738585072014e-308;
    }
    const double piv = sqrt(d);
    __syncwarp();
    if (lane > c && lane < nb) D[lane][c] = make_double2(D[lane][c].x / piv, D[lane][c].y / piv);
    if (lane == c) D[c][c] = make_double2(piv, 0.0);
    __syncwarp();
    if (lane > c && lane < nb) {
      const double2 li = D[lane][c];
      for (int j = c + 1; j <= lane; ++j) {
        const double2 v = zmulc(li, D[j][c]);
        D[lane][j] = make_double2(D[lane][j].x - v.x, D[lane][j].y - v.y);
      }
    }
    __syncwarp();
  }
  for (int c = 0; c < nb; ++c)
    if (lane < nb && lane >= c) A[static_cast<long long>(k + c) * M + k + lane] = D[lane][c];
}

// The panel below the diagonal block: L21 = A21 L11^-H, one warp per row r
// (lane c holding column k + c), forward over the block's columns.
__global__ void __launch_bounds__(256) dense_panel_trsm_kernel(double2* Q, int M, int k) {
  double2* A = Q + static_cast<long long>(blockIdx.y) * M * M;
  const int r = k + kPanel + blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= M) return;  // whole warps: r is uniform in a warp
  double2 a = A[static_cast<long long>(k + lane) * M + r];
  for (int c = 0; c < kPanel; ++c) {
    if (lane == c) {
      const double piv = A[static_cast<long long>(k + c) * M + k + c].x;
      a = make_double2(a.x / piv, a.y / piv);
    }
    const double2 x = make_double2(__shfl_sync(0xffffffffu, a.x, c), __shfl_sync(0xffffffffu, a.y, c));
    if (lane > c) {
      const double2 v = zmulc(x, A[static_cast<long long>(k + c) * M + k + lane]);  // x conj(L11[lane][c])
      a = make_double2(a.x - v.x, a.y - v.y);
    }
  }
  A[static_cast<long long>(k + lane) * M + r] = a;
}

// Rows [k, k + 32) of X = L^-1, forward substitution within the diagonal
// block: one warp per column j < k + 32, lane i holding row k + i.
__global__ void __launch_bounds__(256) dense_inv_panel_kernel(const double2* L, double2* X, int M, int k) {
  const long long MM = static_cast<long long>(M) * M;
  const double2* Lb = L + blockIdx.y * MM;
  double2* Xb = X + blockIdx.y * MM;
  const int nb = M - k < kPanel ? M - k : kPanel;
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= k + nb) return;
  const int row = k + lane;
  const bool own = lane < nb && row >= j;  // X is lower triangular
  double2 v = own ? Xb[static_cast<long long>(j) * M + row] : make_double2(0.0, 0.0);
  for (int c = 0; c < nb; ++c) {
    if (lane == c) {
      const double piv = Lb[static_cast<long long>(k + c) * M + k + c].x;
      v = make_double2(v.x / piv, v.y / piv);
    }
    const double2 x = make_double2(__shfl_sync(0xffffffffu, v.x, c), __shfl_sync(0xffffffffu, v.y, c));
    if (lane > c && lane < nb) {
      const double2 p = zmul(Lb[static_cast<long long>(k + c) * M + row], x);
      v = make_double2(v.x - p.x, v.y - p.y);
    }
  }
  if (own) Xb[static_cast<long long>(j) * M + row] = v;
}

// Tile updates over 64 x 64 output tiles (grid: tiles x scenes), depth in
// chunks of kDk staged in shared memory; thread (ti, tj) of 16 x 16 owns the
// rows i0 + ti + 16 a and columns j0 + tj + 16 b (a, b < 4), so that stores
// of consecutive threads are consecutive in a column.
//   MODE 0  Cholesky trailing update, lower tiles of rows/cols [k1, M):
//           Q[i][j] -= sum_{c in [k0, k1)} Q[i][c] conj(Q[j][c])
//   MODE 1  inverse update, rows [k1, M) x columns [0, k1):
//           X[i][j] -= sum_{c in [k0, k1)} L[i][c] X[c][j]
//   MODE 2  R = X^H X, lower tiles of [0, M), stored in both triangles:
//           R[i][j] = sum_{r >= i0} conj(X[r][i]) X[r][j]
template <int MODE>
__global__ void __launch_bounds__(256) dense_tile_kernel(double2* C, const double2* A, const double2* Xm, int M,
                                                         int k0, int k1) {
  __shared__ double2 As[kDk][kTile];
  __shared__ double2 Bs[kDk][kTile];
  const long long MM = static_cast<long long>(M) * M;
  const int scene = blockIdx.y;
  C += scene * MM;
  A += scene * MM;
  if (Xm) Xm += scene * MM;
  // tile coordinates
  int ti, tj, base_i, base_j;
  const int t = blockIdx.x;
  if (MODE == 1) {
    const int tcols = (k1 + kTile - 1) / kTile;
    ti = t / tcols;
    tj = t - ti * tcols;
    base_i = k1;
    base_j = 0;
  } else {
    ti = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    while (ti * (ti + 1) / 2 > t) --ti;
    tj = t - ti * (ti + 1) / 2;
    base_i = base_j = MODE == 0 ? k1 : 0;
  }
  const int i0 = base_i + ti * kTile, j0 = base_j + tj * kTile;
  const int tid = threadIdx.x, ri = tid & 15, rj = tid >> 4;
  double2 acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0.0, 0.0);
  const int d_begin = MODE == 2 ? i0 : k0;
  const int d_end = MODE == 2 ? M : (k1 < M ? k1 : M);
  for (int d0 = d_begin; d0 < d_end; d0 += kDk) {
    for (int u = tid; u < kDk * kTile; u += 256) {
      if (MODE == 2) {  // both operands read along a column of X (d fastest)
        const int d = u % kDk, e = u / kDk;
        const int r = d0 + d;
        const int i = i0 + e, j = j0 + e;
        double2 av = make_double2(0.0, 0.0), bv = make_double2(0.0, 0.0);
        // X is lower triangular; its upper part is never written
        if (r < d_end && i < M && r >= i) {
          const double2 x = Xm[static_cast<long long>(i) * M + r];
          av = make_double2(x.x, -x.y);
        }
        if (r < d_end && j < M && r >= j) bv = Xm[static_cast<long long>(j) * M + r];
        As[d][e] = av;
        Bs[d][e] = bv;
      } else {
        const int e = u % kTile, d = u / kTile;
        const int c = d0 + d;
        const int i = i0 + e;
        As[d][e] = (c < d_end && i < M) ? A[static_cast<long long>(c) * M + i] : make_double2(0.0, 0.0);
        if (MODE == 0) {
          const int j = j0 + e;
          double2 bv = make_double2(0.0, 0.0);
          if (c < d_end && j < M) {
            const double2 q = A[static_cast<long long>(c) * M + j];
            bv = make_double2(q.x, -q.y);
          }
          Bs[d][e] = bv;
        }
      }
    }
    if (MODE == 1) {  // X[c][j]: along a column of X (d fastest)
      for (int u = tid; u < kDk * kTile; u += 256) {
        const int d = u % kDk, e = u / kDk;
        const int c = d0 + d, j = j0 + e;
        Bs[d][e] = (c < d_end && j < M && c >= j) ? Xm[static_cast<long long>(j) * M + c] : make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int d = 0; d < kDk; ++d) {
      double2 av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[d][ri + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[d][rj + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          acc[a][b].x = fma(av[a].x, bv[b].x, fma(-av[a].y, bv[b].y, acc[a][b].x));
          acc[a][b].y = fma(av[a].x, bv[b].y, fma(av[a].y, bv[b].x, acc[a][b].y));
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int j = j0 + rj + 16 * b;
    if (j >= M) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = i0 + ri + 16 * a;
      if (i >= M || (MODE != 1 && i < j)) continue;
      double2* dst = C + static_cast<long long>(j) * M + i;
      if (MODE == 2) {  // R is stored in full (both triangles)
        *dst = acc[a][b];
        if (i != j) C[static_cast<long long>(i) * M + j] = make_double2(acc[a][b].x, -acc[a][b].y);
      } else {
        *dst = make_double2(dst->x - acc[a][b].x, dst->y - acc[a][b].y);
      }
    }
  }
}

// X = I (lower triangle) before the blocked inversion.
__global__ void dense_identity_kernel(double2* X, int B, int M) {
  const long long MM = static_cast<long long>(M) * M, total = B * MM;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long r = t % MM;
    const int j = static_cast<int>(r / M), i = static_cast<int>(r - static_cast<long long>(j) * M);
    if (i >= j) X[t] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
}


__device__ __forceinline__ double2 warp_sum2(double2 v) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  return v;
}

// z = Q^-1 y (y complex64 [B][M]): one warp per row i, over column i of the
// Hermitian R (z_i = sum_j conj(R[j][i]) y_j), coalesced.
__global__ void __launch_bounds__(256) dense_qinv_y_kernel(const double2* R, const float2* y, int B, int M,
                                                            double2* z) {
  const int b = blockIdx.y;
  const int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= M) return;
  const double2* col = R + static_cast<long long>(b) * M * M + static_cast<long long>(i) * M;
  const float2* yb = y + static_cast<long long>(b) * M;
  double2 acc = make_double2(0.0, 0.0);
  for (int j = lane; j < M; j += 32) {
    const double2 r = col[j];
    const float2 v = yb[j];
    acc.x += r.x * v.x + r.y * v.y;  // conj(r) * v
    acc.y += r.x * v.y - r.y * v.x;
  }
  acc = warp_sum2(acc);
  if (lane == 0) z[static_cast<long long>(b) * M + i] = acc;
}

// Lag sums of Q^-1 (operators.py:427-435): S[e1][e2] = sum of R[i][j] over
// the sample pairs with m_i - m_j = (e1 - (M1-1), e2 - (M2-1)); one warp
// per lag, lanes over the pairs in a fixed order.
__global__ void __launch_bounds__(256) dense_lag_sum_kernel(const double2* R, int B, int m1, int m2,
                                                             double2* S) {
  const int M = m1 * m2, W1 = 2 * m1 - 1, W2 = 2 * m2 - 1;
  const long long total = static_cast<long long>(B) * W1 * W2;
  const long long t = blockIdx.x * 8LL + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= total) return;
  const int e2 = static_cast<int>(t % W2);
  const long long r = t / W2;
  const int e1 = static_cast<int>(r % W1), b = static_cast<int>(r / W1);
  const int d1 = e1 - (m1 - 1), d2 = e2 - (m2 - 1);
  const double2* Rb = R + static_cast<long long>(b) * M * M;
  const int a1lo = d1 > 0 ? d1 : 0, a1hi = d1 < 0 ? m1 + d1 : m1;
  const int a2lo = d2 > 0 ? d2 : 0, a2hi = d2 < 0 ? m2 + d2 : m2;
  const int w = a2hi - a2lo, cnt = (a1hi - a1lo) * w;
  const int shift = d1 * m2 + d2;  // j = i - shift
  double2 acc = make_double2(0.0, 0.0);
  for (int u = lane; u < cnt; u += 32) {
    const int a1 = a1lo + u / w, a2 = a2lo + u % w;
    const int i = a1 * m2 + a2;
    acc = zadd(acc, Rb[static_cast<long long>(i - shift) * M + i]);
  }
  acc = warp_sum2(acc);
  if (lane == 0) S[t] = acc;
}

// Inverse-sign separable transform of a W1 x W2 rectangle of frequencies
// (offsets o1, o2) to the N1 x N2 grid:
//   out[n1][n2] = sum_{e1,e2} S[e1][e2] exp(+2 pi i ((e1+o1) n1 / N1 + (e2+o2) n2 / N2))
// pass 1: U[b][e1][n2]; pass 2: out (complex, or its real part).
__global__ void dense_inv1_kernel(const double2* S, int B, int W1, int W2, int o2, int n2, const double2* tw2,
                                  double2* U) {
  const long long total = static_cast<long long>(B) * W1 * n2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int k2 = static_cast<int>(t % n2);
    const long long r = t / n2;  // b * W1 + e1
    const double2* row = S + r * W2;
    double2 acc = make_double2(0.0, 0.0);
    for (int e2 = 0; e2 < W2; ++e2)
      acc = zadd(acc, zmul(row[e2], twid(tw2, n2, static_cast<long long>(e2 + o2) * k2, +1)));
    U[t] = acc;
  }
}
template <bool REAL>
__global__ void dense_inv2_kernel(const double2* U, int B, int W1, int o1, int n1, int n2, const double2* tw1,
                                  double2* out, double* out_re) {
  const long long total = static_cast<long long>(B) * n1 * n2;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int k2 = static_cast<int>(t % n2);
    const long long r = t / n2;
    const int k1 = static_cast<int>(r % n1), b = static_cast<int>(r / n1);
    const double2* ub = U + static_cast<long long>(b) * W1 * n2 + k2;
    double2 acc = make_double2(0.0, 0.0);
    for (int e1 = 0; e1 < W1; ++e1)
      acc = zadd(acc, zmul(twid(tw1, n1, static_cast<long long>(e1 + o1) * k1, +1), ub[static_cast<long long>(e1) * n2]));
    if (REAL)
      out_re[t] = acc.x;
    else
      out[t] = acc;
  }
}

// Residual energy |y - A mean|^2 of the exact posterior: A Gamma A^H =
// Q - (noise + loading) I, so y - A Gamma A^H Q^-1 y = (noise + loading) z
// with z = Q^-1 y; FP64, into the energy slots of the scalar update
// (slot 2 of tile 0; its other warps' slots zero).
__global__ void __launch_bounds__(256) dense_energy_kernel(const double2* z, const double2* lag, const float* noise,
                                                          float jitter, int m1, int m2, double* part) {
  __shared__ double red[8];
  const int b = blockIdx.x, M = m1 * m2, W1 = 2 * m1 - 1, W2 = 2 * m2 - 1;
  double acc = 0.0;
  for (int i = threadIdx.x; i < M; i += blockDim.x) {
    const double2 v = z[static_cast<long long>(b) * M + i];
    acc += v.x * v.x + v.y * v.y;
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double e = 0.0;
    for (int w = 0; w < 8; ++w) e += red[w];
    const double dg = lag[static_cast<long long>(b) * W1 * W2 + (m1 - 1) * W2 + (m2 - 1)].x + noise[b];
    const double load = static_cast<double>(noise[b]) + static_cast<double>(jitter) * kEps64 * fabs(dg);
    double* slot = part + static_cast<long long>(b) * kMaxTilesPerScene * kPartSlots + 2 * kPartWarps;
    slot[0] = load * load * e;
    for (int w = 1; w < kPartWarps; ++w) slot[w] = 0.0;
  }
}

// mean = gamma A^H Q^-1 y, posterior variance max(gamma - gamma^2 dd, 0),
// clipped relevance gamma dd (solver.py:3025-3029, 3156-3163); per-block
// relevance sums in partial slot 0, as cg_hutch_kernel's.
__global__ void __launch_bounds__(kEwThreads)
dense_finish_kernel(BatchShape s, const float* gamma, const double2* lift, const double* dd, float2* mean,
                    float* relc, float* pv_out, double* part) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const long long N = s.n();
  double acc = 0.0;
  for (long long n = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; n < N;
       n += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long e = b * N + n;
    const double g = gamma[e];
    const double2 l = lift[e];
    mean[e] = make_float2(static_cast<float>(g * l.x), static_cast<float>(g * l.y));
    const double d = dd[e];
    const float rc = static_cast<float>(fmin(fmax(g * d, 0.0), 1.0));
    relc[e] = rc;
    if (pv_out) pv_out[e] = static_cast<float>(fmax(g - g * g * d, 0.0));
    acc += rc;
  }
  write_block_partial(acc, red, part, b, blockIdx.x, 0 * kPartWarps);
}

int grid_of(long long n) {
  const long long g = (n + 255) / 256;
  return static_cast<int>(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

}  // namespace

// Workspace of the dense posterior: [Q / L / R][X] per scene (FP64
// complex M x M each), lags, pass buffers, Q^-1 y, lift, data diagonal and
// the FP64 twiddle tables.
size_t dense_bytes(const BatchShape& s) {
  const size_t B = s.B, M = s.m(), N = s.n();
  const size_t W1 = 2 * s.m1 - 1, W2 = 2 * s.m2 - 1;
  auto up = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t pass = std::max(std::max(static_cast<size_t>(s.n1) * W2, W1 * static_cast<size_t>(s.n2)),
                               static_cast<size_t>(s.m1) * s.n2);
  return 2 * up(B * M * M * sizeof(double2)) + 2 * up(B * W1 * W2 * sizeof(double2)) +
         up(B * pass * sizeof(double2)) + up(B * M * sizeof(double2)) + up(B * N * sizeof(double2)) +
         up(B * N * sizeof(double)) + up(s.n1 * sizeof(double2)) + up(s.n2 * sizeof(double2));
}

DenseBufs dense_bind(uint8_t* w, const BatchShape& s, cudaStream_t st) {
  const size_t B = s.B, M = s.m(), N = s.n();
  const size_t W1 = 2 * s.m1 - 1, W2 = 2 * s.m2 - 1;
  auto up = [](size_t v) { return (v + 255) & ~static_cast<size_t>(255); };
  const size_t pass = std::max(std::max(static_cast<size_t>(s.n1) * W2, W1 * static_cast<size_t>(s.n2)),
                               static_cast<size_t>(s.m1) * s.n2);
  DenseBufs d;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    uint8_t* p = w + o;
    o += up(bytes);
    return p;
  };
  d.Q = reinterpret_cast<double2*>(take(B * M * M * sizeof(double2)));
  d.X = reinterpret_cast<double2*>(take(B * M * M * sizeof(double2)));
  d.lag = reinterpret_cast<double2*>(take(B * W1 * W2 * sizeof(double2)));
  d.lsum = reinterpret_cast<double2*>(take(B * W1 * W2 * sizeof(double2)));
  d.pass = reinterpret_cast<double2*>(take(B * pass * sizeof(double2)));
  d.z = reinterpret_cast<double2*>(take(B * M * sizeof(double2)));
  d.lift = reinterpret_cast<double2*>(take(B * N * sizeof(double2)));
  d.dd = reinterpret_cast<double*>(take(B * N * sizeof(double)));
  d.tw1 = reinterpret_cast<double2*>(take(s.n1 * sizeof(double2)));
  d.tw2 = reinterpret_cast<double2*>(take(s.n2 * sizeof(double2)));
  dense_twiddle_kernel<<<(s.n1 + 255) / 256, 256, 0, st>>>(d.tw1, s.n1);
  dense_twiddle_kernel<<<(s.n2 + 255) / 256, 256, 0, st>>>(d.tw2, s.n2);
  return d;
}

void dense_posterior(const BatchShape& s, const DenseBufs& d, const float* gamma, const float* noise,
                     const float2* y, float jitter, float2* mean, float* relc, float* pv_out, double* part, int nb,
                     int* status, cudaStream_t st) {
  const int B = s.B, M = static_cast<int>(s.m()), m1 = s.m1, m2 = s.m2, n1 = s.n1, n2 = s.n2;
  const int W1 = 2 * m1 - 1, W2 = 2 * m2 - 1;
  // lags of the prior and the data covariance
  dense_lag1_kernel<<<grid_of(1LL * B * n1 * W2), 256, 0, st>>>(gamma, B, n1, n2, m2, d.tw2, d.pass);
  dense_lag2_kernel<<<grid_of(1LL * B * W1 * W2), 256, 0, st>>>(d.pass, B, n1, m1, m2, d.tw1, d.lag);
  dense_build_q_kernel<<<grid_of(1LL * B * M * M), 256, 0, st>>>(d.lag, B, m1, m2, noise, jitter, d.Q);
  // Cholesky
  for (int k = 0; k < M; k += kPanel) {
    dense_diag_chol_kernel<<<B, 32, 0, st>>>(d.Q, M, k, status);
    const int k1 = k + kPanel;
    if (k1 < M) {
      dense_panel_trsm_kernel<<<dim3((M - k1 + 7) / 8, B), 256, 0, st>>>(d.Q, M, k);
      const int T = (M - k1 + kTile - 1) / kTile;
      dense_tile_kernel<0><<<dim3(T * (T + 1) / 2, B), 256, 0, st>>>(d.Q, d.Q, nullptr, M, k, k1);
    }
  }
  // X = L^-1
  dense_identity_kernel<<<grid_of(1LL * B * M * M), 256, 0, st>>>(d.X, B, M);
  for (int k = 0; k < M; k += kPanel) {
    dense_inv_panel_kernel<<<dim3((std::min(k + kPanel, M) + 7) / 8, B), 256, 0, st>>>(d.Q, d.X, M, k);
    const int k1 = k + kPanel;
    if (k1 < M) {
      const int TI = (M - k1 + kTile - 1) / kTile, TJ = (k1 + kTile - 1) / kTile;
      dense_tile_kernel<1><<<dim3(TI * TJ, B), 256, 0, st>>>(d.X, d.Q, d.X, M, k, k1);
    }
  }
  // Q^-1 = X^H X into the factor's storage
  {
    const int T = (M + kTile - 1) / kTile;
    dense_tile_kernel<2><<<dim3(T * (T + 1) / 2, B), 256, 0, st>>>(d.Q, d.Q, d.X, M, 0, 0);
  }
  dense_qinv_y_kernel<<<dim3((M + 7) / 8, B), 256, 0, st>>>(d.Q, y, B, M, d.z);
  dense_energy_kernel<<<B, 256, 0, st>>>(d.z, d.lag, noise, jitter, m1, m2, part);
  // data diagonal: Re N ifft2 of the lag sums
  dense_lag_sum_kernel<<<static_cast<int>((1LL * B * W1 * W2 + 7) / 8), 256, 0, st>>>(d.Q, B, m1, m2, d.lsum);
  dense_inv1_kernel<<<grid_of(1LL * B * W1 * n2), 256, 0, st>>>(d.lsum, B, W1, W2, -(m2 - 1), n2, d.tw2, d.pass);
  dense_inv2_kernel<true><<<grid_of(1LL * B * n1 * n2), 256, 0, st>>>(d.pass, B, W1, -(m1 - 1), n1, n2, d.tw1,
                                                                         nullptr, d.dd);
  // A^H Q^-1 y: the same transform of the M1 x M2 block
  dense_inv1_kernel<<<grid_of(1LL * B * m1 * n2), 256, 0, st>>>(d.z, B, m1, m2, 0, n2, d.tw2, d.pass);
  dense_inv2_kernel<false><<<grid_of(1LL * B * n1 * n2), 256, 0, st>>>(d.pass, B, m1, 0, n1, n2, d.tw1, d.lift,
                                                                          nullptr);
  dense_finish_kernel<<<dim3(nb, B), kEwThreads, 0, st>>>(s, gamma, d.lift, d.dd, mean, relc, pv_out, part);
}

}  // namespace fbme
