// FP64 GEMM for the fitting network of the FP64 plain path (and the FP64
// training step): C[M, N] = op(A) op(B) (+ bias[N]) (+ C), row-major, with
// op(X) = X or X^T. The fitting layers are y = x W + b (forward, W [in, out]
// as stored), g_in = g W^T (input gradient) and gW += x^T g (weight
// gradient), the layer algebra of deepmd/dpmodel/utils/network.py:282-330.
//
// Kernel: one CTA of 256 threads per 64 x 64 tile of C, K in steps of 16.
// The A and B tiles are staged in shared memory k-major (each thread reads
// its 4 rows / 4 columns as two 16-byte loads per k), the next k-step's tile
// is fetched into registers while the current one is multiplied, and every
// thread accumulates a 4 x 4 block of C with FP64 FMAs (B200 has no tensor
// path for FP64 faster than its FMA pipe). Edges are zero-filled, so any M,
// N, K are accepted.
#include "dpb_common.cuh"

namespace dpb {
namespace {

constexpr int GB_M = 64, GB_N = 64, GB_K = 16, GB_T = 256;

// element (r, c) of op(X) for an [rows, cols] operand with leading dim ld
template <bool TRANS>
__device__ __forceinline__ double ld_op(const double* __restrict__ X, int r, int c, int rows,
                                        int cols, int ld) {
  if (r >= rows || c >= cols) return 0.0;
  return TRANS ? X[(size_t)c * ld + r] : X[(size_t)r * ld + c];
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(GB_T)
k_gemm_f64(double* __restrict__ C, const double* __restrict__ A, const double* __restrict__ B,
           const double* __restrict__ bias, int M, int N, int K, int lda, int ldb, int ldc,
           int accumulate) {
  __shared__ __align__(16) double As[2][GB_K][GB_M + 2];
  __shared__ __align__(16) double Bs[2][GB_K][GB_N + 2];
  pdl_wait();
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
  const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 threads, 4 x 4 outputs each
  // staging assignment: 64 x 16 = 1024 elements per operand, 4 per thread.
  // A (op(A) is M x K): element q = tid + 256 j -> (row, k); for a plain A
  // consecutive threads walk k (contiguous in memory), for A^T they walk m.
  double ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int q = tid + GB_T * j;
      int r, k;
      if (TA) { r = q & 63; k = q >> 6; } else { k = q & 15; r = q >> 4; }
      ra[j] = TA ? ld_op<true>(A, m0 + r, k0 + k, M, K, lda)
                 : ld_op<false>(A, m0 + r, k0 + k, M, K, lda);
      int c, kk;
      if (TB) { kk = q & 15; c = q >> 4; } else { c = q & 63; kk = q >> 6; }
      rb[j] = TB ? ld_op<true>(B, k0 + kk, n0 + c, K, N, ldb)
                 : ld_op<false>(B, k0 + kk, n0 + c, K, N, ldb);
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int q = tid + GB_T * j;
      int r, k;
      if (TA) { r = q & 63; k = q >> 6; } else { k = q & 15; r = q >> 4; }
      As[buf][k][r] = ra[j];
      int c, kk;
      if (TB) { kk = q & 15; c = q >> 4; } else { c = q & 63; kk = q >> 6; }
      Bs[buf][kk][c] = rb[j];
    }
  };
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  const int nk = (K + GB_K - 1) / GB_K;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) fetch((t + 1) * GB_K);
#pragma unroll
    for (int k = 0; k < GB_K; ++k) {
      const double2 a01 = *reinterpret_cast<const double2*>(&As[buf][k][ty * 4]);
      const double2 a23 = *reinterpret_cast<const double2*>(&As[buf][k][ty * 4 + 2]);
      const double2 b01 = *reinterpret_cast<const double2*>(&Bs[buf][k][tx * 4]);
      const double2 b23 = *reinterpret_cast<const double2*>(&Bs[buf][k][tx * 4 + 2]);
      const double a[4] = {a01.x, a01.y, a23.x, a23.y};
      const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (t + 1 < nk) {
      stash(buf ^ 1);
      __syncthreads();
    }
  }
  pdl_trigger();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = m0 + ty * 4 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = n0 + tx * 4 + j;
      if (c >= N) continue;
      double v = acc[i][j];
      if (bias) v += bias[c];
      double* p = C + (size_t)r * ldc + c;
      if (accumulate) v += *p;
      *p = v;
    }
  }
}

}  // namespace
}  // namespace dpb

using namespace dpb;

extern "C" int dpb_gemm_f64(double* C, const double* A, const double* B, const double* bias,
                            int M, int N, int K, int lda, int ldb, int ldc, int trans_a,
                            int trans_b, int accumulate, dpb_stream_t stream) {
  if (M < 0 || N < 0 || K < 0 || (M > 0 && N > 0 && (!C || (K > 0 && (!A || !B))))) {
    set_error("gemm_f64: invalid arguments (M=%d N=%d K=%d)", M, N, K);
    return DPB_ERR_INVALID;
  }
  const int a_cols = trans_a ? M : K, b_cols = trans_b ? K : N;
  if (ldc < N || lda < a_cols || ldb < b_cols) {
    set_error("gemm_f64: leading dimensions too small (lda=%d ldb=%d ldc=%d)", lda, ldb, ldc);
    return DPB_ERR_INVALID;
  }
  if (M == 0 || N == 0) return DPB_OK;
  const dim3 grid((N + GB_N - 1) / GB_N, (M + GB_M - 1) / GB_M);
  if (grid.y > 65535) {
    set_error("gemm_f64: M=%d needs more than 65535 row tiles", M);
    return DPB_ERR_INVALID;
  }
  cudaStream_t st = as_stream(stream);
  const int ta = trans_a != 0, tb = trans_b != 0;
  if (!ta && !tb)
    launch_pdl(k_gemm_f64<false, false>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K, lda,
               ldb, ldc, accumulate);
  else if (!ta && tb)
    launch_pdl(k_gemm_f64<false, true>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K, lda,
               ldb, ldc, accumulate);
  else if (ta && !tb)
    launch_pdl(k_gemm_f64<true, false>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K, lda,
               ldb, ldc, accumulate);
  else
    launch_pdl(k_gemm_f64<true, true>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K, lda,
               ldb, ldc, accumulate);
  DPB_CHECK_LAUNCH("gemm_f64");
  return DPB_OK;
}
