// FP64 GEMM for the fitting network of the FP64 plain path (and the FP64
// training step), and its FP32 instance for the shapes the tensor-core GEMM
// does not take (N not a multiple of 80): C[M, N] = op(A) op(B) (+ bias[N])
// (+ C), row-major, with
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
template <bool TRANS, typename T>
__device__ __forceinline__ T ld_op(const T* __restrict__ X, int r, int c, int rows, int cols,
                                   int ld) {
  if (r >= rows || c >= cols) return (T)0;
  return TRANS ? X[(size_t)c * ld + r] : X[(size_t)r * ld + c];
}

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

template <bool TA, bool TB, typename T>
__global__ void __launch_bounds__(GB_T)
k_gemm_f64(T* __restrict__ C, const T* __restrict__ A, const T* __restrict__ B,
           const T* __restrict__ bias, int M, int N, int K, int lda, int ldb, int ldc,
           int accumulate) {
  using T2 = typename Vec2<T>::type;
  __shared__ __align__(16) T As[2][GB_K][GB_M + 2];
  __shared__ __align__(16) T Bs[2][GB_K][GB_N + 2];
  pdl_wait();
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
  const int tx = tid & 15, ty = tid >> 4;  // 16 x 16 threads, 4 x 4 outputs each
  // staging assignment: 64 x 16 = 1024 elements per operand, 4 per thread.
  // A (op(A) is M x K): element q = tid + 256 j -> (row, k); for a plain A
  // consecutive threads walk k (contiguous in memory), for A^T they walk m.
  T ra[4], rb[4];
  auto fetch = [&](int k0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int q = tid + GB_T * j;
      int r, k;
      if (TA) { r = q & 63; k = q >> 6; } else { k = q & 15; r = q >> 4; }
      ra[j] = TA ? ld_op<true, T>(A, m0 + r, k0 + k, M, K, lda)
                 : ld_op<false, T>(A, m0 + r, k0 + k, M, K, lda);
      int c, kk;
      if (TB) { kk = q & 15; c = q >> 4; } else { c = q & 63; kk = q >> 6; }
      rb[j] = TB ? ld_op<true, T>(B, k0 + kk, n0 + c, K, N, ldb)
                 : ld_op<false, T>(B, k0 + kk, n0 + c, K, N, ldb);
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
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = (T)0;
  const int nk = (K + GB_K - 1) / GB_K;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) fetch((t + 1) * GB_K);
#pragma unroll
    for (int k = 0; k < GB_K; ++k) {
      const T2 a01 = *reinterpret_cast<const T2*>(&As[buf][k][ty * 4]);
      const T2 a23 = *reinterpret_cast<const T2*>(&As[buf][k][ty * 4 + 2]);
      const T2 b01 = *reinterpret_cast<const T2*>(&Bs[buf][k][tx * 4]);
      const T2 b23 = *reinterpret_cast<const T2*>(&Bs[buf][k][tx * 4 + 2]);
      const T a[4] = {a01.x, a01.y, a23.x, a23.y};
      const T b[4] = {b01.x, b01.y, b23.x, b23.y};
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
      T v = acc[i][j];
      if (bias) v += bias[c];
      T* p = C + (size_t)r * ldc + c;
      if (accumulate) v += *p;
      *p = v;
    }
  }
}

// The large-M form: 128 x 64 tiles, K in steps of 8, each thread a block of
// 8 rows (ty * 4 + i and 64 + ty * 4 + i) by 4 columns, so every k step
// reads 6 shared-memory vectors for 32 FMAs (the 64 x 64 form above: 4 for
// 16).
constexpr int GL_M = 128, GL_N = 64, GL_K = 8;

template <bool TA, bool TB, typename T>
__global__ void __launch_bounds__(GB_T)
k_gemm_big(T* __restrict__ C, const T* __restrict__ A, const T* __restrict__ B,
           const T* __restrict__ bias, int M, int N, int K, int lda, int ldb, int ldc,
           int accumulate) {
  using T2 = typename Vec2<T>::type;
  __shared__ __align__(16) T As[2][GL_K][GL_M + 2];
  __shared__ __align__(16) T Bs[2][GL_K][GL_N + 2];
  pdl_wait();
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * GL_M, n0 = blockIdx.x * GL_N;
  const int tx = tid & 15, ty = tid >> 4;
  T ra[4], rb[2];
  auto a_at = [&](int q, int& r, int& k) {
    if (TA) { r = q & 127; k = q >> 7; } else { k = q & 7; r = q >> 3; }
  };
  auto b_at = [&](int q, int& c, int& k) {
    if (TB) { k = q & 7; c = q >> 3; } else { c = q & 63; k = q >> 6; }
  };
  auto fetch = [&](int k0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int r, k;
      a_at(tid + GB_T * j, r, k);
      ra[j] = ld_op<TA, T>(A, m0 + r, k0 + k, M, K, lda);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int c, k;
      b_at(tid + GB_T * j, c, k);
      rb[j] = ld_op<TB, T>(B, k0 + k, n0 + c, K, N, ldb);
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int r, k;
      a_at(tid + GB_T * j, r, k);
      As[buf][k][r] = ra[j];
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int c, k;
      b_at(tid + GB_T * j, c, k);
      Bs[buf][k][c] = rb[j];
    }
  };
  T acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = (T)0;
  const int nk = (K + GL_K - 1) / GL_K;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int buf = t & 1;
    if (t + 1 < nk) fetch((t + 1) * GL_K);
#pragma unroll
    for (int k = 0; k < GL_K; ++k) {
      const T2 a0 = *reinterpret_cast<const T2*>(&As[buf][k][ty * 4]);
      const T2 a1 = *reinterpret_cast<const T2*>(&As[buf][k][ty * 4 + 2]);
      const T2 a2 = *reinterpret_cast<const T2*>(&As[buf][k][64 + ty * 4]);
      const T2 a3 = *reinterpret_cast<const T2*>(&As[buf][k][64 + ty * 4 + 2]);
      const T2 b0 = *reinterpret_cast<const T2*>(&Bs[buf][k][tx * 4]);
      const T2 b1 = *reinterpret_cast<const T2*>(&Bs[buf][k][tx * 4 + 2]);
      const T a[8] = {a0.x, a0.y, a1.x, a1.y, a2.x, a2.y, a3.x, a3.y};
      const T b[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int i = 0; i < 8; ++i)
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
  for (int i = 0; i < 8; ++i) {
    const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = n0 + tx * 4 + j;
      if (c >= N) continue;
      T v = acc[i][j];
      if (bias) v += bias[c];
      T* p = C + (size_t)r * ldc + c;
      if (accumulate) v += *p;
      *p = v;
    }
  }
}

}  // namespace
}  // namespace dpb

using namespace dpb;

template <typename T>
static int gemm(const char* what, T* C, const T* A, const T* B, const T* bias, int M, int N,
                int K, int lda, int ldb, int ldc, int trans_a, int trans_b, int accumulate,
                dpb_stream_t stream) {
  if (M < 0 || N < 0 || K < 0 || (M > 0 && N > 0 && (!C || (K > 0 && (!A || !B))))) {
    set_error("%s: invalid arguments (M=%d N=%d K=%d)", what, M, N, K);
    return DPB_ERR_INVALID;
  }
  const int a_cols = trans_a ? M : K, b_cols = trans_b ? K : N;
  if (ldc < N || lda < a_cols || ldb < b_cols) {
    set_error("%s: leading dimensions too small (lda=%d ldb=%d ldc=%d)", what, lda, ldb, ldc);
    return DPB_ERR_INVALID;
  }
  if (M == 0 || N == 0) return DPB_OK;
  cudaStream_t st = as_stream(stream);
  const int ta = trans_a != 0, tb = trans_b != 0;
  if (M >= GL_M && tune_value("gemm_simt_big", 1)) {
    const dim3 grid((N + GL_N - 1) / GL_N, (M + GL_M - 1) / GL_M);
    if (grid.y > 65535) {
      set_error("%s: M=%d needs more than 65535 row tiles", what, M);
      return DPB_ERR_INVALID;
    }
    if (!ta && !tb)
      launch_pdl(k_gemm_big<false, false, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
                 lda, ldb, ldc, accumulate);
    else if (!ta && tb)
      launch_pdl(k_gemm_big<false, true, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
                 lda, ldb, ldc, accumulate);
    else if (ta && !tb)
      launch_pdl(k_gemm_big<true, false, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
                 lda, ldb, ldc, accumulate);
    else
      launch_pdl(k_gemm_big<true, true, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
                 lda, ldb, ldc, accumulate);
    DPB_CHECK_LAUNCH(what);
    return DPB_OK;
  }
  const dim3 grid((N + GB_N - 1) / GB_N, (M + GB_M - 1) / GB_M);
  if (grid.y > 65535) {
    set_error("%s: M=%d needs more than 65535 row tiles", what, M);
    return DPB_ERR_INVALID;
  }
  if (!ta && !tb)
    launch_pdl(k_gemm_f64<false, false, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
               lda, ldb, ldc, accumulate);
  else if (!ta && tb)
    launch_pdl(k_gemm_f64<false, true, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
               lda, ldb, ldc, accumulate);
  else if (ta && !tb)
    launch_pdl(k_gemm_f64<true, false, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
               lda, ldb, ldc, accumulate);
  else
    launch_pdl(k_gemm_f64<true, true, T>, grid, dim3(GB_T), 0, st, C, A, B, bias, M, N, K,
               lda, ldb, ldc, accumulate);
  DPB_CHECK_LAUNCH(what);
  return DPB_OK;
}

extern "C" int dpb_gemm_f64(double* C, const double* A, const double* B, const double* bias,
                            int M, int N, int K, int lda, int ldb, int ldc, int trans_a,
                            int trans_b, int accumulate, dpb_stream_t stream) {
  return gemm<double>("gemm_f64", C, A, B, bias, M, N, K, lda, ldb, ldc, trans_a, trans_b,
                      accumulate, stream);
}

extern "C" int dpb_gemm_f32(float* C, const float* A, const float* B, const float* bias, int M,
                            int N, int K, int lda, int ldb, int ldc, int trans_a, int trans_b,
                            int accumulate, dpb_stream_t stream) {
  return gemm<float>("gemm_f32", C, A, B, bias, M, N, K, lda, ldb, ldc, trans_a, trans_b,
                     accumulate, stream);
}

// out[c * ld_out + r] = in[r * ld_in + c] for r < rows, c < cols, and zero for
// rows <= r < out_rows (a K padded to a multiple of 4 for the tensor-core
// GEMM's 16-byte rows, or one block of a concatenation along K)
__global__ void k_transpose_f32(float* __restrict__ out, const float* __restrict__ in, int rows,
                                int cols, int ld_in, int ld_out, int out_rows) {
  __shared__ float tile[32][33];
  pdl_wait();
  pdl_trigger();
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ld_in + c] : 0.f;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (c < cols && r < out_rows) out[(size_t)c * ld_out + r] = tile[threadIdx.x][k];
  }
}

extern "C" int dpb_transpose_f32(float* out, const float* in, int rows, int cols, int ld_in,
                                 int ld_out, int out_rows, dpb_stream_t stream) {
  if (rows < 0 || cols < 0 || out_rows < rows || ld_out < out_rows || ld_in < cols ||
      (out_rows > 0 && cols > 0 && (!out || (rows > 0 && !in)))) {
    set_error("transpose_f32: invalid arguments (rows=%d cols=%d ld_in=%d ld_out=%d "
              "out_rows=%d)", rows, cols, ld_in, ld_out, out_rows);
    return DPB_ERR_INVALID;
  }
  if (cols == 0 || out_rows == 0) return DPB_OK;
  const dim3 grid((cols + 31) / 32, (out_rows + 31) / 32);
  DPB_CUDA(launch_pdl(k_transpose_f32, grid, dim3(32, 8), 0, as_stream(stream), out, in, rows,
                      cols, ld_in, ld_out, out_rows),
           "transpose_f32");
  return DPB_OK;
}
