// FP32-accurate GEMM on the 5th-generation tensor cores (sm_100a tcgen05)
// for the per-type fitting networks, with the layer's elementwise math fused
// into the epilogue.
//
//   C[m, n] = sum_k A[m, k] B[n, k]      A: [M, K] FP32 row-major (activations)
//                                        B: [N, K] FP32 row-major (weights),
//                                           given pre-split into TF32 hi / lo
// 3xTF32: A = Ah + Al and B = Bh + Bl with Ah, Bh the TF32 roundings; the
// product is Ah Bh + Al Bh + Ah Bl (the Al Bl term, ~2^-22 relative, is
// dropped), accumulated in FP32 in tensor memory.
//
// CTA (192 threads, one per SM): warp 0 issues the TMA loads of a 4-stage ring
// (A tile 128 x 32, B hi/lo tiles BN x 32, 128-byte swizzle); warps 2-5 split
// the A tile into hi/lo in shared memory (an elementwise operation, so the
// swizzled layout is preserved) and later run the epilogue from TMEM; one
// elected lane of warp 1 issues tcgen05.mma (M=128, N=BN, K=8) and commits to
// the ring's mbarriers. Every mbarrier wait is bounded: on time-out the CTA
// raises an error bit in the caller's status word, stops issuing work and
// frees its tensor memory before returning.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "dpb_common.cuh"

namespace dpb {

constexpr int GT_THREADS = 192;
constexpr int GT_BM = 128;
constexpr int GT_BK = 32;  // 32 FP32 = one 128-byte swizzle row
constexpr int GT_MAXT = 4;
constexpr unsigned GT_WAIT_LIMIT = 1u << 24;

enum : int {
  ST_MMA_TIMEOUT = 1 << 8,
};

enum GemmMode : int {
  EPI_STORE = 0,     // out0 = acc
  EPI_TANH = 1,      // out0 = tanh(acc + bias)
  EPI_RES_DT = 2,    // y = tanh(acc + bias); out0 = y; out1 = aux0 + idt * y
  EPI_LAST = 3,      // y = tanh(acc + bias); h = aux0 + idt * y; e += h . w;
                     // out0 = w * idt * (1 - y^2)
  EPI_BWD_DT = 4,    // g = w + acc; out1 = g; out0 = g * idt * (1 - aux0^2)
  EPI_BWD_RES = 5,   // g = aux1 + acc; out0 = g * (1 - aux0^2)
};

struct GemmEpi {
  int mode;
  float* out0;
  float* out1;
  const float* aux0;
  const float* aux1;
  int ld;  // leading dimension of out0/out1/aux0/aux1 (= N)
  const float* bias[GT_MAXT];
  const float* idt[GT_MAXT];
  const float* w[GT_MAXT];
  float* e;
};

struct GemmShape {
  int ntypes;
  int row_start[GT_MAXT + 1];
  int tile_start[GT_MAXT + 1];
  int n_tiles;
  int N, K;
};

struct GemmMaps {
  CUtensorMap a;
  CUtensorMap bh[GT_MAXT];
  CUtensorMap bl[GT_MAXT];
};

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false on time-out or when another role already aborted
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
  for (unsigned it = 0; it < GT_WAIT_LIMIT; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 1023u) == 1023u && *abort) return false;
  }
  *abort = 1;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(su32(dst)),
      "l"((uint64_t)map), "r"(su32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  // K-major, 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart
  // (SBO), leading offset unused (1), descriptor version 1, base offset 0.
  const uint64_t addr = su32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u),
      "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          su32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

template <int BN, int STAGES, int MODE>
__global__ void __launch_bounds__(GT_THREADS, STAGES <= 2 ? 2 : 1)
k_gemm_tf32x3(const __grid_constant__ GemmMaps maps, GemmShape shp, GemmEpi epi, int* status) {
  constexpr int A_BYTES = GT_BM * GT_BK * 4;  // 16 KB
  constexpr int B_BYTES = BN * GT_BK * 4;
  constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  constexpr uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  constexpr uint32_t IDESC = (1u << 4)            // D: FP32
                             | (2u << 7)          // A: TF32
                             | (2u << 10)         // B: TF32
                             | ((uint32_t)(BN >> 3) << 17)  // N
                             | ((uint32_t)(GT_BM >> 4) << 24);  // M = 128
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[STAGES], conv_bar[STAGES], empty_bar[STAGES];
  __shared__ __align__(8) uint64_t acc_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // tile of this CTA
  const int nt = blockIdx.x % shp.n_tiles, rt = blockIdx.x / shp.n_tiles;
  int ty = 0;
  while (ty + 1 < shp.ntypes && rt >= shp.tile_start[ty + 1]) ++ty;
  const int row0 = shp.row_start[ty] + (rt - shp.tile_start[ty]) * GT_BM;
  const int row_end = shp.row_start[ty + 1];
  const int n0 = nt * BN;
  const int nk = (shp.K + GT_BK - 1) / GT_BK;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&conv_bar[s], 128);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  volatile int* abort = &abort_flag;

  if (warp == 0) {
    // ---------------------------------------------------------------- TMA
    if (lane == 0) {
      int issued = 0;
      for (int kb = 0; kb < nk; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = (kb / STAGES) & 1;
        if (!mbar_wait(&empty_bar[s], ph ^ 1, abort)) break;
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_expect_tx(&full_bar[s], A_BYTES + 2 * B_BYTES);
        tma_load_2d(st, &maps.a, &full_bar[s], kb * GT_BK, row0);
        tma_load_2d(st + 2 * A_BYTES, &maps.bh[ty], &full_bar[s], kb * GT_BK, n0);
        tma_load_2d(st + 2 * A_BYTES + B_BYTES, &maps.bl[ty], &full_bar[s], kb * GT_BK, n0);
        issued = kb + 1;
      }
      if (*abort) {
        // let the copies already in flight land before the CTA's shared memory
        // is released (bounded, like every other wait here)
        for (int kb = issued - STAGES < 0 ? 0 : issued - STAGES; kb < issued; ++kb) {
          const int s = kb % STAGES;
          for (unsigned it = 0; it < GT_WAIT_LIMIT; ++it)
            if (mbar_try(&full_bar[s], (kb / STAGES) & 1)) break;
        }
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      bool ok = true;
      for (int kb = 0; kb < nk && ok; ++kb) {
        const int s = kb % STAGES;
        const uint32_t ph = (kb / STAGES) & 1;
        if (!mbar_wait(&conv_bar[s], ph, abort)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        unsigned char* st = smem + s * STAGE_BYTES;
        const uint64_t ah = smem_desc(st), al = smem_desc(st + A_BYTES);
        const uint64_t bh = smem_desc(st + 2 * A_BYTES);
        const uint64_t bl = smem_desc(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
        for (int j = 0; j < GT_BK / 8; ++j) {  // K = 8 per instruction: +32 B
          const uint64_t o = (uint64_t)(j * 32) >> 4;
          const uint32_t acc = (kb > 0 || j > 0) ? 1u : 0u;
          mma_tf32(tmem, ah + o, bh + o, IDESC, acc);
          mma_tf32(tmem, al + o, bh + o, IDESC, 1u);
          mma_tf32(tmem, ah + o, bl + o, IDESC, 1u);
        }
        mma_commit(&empty_bar[s]);  // frees the stage once these MMAs have read it
      }
      mma_commit(&acc_bar);  // accumulator complete (or all issued work drained)
      if (!ok) *abort = 1;
    }
  } else {
    // ------------------------------------------- split A, then epilogue
    const int ct = threadIdx.x - 64;  // 0..127
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (kb / STAGES) & 1;
      if (!mbar_wait(&full_bar[s], ph, abort)) break;
      float4* ah = reinterpret_cast<float4*>(smem + s * STAGE_BYTES);
      float4* al = reinterpret_cast<float4*>(smem + s * STAGE_BYTES + A_BYTES);
#pragma unroll
      for (int q = 0; q < A_BYTES / 16 / 128; ++q) {
        const int idx = q * 128 + ct;
        float4 x = ah[idx];
        float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
        ah[idx] = h;
        al[idx] = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&conv_bar[s]);
    }
    // epilogue: warp (warp % 4) owns TMEM lanes 32 * (warp % 4) ..., one row
    // per thread; each 16-column chunk moves as 4 x 16-byte loads / stores
    // per operand (64 contiguous bytes per thread and row)
    bool have = mbar_wait(&acc_bar, 0, abort) && !*abort;
    have = __shfl_sync(0xffffffffu, have ? 1 : 0, 0) != 0;  // tcgen05.ld is warp-wide
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (have) {
      const int lane_base = 32 * (warp & 3);
      const int row = row0 + lane_base + lane;
      const bool ok = row < row_end;
      const size_t at = (size_t)(ok ? row : row0) * epi.ld + n0;
      const float* bias = epi.bias[ty];
      const float* idt = epi.idt[ty];
      const float* wv = epi.w[ty];
      constexpr bool NEED0 = MODE >= EPI_RES_DT, NEED1 = MODE == EPI_BWD_RES;
      float esum = 0.f;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 16) {
        float4 x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // in flight during the TMEM load
          x0[j] = x1[j] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (NEED0 && ok) x0[j] = __ldg(reinterpret_cast<const float4*>(epi.aux0 + at + c0) + j);
          if (NEED1 && ok) x1[j] = __ldg(reinterpret_cast<const float4*>(epi.aux1 + at + c0) + j);
        }
        float v[16];
        tmem_ld16(tmem + ((uint32_t)lane_base << 16) + (uint32_t)c0, v);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cj = n0 + c0 + 4 * j;
          float4 bb = make_float4(0.f, 0.f, 0.f, 0.f), dd = bb, ww = bb;
          if (MODE == EPI_TANH || MODE == EPI_RES_DT || MODE == EPI_LAST)
            bb = __ldg(reinterpret_cast<const float4*>(bias + cj));
          if (MODE == EPI_RES_DT || MODE == EPI_LAST || MODE == EPI_BWD_DT)
            dd = __ldg(reinterpret_cast<const float4*>(idt + cj));
          if (MODE == EPI_LAST || MODE == EPI_BWD_DT)
            ww = __ldg(reinterpret_cast<const float4*>(wv + cj));
          const float a[4] = {v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]};
          const float b4[4] = {bb.x, bb.y, bb.z, bb.w}, d4[4] = {dd.x, dd.y, dd.z, dd.w};
          const float w4[4] = {ww.x, ww.y, ww.z, ww.w};
          const float p0[4] = {x0[j].x, x0[j].y, x0[j].z, x0[j].w};
          const float p1[4] = {x1[j].x, x1[j].y, x1[j].z, x1[j].w};
          float o0[4], o1[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (MODE == EPI_STORE) {
              o0[u] = a[u];
            } else if (MODE == EPI_TANH) {
              o0[u] = tanhf(a[u] + b4[u]);
            } else if (MODE == EPI_RES_DT) {
              const float y = tanhf(a[u] + b4[u]);
              o0[u] = y;
              o1[u] = p0[u] + d4[u] * y;
            } else if (MODE == EPI_LAST) {
              const float y = tanhf(a[u] + b4[u]);
              const float h = p0[u] + d4[u] * y;
              esum += h * w4[u];
              o0[u] = w4[u] * d4[u] * (1.f - y * y);
            } else if (MODE == EPI_BWD_DT) {
              const float g = w4[u] + a[u];
              o1[u] = g;
              o0[u] = g * d4[u] * (1.f - p0[u] * p0[u]);
            } else {  // EPI_BWD_RES
              const float g = p1[u] + a[u];
              o0[u] = g * (1.f - p0[u] * p0[u]);
            }
          }
          if (ok) {
            reinterpret_cast<float4*>(epi.out0 + at + c0)[j] =
                make_float4(o0[0], o0[1], o0[2], o0[3]);
            if (MODE == EPI_RES_DT || MODE == EPI_BWD_DT)
              reinterpret_cast<float4*>(epi.out1 + at + c0)[j] =
                  make_float4(o1[0], o1[1], o1[2], o1[3]);
          }
        }
      }
      if (MODE == EPI_LAST && ok) atomicAdd(&epi.e[row], esum);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_MMA_TIMEOUT);
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// ---------------------------------------------------------------- host -----
template <int BN, int STAGES, int MODE>
static int launch_mode(const struct GemmMaps& maps, const struct GemmShape& shp,
                       const struct GemmEpi& epi, int* status, cudaStream_t st);

template <int BN, int STAGES>
static int launch(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi, int* status,
                  cudaStream_t st) {
  switch (epi.mode) {
    case EPI_STORE: return launch_mode<BN, STAGES, EPI_STORE>(maps, shp, epi, status, st);
    case EPI_TANH: return launch_mode<BN, STAGES, EPI_TANH>(maps, shp, epi, status, st);
    case EPI_RES_DT: return launch_mode<BN, STAGES, EPI_RES_DT>(maps, shp, epi, status, st);
    case EPI_LAST: return launch_mode<BN, STAGES, EPI_LAST>(maps, shp, epi, status, st);
    case EPI_BWD_DT: return launch_mode<BN, STAGES, EPI_BWD_DT>(maps, shp, epi, status, st);
    default: return launch_mode<BN, STAGES, EPI_BWD_RES>(maps, shp, epi, status, st);
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static int get_encoder() {
  if (g_encode) return DPB_OK;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e =
      cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
  if (e != cudaSuccess || fn == nullptr || q != cudaDriverEntryPointSuccess) {
    set_error("gemm: cuTensorMapEncodeTiled is not available from the driver");
    return DPB_ERR_CUDA;
  }
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return DPB_OK;
}

// 2-D FP32 row-major [rows, cols] (cols contiguous), box rows x 32 cols, SW128
static int make_map(CUtensorMap* m, const float* base, int rows, int cols, int box_rows) {
  if (((uintptr_t)base & 15) != 0 || (cols * 4) % 16 != 0) {
    set_error("gemm: operand base must be 16-byte aligned and rows a multiple of 16 bytes");
    return DPB_ERR_INVALID;
  }
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 4};
  cuuint32_t box[2] = {(cuuint32_t)GT_BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("gemm: cuTensorMapEncodeTiled failed (%d)", (int)r);
    return DPB_ERR_INVALID;
  }
  return DPB_OK;
}

template <int BN, int STAGES, int MODE>
static int launch_mode(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi,
                       int* status, cudaStream_t st) {
  constexpr int SMEM = STAGES * (2 * GT_BM * GT_BK * 4 + 2 * BN * GT_BK * 4) + 1024;
  DPB_CUDA(cudaFuncSetAttribute(k_gemm_tf32x3<BN, STAGES, MODE>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM),
           "gemm");
  const int tiles = shp.tile_start[shp.ntypes] * shp.n_tiles;
  if (tiles == 0) return DPB_OK;
  k_gemm_tf32x3<BN, STAGES, MODE><<<tiles, GT_THREADS, SMEM, st>>>(maps, shp, epi, status);
  DPB_CHECK_LAUNCH("gemm_tf32x3");
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_gemm_tf32x3_f32(const float* A, int M, int K, const float* const* b_hi,
                        const float* const* b_lo, int N, const int* type_rows, int ntypes,
                        int mode, float* out0, float* out1, const float* aux0,
                        const float* aux1, const float* const* bias, const float* const* idt,
                        const float* const* w, float* e, int* status, dpb_stream_t stream) {
  if (ntypes < 1 || ntypes > GT_MAXT || M < 0 || K <= 0 || N <= 0 || mode < 0 ||
      mode > EPI_BWD_RES || status == nullptr) {
    set_error("gemm_tf32x3: invalid arguments (ntypes=%d M=%d K=%d N=%d mode=%d)", ntypes, M,
              K, N, mode);
    return DPB_ERR_INVALID;
  }
  int rc = get_encoder();
  if (rc) return rc;
  if (N % 80 != 0) {
    set_error("gemm_tf32x3: N=%d must be a multiple of 80", N);
    return DPB_ERR_INVALID;
  }
  const int BN = 80;
  GemmMaps maps;
  GemmShape shp;
  shp.ntypes = ntypes;
  shp.N = N;
  shp.K = K;
  shp.n_tiles = N / BN;
  shp.row_start[0] = 0;
  shp.tile_start[0] = 0;
  for (int t = 0; t < ntypes; ++t) {
    shp.row_start[t + 1] = shp.row_start[t] + type_rows[t];
    shp.tile_start[t + 1] = shp.tile_start[t] + (type_rows[t] + GT_BM - 1) / GT_BM;
  }
  if (shp.row_start[ntypes] != M) {
    set_error("gemm_tf32x3: type_rows must sum to M");
    return DPB_ERR_INVALID;
  }
  if (M == 0) return DPB_OK;
  rc = make_map(&maps.a, A, M, K, GT_BM);
  if (rc) return rc;
  for (int t = 0; t < ntypes; ++t) {
    if ((rc = make_map(&maps.bh[t], b_hi[t], N, K, BN))) return rc;
    if ((rc = make_map(&maps.bl[t], b_lo[t], N, K, BN))) return rc;
  }
  auto misaligned = [](const void* q) { return ((uintptr_t)q & 15) != 0; };
  bool bad = misaligned(out0) || misaligned(out1) || misaligned(aux0) || misaligned(aux1);
  for (int t = 0; t < ntypes; ++t)
    bad = bad || (bias && misaligned(bias[t])) || (idt && misaligned(idt[t])) ||
          (w && misaligned(w[t]));
  if (bad) {
    set_error("gemm_tf32x3: outputs, aux operands and per-type vectors must be 16-byte aligned");
    return DPB_ERR_INVALID;
  }
  GemmEpi ep{};
  ep.mode = mode;
  ep.out0 = out0;
  ep.out1 = out1;
  ep.aux0 = aux0;
  ep.aux1 = aux1;
  ep.ld = N;
  ep.e = e;
  for (int t = 0; t < ntypes; ++t) {
    ep.bias[t] = bias ? bias[t] : nullptr;
    ep.idt[t] = idt ? idt[t] : nullptr;
    ep.w[t] = w ? w[t] : nullptr;
  }
  cudaStream_t st = as_stream(stream);
  // short reductions: two CTAs per SM (2 stages each) so one CTA's epilogue
  // overlaps the other's main loop; long reductions: a deep 4-stage ring
  if (K <= 256) return launch<BN, 2>(maps, shp, ep, status, st);
  return launch<BN, 4>(maps, shp, ep, status, st);
}

}  // extern "C"
