// FP32-accurate GEMM on the 5th-generation tensor cores (sm_100a tcgen05)
// for the per-type fitting networks, with the layer's elementwise math fused
// into the epilogue.
//
//   C[m, n] = sum_k A[m, k] B[n, k]      A: [M, K] FP32 row-major (activations)
//                                        B: [N, K] FP32 row-major (weights),
//                                           given pre-split into TF32 hi / lo,
//                                           or in FP32 and split in the kernel
// 3xTF32: A = Ah + Al and B = Bh + Bl with Ah, Bh the TF32 roundings; the
// product is Ah Bh + Al Bh + Ah Bl (the Al Bl term, ~2^-22 relative, is
// dropped), accumulated in FP32 in tensor memory.
//
// Persistent, warp-specialised CTA (one per SM) walking output tiles of 128
// rows x BN columns (the widest of 240 (K <= 512), 160, 80 that divides N and the
// fit_n_tile knob allows):
//   warp 0      TMA producer: A tile 128 x 32 and B hi/lo tiles BN x 32 per
//               k-block into a STAGES-deep shared-memory ring (128-byte
//               swizzle);
//   warps 2-5   split each A tile row by row (one row per thread) into TF32
//               hi / lo and store both straight into one of ASLOTS tensor-
//               memory slots, so the MMAs read A from TMEM and only B from
//               shared memory;
//   warps 6-9   with FP32 weights, split each B tile into TF32 hi / lo in
//               shared memory (half the weight bytes from L2), else idle;
//   warp 1      one elected lane issues tcgen05.mma (M=128, N=BN, K=8) into
//               one of ACCBUF TMEM accumulators and commits to the ring's,
//               the A slots' and the accumulator's mbarriers;
//   warps 10..  EPIW epilogue warps (two per TMEM lane quadrant when EPIW = 8,
//               splitting the columns): one row per thread, 16-byte loads /
//               stores; with two accumulators the epilogue of one tile
//               overlaps the next tile's MMAs.
// Tensor memory (512 columns): accumulators from column 0, A slot s hi / lo at
// A0 + 64 s and A0 + 64 s + 32. Every mbarrier wait is bounded: on time-out
// the CTA raises an error bit in the caller's status word, stops issuing
// work, waits (bounded) for its copies and MMAs in flight and frees its
// tensor memory before returning.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>

#include "dpb_common.cuh"

namespace dpb {

constexpr int GT_BM = 128;
constexpr int GT_BK = 32;  // 32 FP32 = one 128-byte swizzle row
constexpr int GT_MAXT = 4;
constexpr unsigned GT_WAIT_LIMIT = 1u << 24;
constexpr uint32_t TM_COLS = 512;

// one kernel configuration: tile width, ring depth, TMEM A slots,
// accumulator buffers and epilogue warps
template <int BN_, int STAGES_, int ASLOTS_, int ACCBUF_, int EPIW_>
struct GemmCfg {
  static constexpr int BN = BN_, STAGES = STAGES_, ASLOTS = ASLOTS_, ACCBUF = ACCBUF_,
                       EPIW = EPIW_;
  static constexpr int THREADS = 64 + 128 + 128 + 32 * EPIW;
  static constexpr uint32_t ACC_STRIDE = BN <= 128 ? 128u : (uint32_t)((BN + 31) / 32 * 32);
  static constexpr uint32_t A0 = ACCBUF * ACC_STRIDE;
  static constexpr int A_BYTES = GT_BM * GT_BK * 4;  // 16 KB
  static constexpr int B_BYTES = BN * GT_BK * 4;
  static constexpr int STAGE_BYTES = A_BYTES + 2 * B_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024;
  static_assert(BN % 16 == 0 && BN <= 256, "MMA N");
  static_assert(A0 + 64u * ASLOTS <= TM_COLS, "tensor memory columns");
  static_assert(STAGE_BYTES % 1024 == 0, "stage alignment for the 128-byte swizzle");
  static_assert(SMEM <= 232448, "shared memory per CTA");
  static_assert(EPIW == 4 || EPIW == 8, "epilogue warps");
};
// Measured on the fitting layers of 12,288-atom water: 80-column tiles are
// fastest for N = 240 (288 tiles keep every SM busy; a single 240-column tile
// per row block leaves 52 SMs idle), 160-column tiles for N = 1600 (half the
// A re-reads).
using CfgN80 = GemmCfg<80, 4, 4, 2, 4>;
using CfgN160 = GemmCfg<160, 4, 2, 2, 8>;
// one 240-column tile per 128 rows (one accumulator, two stages): for the
// short-K 240 x 240 layers, one wave instead of two over the row tiles
using CfgN240 = GemmCfg<240, 2, 4, 1, 8>;

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
  int n_tiles;  // column tiles per row tile
  int N, K;
  int split_b;  // 1: B given in FP32 and split into hi / lo in shared memory
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

// D (TMEM) += A (TMEM, lanes = rows, one TF32 per column) x B (shared memory)
__device__ __forceinline__ void mma_tf32_ta(uint32_t tmem_d, uint32_t tmem_a, uint64_t b,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      ::"r"(tmem_d), "r"(tmem_a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
      "r"(0u), "r"(0u));
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

// 16 consecutive columns of this warp's 32 lanes, one row per thread
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}

__device__ __forceinline__ float tf32_hi(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// tile t -> (type, first row, end of the type's rows, first column)
struct TileCoord {
  int ty, row0, row_end, n0;
};
__device__ __forceinline__ TileCoord tile_coord(const GemmShape& shp, int t, int BN) {
  TileCoord c;
  const int nt = t % shp.n_tiles, rt = t / shp.n_tiles;
  int ty = 0;
  while (ty + 1 < shp.ntypes && rt >= shp.tile_start[ty + 1]) ++ty;
  c.ty = ty;
  c.row0 = shp.row_start[ty] + (rt - shp.tile_start[ty]) * GT_BM;
  c.row_end = shp.row_start[ty + 1];
  c.n0 = nt * BN;
  return c;
}

template <class CFG, int MODE>
__global__ void __launch_bounds__(CFG::THREADS, 1)
k_gemm_tf32x3(const __grid_constant__ GemmMaps maps, GemmShape shp, GemmEpi epi, int* status) {
  constexpr int BN = CFG::BN;
  constexpr int STAGES = CFG::STAGES;
  constexpr int ASLOTS = CFG::ASLOTS;
  constexpr int ACCBUF = CFG::ACCBUF;
  constexpr int EPIW = CFG::EPIW;
  constexpr uint32_t TM_ACC = CFG::ACC_STRIDE;
  constexpr uint32_t TM_A0 = CFG::A0;
  constexpr int A_BYTES = CFG::A_BYTES;
  constexpr int B_BYTES = CFG::B_BYTES;
  constexpr int STAGE_BYTES = CFG::STAGE_BYTES;
  constexpr uint32_t IDESC = (1u << 4)            // D: FP32
                             | (2u << 7)          // A: TF32
                             | (2u << 10)         // B: TF32
                             | ((uint32_t)(BN >> 3) << 17)  // N
                             | ((uint32_t)(GT_BM >> 4) << 24);  // M = 128
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t full_bar[STAGES], conv_bar[STAGES], empty_bar[STAGES];
  __shared__ __align__(8) uint64_t afree_bar[ASLOTS];
  __shared__ __align__(8) uint64_t tfull_bar[ACCBUF], tempty_bar[ACCBUF], drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_total = shp.tile_start[shp.ntypes] * shp.n_tiles;
  const int nk = (shp.K + GT_BK - 1) / GT_BK;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&conv_bar[s], shp.split_b ? 256 : 128);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < ASLOTS; ++a) mbar_init(&afree_bar[a], 1);
    for (int b = 0; b < ACCBUF; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 32 * EPIW);
    }
    mbar_init(&drain_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&tmem_slot)),
                 "r"(TM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  volatile int* abort = &abort_flag;
  // barriers and tensor memory are set up: wait for the previous kernel of
  // the stream before the first global access
  pdl_wait();
  pdl_trigger();

  if (warp == 0) {
    // ---------------------------------------------------------------- TMA
    if (lane == 0) {
      int g = 0;  // k-blocks issued over all tiles
      bool ok = true;
      for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x) {
        const TileCoord tc = tile_coord(shp, t, BN);
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % STAGES;
          const uint32_t ph = (g / STAGES) & 1;
          if (!mbar_wait(&empty_bar[s], ph ^ 1, abort)) {
            ok = false;
            break;
          }
          unsigned char* st = smem + s * STAGE_BYTES;
          mbar_expect_tx(&full_bar[s], A_BYTES + (shp.split_b ? 1 : 2) * B_BYTES);
          tma_load_2d(st, &maps.a, &full_bar[s], kb * GT_BK, tc.row0);
          tma_load_2d(st + A_BYTES, &maps.bh[tc.ty], &full_bar[s], kb * GT_BK, tc.n0);
          if (!shp.split_b)
            tma_load_2d(st + A_BYTES + B_BYTES, &maps.bl[tc.ty], &full_bar[s], kb * GT_BK,
                        tc.n0);
        }
      }
      if (!ok) {
        // let the copies already in flight land before the CTA's shared
        // memory is released (bounded, like every other wait here)
        for (int q = g - STAGES < 0 ? 0 : g - STAGES; q < g; ++q) {
          const int s = q % STAGES;
          for (unsigned it = 0; it < GT_WAIT_LIMIT; ++it)
            if (mbar_try(&full_bar[s], (q / STAGES) & 1)) break;
        }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      int g = 0, lt = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x, ++lt) {
        const int b = lt % ACCBUF;
        if (!mbar_wait(&tempty_bar[b], ((lt / ACCBUF) & 1) ^ 1, abort)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)b * TM_ACC;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % STAGES;
          const uint32_t ph = (g / STAGES) & 1;
          if (!mbar_wait(&conv_bar[s], ph, abort)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char* st = smem + s * STAGE_BYTES;
          const int as = g % ASLOTS;
          const uint32_t ah = tmem + TM_A0 + 64u * (uint32_t)as, al = ah + 32u;
          const uint64_t bh = smem_desc(st + A_BYTES);
          const uint64_t bl = smem_desc(st + A_BYTES + B_BYTES);
#pragma unroll
          for (int j = 0; j < GT_BK / 8; ++j) {  // K = 8 per instruction
            const uint32_t ca = 8u * (uint32_t)j;           // TMEM columns
            const uint64_t ob = (uint64_t)(j * 32) >> 4;    // +32 B in the swizzled row
            const uint32_t acc = (kb > 0 || j > 0) ? 1u : 0u;
            mma_tf32_ta(d, ah + ca, bh + ob, IDESC, acc);
            mma_tf32_ta(d, al + ca, bh + ob, IDESC, 1u);
            mma_tf32_ta(d, ah + ca, bl + ob, IDESC, 1u);
          }
          mma_commit(&empty_bar[s]);    // frees the shared-memory stage once read
          mma_commit(&afree_bar[as]);   // and the TMEM A slot
        }
        if (!ok) break;
        mma_commit(&tfull_bar[b]);  // accumulator b complete
      }
      if (!ok) *abort = 1;
      // every MMA issued by this thread has completed before teardown
      mma_commit(&drain_bar);
      for (unsigned it = 0; it < GT_WAIT_LIMIT; ++it)
        if (mbar_try(&drain_bar, 0)) break;
    }
    __syncwarp();
  } else if (warp < 6) {
    // ------------------------------------------- split A into TMEM hi / lo
    const uint32_t lane_base = 32u * (uint32_t)(warp & 3);
    const int r = (int)lane_base + lane;  // tile row of this thread
    int g = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x) {
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1;
        const int as = g % ASLOTS;
        // the stage has landed and the TMEM slot's previous MMAs are done
        const bool got = mbar_wait(&full_bar[s], ph, abort) &&
                         mbar_wait(&afree_bar[as], ((g / ASLOTS) & 1) ^ 1, abort);
        if (!__all_sync(0xffffffffu, got)) {  // tcgen05.st below is warp-wide
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // row r of the 128-byte-swizzled tile: 16-byte chunk c at c ^ (r & 7)
        const unsigned char* rowp = smem + s * STAGE_BYTES + r * 128;
        uint32_t hi[32], lo[32];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float4 x = *reinterpret_cast<const float4*>(rowp + ((c ^ (r & 7)) << 4));
          const float xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float h = tf32_hi(xs[u]);
            hi[4 * c + u] = __float_as_uint(h);
            lo[4 * c + u] = __float_as_uint(xs[u] - h);
          }
        }
        const uint32_t ta = tmem + (lane_base << 16) + TM_A0 + 64u * (uint32_t)as;
        tmem_st16(ta, hi);
        tmem_st16(ta + 16u, hi + 16);
        tmem_st16(ta + 32u, lo);
        tmem_st16(ta + 48u, lo + 16);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(&conv_bar[s]);
      }
    }
  } else if (warp < 10) {
    // ------------------------------------- split FP32 B tiles into hi / lo
    // (only with FP32 weights): TF32 hi in place, lo into the lo buffer at the
    // same swizzled offset; rows r and r + 128 of the BN-row tile
    if (shp.split_b) {
      const int r = 32 * (warp - 6) + lane;
      int g = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x) {
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % STAGES;
          const uint32_t ph = (g / STAGES) & 1;
          if (!mbar_wait(&full_bar[s], ph, abort)) {
            ok = false;
            break;
          }
          unsigned char* bh = smem + s * STAGE_BYTES + A_BYTES;
          unsigned char* bl = bh + B_BYTES;
#pragma unroll
          for (int rr = 0; rr < (BN + 127) / 128; ++rr) {
            const int n = r + 128 * rr;
            if (n < BN) {
#pragma unroll
              for (int c = 0; c < 8; ++c) {
                const int off = n * 128 + ((c ^ (n & 7)) << 4);
                const float4 x = *reinterpret_cast<const float4*>(bh + off);
                const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z),
                                             tf32_hi(x.w));
                *reinterpret_cast<float4*>(bh + off) = h;
                *reinterpret_cast<float4*>(bl + off) =
                    make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
              }
            }
          }
          // generic-proxy writes, read next by the tensor cores (async proxy)
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(&conv_bar[s]);
        }
      }
    }
  } else {
    // ---------------------------------------------------------------- epilogue
    // warp (warp % 4) owns TMEM lanes 32 * (warp % 4) ..., one row per
    // thread; each 16-column chunk moves as 4 x 16-byte loads / stores per
    // operand (64 contiguous bytes per thread and row)
    const int lane_base = 32 * (warp & 3);
    const int ehalf = EPIW == 8 ? (warp - 10) >> 2 : 0;  // column share of this warp
    int lt = 0;
    for (int t = blockIdx.x; t < n_total; t += gridDim.x, ++lt) {
      const int b = lt % ACCBUF;
      bool have = mbar_wait(&tfull_bar[b], (lt / ACCBUF) & 1, abort) && !*abort;
      have = __shfl_sync(0xffffffffu, have ? 1 : 0, 0) != 0;  // tcgen05.ld is warp-wide
      if (!have) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const TileCoord tc = tile_coord(shp, t, BN);
      const int row = tc.row0 + lane_base + lane;
      const bool ok = row < tc.row_end;
      const int n0 = tc.n0;
      const size_t at = (size_t)(ok ? row : tc.row0) * epi.ld + n0;
      const float* bias = epi.bias[tc.ty];
      const float* idt = epi.idt[tc.ty];
      const float* wv = epi.w[tc.ty];
      constexpr bool NEED0 = MODE >= EPI_RES_DT, NEED1 = MODE == EPI_BWD_RES;
      const uint32_t acc_base = tmem + ((uint32_t)lane_base << 16) + (uint32_t)b * TM_ACC;
      float esum = 0.f;
#pragma unroll 1
      for (int c0 = 16 * ehalf; c0 < BN; c0 += 16 * (EPIW / 4)) {
        float4 x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // in flight during the TMEM load
          x0[j] = x1[j] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (NEED0 && ok) x0[j] = __ldg(reinterpret_cast<const float4*>(epi.aux0 + at + c0) + j);
          if (NEED1 && ok) x1[j] = __ldg(reinterpret_cast<const float4*>(epi.aux1 + at + c0) + j);
        }
        float v[16];
        tmem_ld16(acc_base + (uint32_t)c0, v);
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
      // accumulator b may be overwritten by the tile after next
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&tempty_bar[b]);
      if (MODE == EPI_LAST && ok) atomicAdd(&epi.e[row], esum);  // per warp's columns
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_MMA_TIMEOUT);
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TM_COLS));
  }
}

// ---------------------------------------------------------------- host -----
template <class CFG, int MODE>
static int launch_mode(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi,
                       int* status, cudaStream_t st) {
  DPB_CUDA(cudaFuncSetAttribute(k_gemm_tf32x3<CFG, MODE>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, CFG::SMEM),
           "gemm");
  const int tiles = shp.tile_start[shp.ntypes] * shp.n_tiles;
  if (tiles == 0) return DPB_OK;
  const int sms = sm_count();
  const int grid = tiles < sms ? tiles : sms;
  DPB_CUDA(launch_pdl(k_gemm_tf32x3<CFG, MODE>, dim3(grid), dim3(CFG::THREADS),
                      (size_t)CFG::SMEM, st, maps, shp, epi, status),
           "gemm_tf32x3");
  return DPB_OK;
}

template <class CFG>
static int launch(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi, int* status,
                  cudaStream_t st) {
  switch (epi.mode) {
    case EPI_STORE: return launch_mode<CFG, EPI_STORE>(maps, shp, epi, status, st);
    case EPI_TANH: return launch_mode<CFG, EPI_TANH>(maps, shp, epi, status, st);
    case EPI_RES_DT: return launch_mode<CFG, EPI_RES_DT>(maps, shp, epi, status, st);
    case EPI_LAST: return launch_mode<CFG, EPI_LAST>(maps, shp, epi, status, st);
    case EPI_BWD_DT: return launch_mode<CFG, EPI_BWD_DT>(maps, shp, epi, status, st);
    default: return launch_mode<CFG, EPI_BWD_RES>(maps, shp, epi, status, st);
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

// Total energy of the fitting rows: energy[0] = e_const + sum_r e[r] in FP64,
// then e[r] = 0, so the next step's output-layer epilogue can accumulate into
// it again. Block b sums the fixed row range [b * chunk, (b + 1) * chunk) into
// part[b]; the last block to finish (ticket) adds the partials in block order,
// so the bits do not depend on scheduling, and resets the ticket.
constexpr int ES_MAXB = 148;
constexpr int ES_ROWS = 1024;  // rows per block at least

__global__ void __launch_bounds__(512) k_energy_sum(double* energy, float* e, int n,
                                                    double e_const, double* part,
                                                    unsigned* ticket) {
  __shared__ double s_w[16];
  __shared__ int s_last;
  pdl_wait();
  pdl_trigger();
  const int chunk = (n + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
  double acc = 0.;
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    acc += (double)e[r];
    e[r] = 0.f;
  }
  acc = warp_sum(acc);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s_w[w] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += s_w[k];
    part[blockIdx.x] = v;
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    double t = e_const;
    for (int k = 0; k < (int)gridDim.x; ++k) t += __ldcg(part + k);
    energy[0] = t;
    *ticket = 0u;
  }
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
  // widest tile allowed by the fit_n_tile knob that divides N (240 only for
  // K <= 512, where two pipeline stages keep the tensor cores fed)
  const int knob = tune_value("fit_n_tile", CfgN160::BN);
  const int BN = (knob >= CfgN240::BN && N % CfgN240::BN == 0 && K <= 512) ? CfgN240::BN
                 : (knob >= CfgN160::BN && N % CfgN160::BN == 0)            ? CfgN160::BN
                                                                            : CfgN80::BN;
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
  // b_lo == NULL: b_hi holds the FP32 weights, split in the kernel
  shp.split_b = b_lo == nullptr ? 1 : 0;
  for (int t = 0; t < ntypes; ++t) {
    if ((rc = make_map(&maps.bh[t], b_hi[t], N, K, BN))) return rc;
    if ((rc = make_map(&maps.bl[t], shp.split_b ? b_hi[t] : b_lo[t], N, K, BN))) return rc;
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
  if (BN == CfgN240::BN) return launch<CfgN240>(maps, shp, ep, status, st);
  if (BN == CfgN160::BN) return launch<CfgN160>(maps, shp, ep, status, st);
  return launch<CfgN80>(maps, shp, ep, status, st);
}

long long dpb_fit_energy_sum_work_bytes(void) {
  return (long long)sizeof(double) * (ES_MAXB + 2);
}

int dpb_fit_energy_sum_f32(double* energy, float* e, int n, double e_const, void* work,
                           dpb_stream_t stream) {
  if (n < 0 || energy == nullptr || work == nullptr || (n > 0 && e == nullptr)) {
    set_error("fit_energy_sum: invalid arguments (n=%d; energy and work required)", n);
    return DPB_ERR_INVALID;
  }
  const int blocks = std::max(1, std::min(ES_MAXB, ceil_div(n, ES_ROWS)));
  double* part = static_cast<double*>(work);
  unsigned* ticket = reinterpret_cast<unsigned*>(part + ES_MAXB);
  DPB_CUDA(launch_pdl(k_energy_sum, dim3(blocks), dim3(512), 0, as_stream(stream), energy, e,
                      n, e_const, part, ticket),
           "fit_energy_sum");
  return DPB_OK;
}

}  // extern "C"
