// Device side of the split-TF32 tensor-core GEMM (dpb_gemm_tcgen05.cu): tile
// configurations, operand / epilogue descriptions, the tcgen05 / TMA / mbarrier
// primitives, and gemm_run, one whole GEMM pass over all output tiles by a
// persistent CTA. Used by the GEMM kernel and by the batched-frames step
// kernel, which runs the six fitting GEMMs as passes of one launch.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "dpb_common.cuh"

namespace dpb {

constexpr int GT_BM = 128;
constexpr int GT_BK = 32;  // 32 FP32 = one 128-byte swizzle row
constexpr int GT_MAXT = 4;
constexpr unsigned GT_WAIT_LIMIT = 1u << 24;
constexpr uint32_t TM_COLS = 512;

// one kernel configuration: tile width, ring depth, TMEM A slots,
// accumulator buffers and epilogue warps
// BSPLIT: with the four warps that split FP32 weights into TF32 hi / lo in
// shared memory (false: pre-split weights only, the epilogue warps follow
// the A-split warps)
template <int BN_, int STAGES_, int ASLOTS_, int ACCBUF_, int EPIW_, bool BSPLIT_ = true>
struct GemmCfg {
  static constexpr int BN = BN_, STAGES = STAGES_, ASLOTS = ASLOTS_, ACCBUF = ACCBUF_,
                       EPIW = EPIW_;
  static constexpr bool BSPLIT = BSPLIT_;
  static constexpr int EPI0 = BSPLIT ? 10 : 6;  // first epilogue warp
  static constexpr int THREADS = 32 * EPI0 + 32 * EPIW;
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
// chunked accumulation on 80-column tiles: six stages, so that a chunk of up
// to four k-blocks (all resident while its cross products and then its
// hi x hi products are issued) still leaves loads in flight for the next;
// eight epilogue warps drain the chunk accumulators
using CfgN80C = GemmCfg<80, 6, 4, 2, 8>;

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
  int terms;    // products per k step: 3 (lo x lo dropped) or 4
  int kchunk;   // k-blocks per accumulator chunk (chunked kernels only)
  int cross_first;  // 1: a chunk's cross products before its Ah Bh products
                    // (all its k-blocks resident); 0: k-block by k-block
};

struct GemmMaps {
  CUtensorMap a;
  CUtensorMap bh[GT_MAXT];
  CUtensorMap bl[GT_MAXT];
};

// the mbarriers of one GEMM pass (sized for every configuration below)
constexpr int GB_MAXS = 6, GB_MAXA = 4, GB_MAXACC = 2;
struct GemmBars {
  uint64_t full[GB_MAXS], conv[GB_MAXS], empty[GB_MAXS];
  uint64_t afree[GB_MAXA];
  uint64_t tfull[GB_MAXACC], tempty[GB_MAXACC];
  uint64_t drain;
  int abort;
};

// tensor memory of a CTA: all 512 columns (one CTA per SM); warp 'w' (all
// its lanes) allocates / frees, the address lands in *slot
__device__ __forceinline__ void tmem_alloc_all(uint32_t* slot);
__device__ __forceinline__ void tmem_free_all(uint32_t tmem);

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

// one lane of a converged warp (elect.sync): the lane that issues the
// warp's tcgen05 / TMA instructions
__device__ __forceinline__ bool elect_one() {
  uint32_t p;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "elect.sync _|P, 0xffffffff;\n\t"
      "selp.b32 %0, 1, 0, P;\n\t}"
      : "=r"(p));
  return p != 0;
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

// 16 columns of this warp's 32 lanes without waiting; tmem_wait16 ties the
// wait to the registers, so no use of them can be scheduled before it
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait16(uint32_t* r) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
}

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

template <class CFG, int MODE, bool CHUNK>
__device__ __forceinline__ void gemm_run(const GemmMaps& maps, const GemmShape& shp,
                                         const GemmEpi& epi, int* status, unsigned char* smem,
                                         GemmBars& bars, uint32_t tmem) {
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
  static_assert(STAGES <= GB_MAXS && ASLOTS <= GB_MAXA && ACCBUF <= GB_MAXACC, "barrier set");
  uint64_t* full_bar = bars.full;
  uint64_t* conv_bar = bars.conv;
  uint64_t* empty_bar = bars.empty;
  uint64_t* afree_bar = bars.afree;
  uint64_t* tfull_bar = bars.tfull;
  uint64_t* tempty_bar = bars.tempty;
  uint64_t* const drain = &bars.drain;
  int& abort_flag = bars.abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_total = shp.tile_start[shp.ntypes] * shp.n_tiles;
  const int nk = (shp.K + GT_BK - 1) / GT_BK;

  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&conv_bar[s], CFG::BSPLIT && shp.split_b ? 256 : 128);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < ASLOTS; ++a) mbar_init(&afree_bar[a], 1);
    for (int b = 0; b < ACCBUF; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], 32 * EPIW);
    }
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  volatile int* abort = &abort_flag;

  // The producer and MMA warps run their loops with all 32 lanes, so every
  // stage index, barrier phase, descriptor and TMEM address is warp-uniform
  // and stays in uniform registers; one elected lane issues the TMA copies,
  // MMAs and commits. Measured on the K = 1600 layer: a loop run by lane 0
  // alone spent ~80 cycles per tcgen05.mma (its operands moved into uniform
  // registers instruction by instruction), the warp-uniform loop ~10.
  if (warp == 0) {
    // ---------------------------------------------------------------- TMA
    int g = 0;  // k-blocks issued over all tiles
    bool ok = true;
    for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x) {
      const TileCoord tc = tile_coord(shp, t, BN);
      for (int kb = 0; kb < nk; ++kb, ++g) {
        const int s = g % STAGES;
        const uint32_t ph = (g / STAGES) & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(&empty_bar[s], ph ^ 1, abort))) {
          ok = false;
          break;
        }
        if (elect_one()) {
          unsigned char* st = smem + s * STAGE_BYTES;
          mbar_expect_tx(&full_bar[s], A_BYTES + (shp.split_b ? 1 : 2) * B_BYTES);
          tma_load_2d(st, &maps.a, &full_bar[s], kb * GT_BK, tc.row0);
          tma_load_2d(st + A_BYTES, &maps.bh[tc.ty], &full_bar[s], kb * GT_BK, tc.n0);
          if (!shp.split_b)
            tma_load_2d(st + A_BYTES + B_BYTES, &maps.bl[tc.ty], &full_bar[s], kb * GT_BK,
                        tc.n0);
        }
        __syncwarp();
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
    __syncwarp();
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA
    bool ok = true, issued = false;
    if constexpr (CHUNK) {
      // Chunked accumulation: every kchunk k-blocks start a fresh accumulator
      // (the epilogue adds the chunks in FP32 on the CUDA cores), and within
      // a chunk the small cross products (Al Bh, Ah Bl, Al Bl) go in first,
      // while the accumulator is still small, then the Ah Bh products. The
      // tensor cores' FP32 accumulation loses up to an ulp of the running
      // sum per instruction, always in the same direction; for rows that are
      // alike (the atoms of a crystal) that loss would not average out.
      const int P = shp.kchunk;
      int g = 0, cc = 0;
      for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x) {
        for (int kb0 = 0; kb0 < nk && ok; kb0 += P, ++cc) {
          const int b = cc % ACCBUF;
          if (!__all_sync(0xffffffffu,
                          mbar_wait(&tempty_bar[b], ((cc / ACCBUF) & 1) ^ 1, abort))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t d = tmem + (uint32_t)b * TM_ACC;
          const int nkc = nk - kb0 < P ? nk - kb0 : P;
          for (int i = 0; i < nkc; ++i) {  // pass 1: cross products
            const int gi = g + i, s = gi % STAGES, as = gi % ASLOTS;
            if (!__all_sync(0xffffffffu, mbar_wait(&conv_bar[s], (gi / STAGES) & 1, abort))) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            unsigned char* st = smem + s * STAGE_BYTES;
            const uint32_t ah = tmem + TM_A0 + 64u * (uint32_t)as, al = ah + 32u;
            const uint64_t bh = smem_desc(st + A_BYTES);
            const uint64_t bl = smem_desc(st + A_BYTES + B_BYTES);
            if (elect_one()) {
#pragma unroll
              for (int j = 0; j < GT_BK / 8; ++j) {
                const uint32_t ca = 8u * (uint32_t)j;
                const uint64_t ob = (uint64_t)(j * 32) >> 4;
                mma_tf32_ta(d, al + ca, bh + ob, IDESC, (i > 0 || j > 0) ? 1u : 0u);
                mma_tf32_ta(d, ah + ca, bl + ob, IDESC, 1u);
                if (shp.terms == 4) mma_tf32_ta(d, al + ca, bl + ob, IDESC, 1u);
                if (!shp.cross_first) mma_tf32_ta(d, ah + ca, bh + ob, IDESC, 1u);
              }
              if (!shp.cross_first) {  // k-block order: its stage is free once read
                mma_commit(&empty_bar[s]);
                mma_commit(&afree_bar[as]);
              }
            }
            __syncwarp();
            issued = true;
          }
          if (!ok) break;
          if (elect_one()) {
            for (int i = 0; i < nkc && shp.cross_first; ++i) {  // pass 2: Ah Bh
              const int gi = g + i, s = gi % STAGES, as = gi % ASLOTS;
              unsigned char* st = smem + s * STAGE_BYTES;
              const uint32_t ah = tmem + TM_A0 + 64u * (uint32_t)as;
              const uint64_t bh = smem_desc(st + A_BYTES);
#pragma unroll
              for (int j = 0; j < GT_BK / 8; ++j)
                mma_tf32_ta(d, ah + 8u * (uint32_t)j, bh + ((uint64_t)(j * 32) >> 4), IDESC,
                            1u);
              mma_commit(&empty_bar[s]);
              mma_commit(&afree_bar[as]);
            }
            mma_commit(&tfull_bar[b]);  // chunk accumulator b complete
          }
          __syncwarp();
          g += nkc;
        }
      }
    } else {
      int g = 0, lt = 0;
      for (int t = blockIdx.x; t < n_total && ok; t += gridDim.x, ++lt) {
        const int b = lt % ACCBUF;
        if (!__all_sync(0xffffffffu,
                        mbar_wait(&tempty_bar[b], ((lt / ACCBUF) & 1) ^ 1, abort))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + (uint32_t)b * TM_ACC;
        for (int kb = 0; kb < nk; ++kb, ++g) {
          const int s = g % STAGES;
          const uint32_t ph = (g / STAGES) & 1;
          if (!__all_sync(0xffffffffu, mbar_wait(&conv_bar[s], ph, abort))) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          unsigned char* st = smem + s * STAGE_BYTES;
          const int as = g % ASLOTS;
          const uint32_t ah = tmem + TM_A0 + 64u * (uint32_t)as, al = ah + 32u;
          const uint64_t bh = smem_desc(st + A_BYTES);
          const uint64_t bl = smem_desc(st + A_BYTES + B_BYTES);
          if (elect_one()) {
#pragma unroll
            for (int j = 0; j < GT_BK / 8; ++j) {  // K = 8 per instruction
              const uint32_t ca = 8u * (uint32_t)j;           // TMEM columns
              const uint64_t ob = (uint64_t)(j * 32) >> 4;    // +32 B in the swizzled row
              const uint32_t acc = (kb > 0 || j > 0) ? 1u : 0u;
              mma_tf32_ta(d, ah + ca, bh + ob, IDESC, acc);
              mma_tf32_ta(d, al + ca, bh + ob, IDESC, 1u);
              mma_tf32_ta(d, ah + ca, bl + ob, IDESC, 1u);
              if (shp.terms == 4) mma_tf32_ta(d, al + ca, bl + ob, IDESC, 1u);
            }
            mma_commit(&empty_bar[s]);    // frees the shared-memory stage once read
            mma_commit(&afree_bar[as]);   // and the TMEM A slot
          }
          __syncwarp();
          issued = true;
        }
        if (!ok) break;
        if (elect_one()) mma_commit(&tfull_bar[b]);  // accumulator b complete
        __syncwarp();
      }
    }
    if (!ok && lane == 0) *abort = 1;
    // every MMA issued by this warp has completed before teardown (a CTA
    // without tiles, when the grid is wider than the tiles, issued nothing)
    if (issued) {
      if (elect_one()) mma_commit(drain);
      __syncwarp();
      for (unsigned it = 0; it < GT_WAIT_LIMIT; ++it)
        if (mbar_try(drain, 0)) break;
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
            lo[4 * c + u] = __float_as_uint(tf32_hi(xs[u] - h));
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
  } else if (CFG::BSPLIT && warp < 10) {
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
                    make_float4(tf32_hi(x.x - h.x), tf32_hi(x.y - h.y), tf32_hi(x.z - h.z),
                                tf32_hi(x.w - h.w));
              }
            }
          }
          // generic-proxy writes, read next by the tensor cores (async proxy)
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(&conv_bar[s]);
        }
      }
    }
  } else if (warp >= CFG::EPI0 && warp < CFG::EPI0 + EPIW) {
    // ---------------------------------------------------------------- epilogue
    // warp (warp % 4) owns TMEM lanes 32 * (warp % 4) ..., one row per
    // thread; each 16-column chunk moves as 4 x 16-byte loads / stores per
    // operand (64 contiguous bytes per thread and row)
    const int lane_base = 32 * (warp & 3);
    const int ehalf = EPIW == 8 ? (warp - CFG::EPI0) >> 2 : 0;  // column share of this warp
    constexpr int CSTEP = 16 * (EPIW / 4);               // column stride of this warp's groups
    // chunked kernels: each warp of a lane quadrant owns a contiguous column
    // range, [0, CH0) or [CH0, BN), in 16-column groups
    constexpr int CH0 = EPIW == 8 ? (BN / 2 + 15) / 16 * 16 : BN;
    constexpr int MAXG = CH0 / 16;
    const int cbeg = ehalf ? CH0 : 0;
    const int ngrp = ((ehalf ? BN - CH0 : CH0) + 15) / 16;
    int lt = 0, cc = 0;
    for (int t = blockIdx.x; t < n_total; t += gridDim.x, ++lt) {
      const int b = lt % ACCBUF;
      // chunked accumulation: drain every chunk accumulator of the tile into
      // FP32 register sums (round-to-nearest adds in chunk order)
      float sacc[CHUNK ? MAXG * 16 : 1];
      bool have = true;
      if constexpr (CHUNK) {
#pragma unroll
        for (int k = 0; k < MAXG * 16; ++k) sacc[k] = 0.f;
        for (int kb0 = 0; kb0 < nk; kb0 += shp.kchunk, ++cc) {
          const int cb = cc % ACCBUF;
          have = mbar_wait(&tfull_bar[cb], (cc / ACCBUF) & 1, abort) && !*abort;
          have = __shfl_sync(0xffffffffu, have ? 1 : 0, 0) != 0;
          if (!have) break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t ab =
              tmem + ((uint32_t)lane_base << 16) + (uint32_t)cb * TM_ACC + (uint32_t)cbeg;
#pragma unroll
          for (int i = 0; i < MAXG; i += 2) {  // two groups' loads in flight per wait
            uint32_t v0[16], v1[16];
            if (i < ngrp) tmem_ld16_async(ab + 16u * (uint32_t)i, v0);
            if (i + 1 < MAXG && i + 1 < ngrp) tmem_ld16_async(ab + 16u * (uint32_t)(i + 1), v1);
            if (i < ngrp) {
              tmem_wait16(v0);
#pragma unroll
              for (int k = 0; k < 16; ++k) sacc[16 * i + k] += __uint_as_float(v0[k]);
            }
            if (i + 1 < MAXG && i + 1 < ngrp) {
              tmem_wait16(v1);
#pragma unroll
              for (int k = 0; k < 16; ++k) sacc[16 * (i + 1) + k] += __uint_as_float(v1[k]);
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          mbar_arrive(&tempty_bar[cb]);
        }
      } else {
        have = mbar_wait(&tfull_bar[b], (lt / ACCBUF) & 1, abort) && !*abort;
        have = __shfl_sync(0xffffffffu, have ? 1 : 0, 0) != 0;  // tcgen05.ld is warp-wide
        if (have) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      }
      if (!have) break;
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
      // one 16-column group: aux operands requested first, then the
      // accumulator values (a TMEM load, or the chunk sums), then the
      // layer's elementwise math and the stores
      auto group = [&](int c0, auto&& load_acc) {
        float4 x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // in flight during the TMEM load
          x0[j] = x1[j] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (NEED0 && ok) x0[j] = __ldg(reinterpret_cast<const float4*>(epi.aux0 + at + c0) + j);
          if (NEED1 && ok) x1[j] = __ldg(reinterpret_cast<const float4*>(epi.aux1 + at + c0) + j);
        }
        float v[16];
        load_acc(v);
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
      };
      if constexpr (CHUNK) {
#pragma unroll
        for (int i = 0; i < MAXG; ++i)
          if (i < ngrp)
            group(cbeg + 16 * i, [&](float* v) {
#pragma unroll
              for (int k = 0; k < 16; ++k) v[k] = sacc[16 * i + k];
            });
      } else {
#pragma unroll 1
        for (int c0 = 16 * ehalf; c0 < BN; c0 += CSTEP)
          group(c0, [&](float* v) { tmem_ld16(acc_base + (uint32_t)c0, v); });
        // accumulator b may be overwritten by the tile after next
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(&tempty_bar[b]);
      }
      if (MODE == EPI_LAST && ok) atomicAdd(&epi.e[row], esum);  // per warp's columns
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (abort_flag && threadIdx.x == 0) atomicOr(status, ST_MMA_TIMEOUT);
}


// host: checks one GEMM's arguments and fills its maps / shape / epilogue
// (dpb_gemm_tcgen05.cu)
int gemm_prepare(const float* A, int M, int K, const float* const* b_hi,
                 const float* const* b_lo, int N, const int* type_rows, int ntypes, int mode,
                 float* out0, float* out1, const float* aux0, const float* aux1,
                 const float* const* bias, const float* const* idt, const float* const* w,
                 float* e, int force_bn, GemmMaps& maps, GemmShape& shp, GemmEpi& ep, int& BN);

__device__ __forceinline__ void tmem_alloc_all(uint32_t* slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   su32(slot)),
               "r"(TM_COLS));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free_all(uint32_t tmem) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TM_COLS));
}

}  // namespace dpb
