// FP32-accurate GEMM on the 5th-generation tensor cores (sm_100a tcgen05)
// for the per-type fitting networks, with the layer's elementwise math fused
// into the epilogue.
//
//   C[m, n] = sum_k A[m, k] B[n, k]      A: [M, K] FP32 row-major (activations)
//                                        B: [N, K] FP32 row-major (weights),
//                                           given pre-split into TF32 hi / lo,
//                                           or in FP32 and split in the kernel
// Split TF32: A = Ah + Al and B = Bh + Bl with Ah, Bh the TF32 roundings and
// Al, Bl the TF32 roundings of the remainders (so A and B are represented to
// 2^-24 relative, FP32 resolution); the product is Ah Bh + Al Bh + Ah Bl
// (3xTF32, the default) or with the Al Bl term too (knob fit_terms = 4),
// accumulated in FP32 in tensor memory. The tensor cores' FP32 accumulation
// loses up to an ulp of the running sum per instruction, always in the same
// direction: over K = 1600 that is ~1.5e-5 of the output scale, and it does
// not average out where rows are alike (the atoms of a crystal). So long
// sums are accumulated in chunks (knob fit_kchunk k-blocks per chunk, 8 by
// default, on the 80-column tiles): each chunk starts a fresh TMEM
// accumulator and the epilogue warps add the chunks in FP32 (round to
// nearest) in registers. With knob fit_kchunk_cross_first a chunk (at most 4
// k-blocks) also takes its small cross products before its Ah Bh products,
// which brings the error to FP32-GEMM level (~5e-7 on the same rows) at
// 15% more fitting time.
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

#include "dpb_gemm_dev.cuh"

namespace dpb {

template <class CFG, int MODE, bool CHUNK>
__global__ void __launch_bounds__(CFG::THREADS, 1)
k_gemm_tf32x3(const __grid_constant__ GemmMaps maps, GemmShape shp, GemmEpi epi, int* status) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ GemmBars bars;
  __shared__ uint32_t tmem_slot;
  if ((threadIdx.x >> 5) == 1) tmem_alloc_all(&tmem_slot);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  // tensor memory is held: wait for the previous kernel of the stream before
  // the first global access
  pdl_wait();
  pdl_trigger();
  gemm_run<CFG, MODE, CHUNK>(maps, shp, epi, status, smem, bars, tmem);
  if ((threadIdx.x >> 5) == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tmem_free_all(tmem);
  }
}

// ---------------------------------------------------------------- host -----
template <class CFG, int MODE, bool CHUNK>
static int launch_mode(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi,
                       int* status, cudaStream_t st) {
  DPB_CUDA(cudaFuncSetAttribute(k_gemm_tf32x3<CFG, MODE, CHUNK>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, CFG::SMEM),
           "gemm");
  const int tiles = shp.tile_start[shp.ntypes] * shp.n_tiles;
  if (tiles == 0) return DPB_OK;
  const int sms = sm_count();
  const int grid = tiles < sms ? tiles : sms;
  DPB_CUDA(launch_pdl(k_gemm_tf32x3<CFG, MODE, CHUNK>, dim3(grid), dim3(CFG::THREADS),
                      (size_t)CFG::SMEM, st, maps, shp, epi, status),
           "gemm_tf32x3");
  return DPB_OK;
}

template <class CFG, bool CHUNK>
static int launch_c(const GemmMaps& maps, const GemmShape& shp, const GemmEpi& epi, int* status,
                    cudaStream_t st) {
  switch (epi.mode) {
    case EPI_STORE: return launch_mode<CFG, EPI_STORE, CHUNK>(maps, shp, epi, status, st);
    case EPI_TANH: return launch_mode<CFG, EPI_TANH, CHUNK>(maps, shp, epi, status, st);
    case EPI_RES_DT: return launch_mode<CFG, EPI_RES_DT, CHUNK>(maps, shp, epi, status, st);
    case EPI_LAST: return launch_mode<CFG, EPI_LAST, CHUNK>(maps, shp, epi, status, st);
    case EPI_BWD_DT: return launch_mode<CFG, EPI_BWD_DT, CHUNK>(maps, shp, epi, status, st);
    default: return launch_mode<CFG, EPI_BWD_RES, CHUNK>(maps, shp, epi, status, st);
  }
}

// Chunked accumulation when the knob asks for it and the tile has more
// k-blocks than one chunk; a chunk's k-blocks must all be resident (stages
// and TMEM A slots). Only the 80-column tile (the N = 240 layers, among them
// the K = 1600 first layer) has it: the wider tiles' epilogue threads cannot
// hold the chunk sums in registers without spilling.
template <class CFG>
static int launch(const GemmMaps& maps, GemmShape shp, const GemmEpi& epi, int* status,
                  cudaStream_t st) {
  shp.kchunk = 0;
  shp.cross_first = 0;
  if constexpr (CFG::BN == 80) {
    using C = CfgN80C;
    const int nk = (shp.K + GT_BK - 1) / GT_BK;
    shp.cross_first = tune_value("fit_kchunk_cross_first", 0) != 0;
    int P = tune_value("fit_kchunk", 8);
    if (shp.cross_first) P = std::min(P, std::min(C::STAGES, C::ASLOTS));
    if (P > 0 && nk > P && shp.K >= tune_value("fit_kchunk_min_k", 0)) {
      shp.kchunk = P;
      return launch_c<C, true>(maps, shp, epi, status, st);
    }
  }
  return launch_c<CFG, false>(maps, shp, epi, status, st);
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

// Checks the arguments of one GEMM and fills its tensor maps, tile shape and
// epilogue. The tile width is force_bn when non-zero (it must divide N),
// else the widest the fit_n_tile knob allows that divides N (240 only for
// K <= 512, where two pipeline stages keep the tensor cores fed). No chunked
// accumulation is set (kchunk = 0).
int gemm_prepare(const float* A, int M, int K, const float* const* b_hi,
                 const float* const* b_lo, int N, const int* type_rows, int ntypes, int mode,
                 float* out0, float* out1, const float* aux0, const float* aux1,
                 const float* const* bias, const float* const* idt, const float* const* w,
                 float* e, int force_bn, GemmMaps& maps, GemmShape& shp, GemmEpi& ep, int& BN) {
  if (ntypes < 1 || ntypes > GT_MAXT || M < 0 || K <= 0 || N <= 0 || mode < 0 ||
      mode > EPI_BWD_RES || type_rows == nullptr || b_hi == nullptr) {
    set_error("gemm_tf32x3: invalid arguments (ntypes=%d M=%d K=%d N=%d mode=%d)", ntypes, M,
              K, N, mode);
    return DPB_ERR_INVALID;
  }
  int rc = get_encoder();
  if (rc) return rc;
  if (N % 80 != 0 || (force_bn && N % force_bn != 0)) {
    set_error("gemm_tf32x3: N=%d must be a multiple of 80 (and of the tile width %d)", N,
              force_bn);
    return DPB_ERR_INVALID;
  }
  const int knob = tune_value("fit_n_tile", CfgN160::BN);
  BN = force_bn ? force_bn
       : (knob >= CfgN240::BN && N % CfgN240::BN == 0 && K <= 512) ? CfgN240::BN
       : (knob >= CfgN160::BN && N % CfgN160::BN == 0)            ? CfgN160::BN
                                                                  : CfgN80::BN;
  shp = GemmShape{};
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
  shp.terms = tune_value("fit_terms", 3) == 4 ? 4 : 3;
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
  ep = GemmEpi{};
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
  if (status == nullptr) {
    set_error("gemm_tf32x3: a status word is required");
    return DPB_ERR_INVALID;
  }
  GemmMaps maps;
  GemmShape shp;
  GemmEpi ep;
  int BN = 0;
  const int rc = gemm_prepare(A, M, K, b_hi, b_lo, N, type_rows, ntypes, mode, out0, out1, aux0,
                              aux1, bias, idt, w, e, 0, maps, shp, ep, BN);
  if (rc || M == 0) return rc;
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
