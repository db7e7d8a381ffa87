// One batched-frames step as ONE persistent cooperative launch (one CTA per
// SM, 18 warps), its passes separated by grid-wide barriers:
//
//   P0  force / virial / atomic-energy accumulators zeroed; every frame's
//       positions wrapped and binned into its cells (one CTA per frame)
//   P1  one warp per center row: the env row and neighbor list over the 27
//       lattice cells (bt_env_row), then at once the row's compressed
//       embedding, contraction and descriptor (desc_fwd_atom), reading the env
//       row just written from L2
//   P2-P7 the six fitting GEMMs on the tensor cores (gemm_run: TMA ring,
//       TF32 hi / lo split into TMEM, tcgen05.mma, fused epilogues), the
//       80-column tiles with chunked accumulation; tensor memory is allocated
//       once for the whole launch
//   P8  one CTA per frame: the frame's energy in FP64; then one warp per row:
//       the descriptor backward (desc_bwd_atom) and at once the row's forces
//       and virial (bt_force_row), reading net_deriv just written from L2
//
// The same device bodies as the per-stage kernels (dpb_batch.cu, dpb_se_a.cu,
// dpb_gemm_tcgen05.cu), so the results agree with the staged step up to the
// order of the atomic sums.
//
// Memory ordering between passes: every grid barrier is a release (fence +
// arrival) and an acquire (acquire loads of the counter, fence) at GPU scope.
// Generic writes that a later pass reads through TMA (descriptor rows, layer
// activations) are followed by fence.proxy.async before the barrier; shared
// memory switches between generic use (P0, P1, P8) and TMA use (P2-P7), with
// a shared-memory proxy fence at each switch. Rows written and read back in
// the same pass (env row, net_deriv) are read with L2-coherent loads.
//
// Every barrier wait is bounded (BS_WAIT_NS); a CTA that gives up sets
// ST_SYNC_TIMEOUT and skips the remaining passes, and every CTA frees its
// tensor memory before it returns. The GEMM passes keep their own bounded
// mbarrier waits (ST_MMA_TIMEOUT).
#include <stddef.h>

#include <algorithm>

#include "dpb_batch_dev.cuh"
#include "dpb_desc_dev.cuh"
#include "dpb_gemm_dev.cuh"

namespace dpb {

constexpr int BS_WARPS = 16;
constexpr int BS_THREADS = 32 * BS_WARPS;
constexpr int BS_CH = 3;  // table-coefficient loads: L1::evict_last
constexpr int BS_PASSES = 6;
constexpr unsigned long long BS_WAIT_NS = 500000000ull;  // per barrier

// The GEMM passes of the step kernel: 80-column tiles (N = 240 and the
// N = 1600 input gradient), chunk-draining epilogue, a THREE-stage ring. The
// L1 cache and shared memory share 256 KB per SM and the split is fixed per
// launch: the descriptor passes gather table rows through L1, so the step
// kernel keeps its shared memory small (the ring, or the per-warp descriptor
// staging, whichever is larger) and leaves the rest to L1.
//
// 16 warps per CTA (512 threads): registers are allocated to warps in
// groups of four, so 16 warps can have 128 registers a thread where 18 have
// 96 (at 96 the descriptor passes spilled). The GEMM passes use 14 of them:
// the weights are pre-split, so no weight-splitting warps, and 8 epilogue
// warps (40 or 48 chunk sums a thread).
using CfgBS = GemmCfg<80, 3, 4, 2, 8, false>;
static_assert(CfgBS::THREADS <= BS_THREADS, "the GEMM passes fit in the step kernel's warps");

struct BtStepArgs {
  GemmMaps maps[BS_PASSES];
  GemmShape shp[BS_PASSES];
  GemmEpi epi[BS_PASSES];
  BtFrames fr;
  BtSec sec;
  TypeTables tt;
  double* cw;
  int* cell_of;
  int* cell_start;
  int* cell_atoms;
  const double* coord;
  const int* type;
  const float* avg;
  const float* std_;
  float* em;
  int* nlist;
  const int* drow;
  float* xyz;
  float* D;
  const float* dD;
  float* net_deriv;
  float* e_rows;
  const double* e_const;
  double* energy;
  double* force;
  double* virial;
  unsigned* sync;  // [0] barrier arrivals, [1]-[4] row counters, [5] frame counter
  int* status;
  unsigned long long* pass_ns;
  int nrows, M, naxis, wsm_floats;
  int split_rows;  // 1: env / descriptor forward (descriptor backward / forces)
                   // as separate passes, rows through memory; 0: one pass each
  float inv_nnei, rcut, rcut_smth;
};

__device__ __forceinline__ unsigned long long bs_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// grid barrier number k (k * gridDim.x arrivals); false in every thread of
// a CTA that gave up waiting
__device__ bool bs_sync(const BtStepArgs& a, unsigned k, int* s_ok) {
  asm volatile("fence.proxy.async.global;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned target = k * gridDim.x;
    __threadfence();
    atomicAdd(a.sync, 1u);
    int ok = 1;
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.sync) : "memory");
    if (v < target) {
      const unsigned long long t0 = bs_clock();
      for (unsigned it = 0;; ++it) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.sync) : "memory");
        if (v >= target) break;
        if (it > (1u << 24) || bs_clock() - t0 > BS_WAIT_NS) {
          atomicOr(a.status, ST_SYNC_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return *s_ok != 0;
}

// next work item of a pass for this warp (rows are taken dynamically: rows
// of Cu and water frames differ in cost)
__device__ __forceinline__ int bs_next_row(unsigned* counter, int lane) {
  int r = 0;
  if (lane == 0) r = (int)atomicAdd(counter, 1u);
  return __shfl_sync(0xffffffffu, r, 0);
}
// next frame for the whole CTA
__device__ __forceinline__ int bs_next_frame(unsigned* counter, int* s_item) {
  __syncthreads();
  if (threadIdx.x == 0) *s_item = (int)atomicAdd(counter, 1u);
  __syncthreads();
  return *s_item;
}
__device__ __forceinline__ void bs_stamp(const BtStepArgs& a, int k) {
  if (a.pass_ns != nullptr && blockIdx.x == 0 && threadIdx.x == 0) a.pass_ns[k] = bs_clock();
}

// shared memory leaves generic use for TMA use (or back)
__device__ __forceinline__ void bs_smem_switch() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
}

// The per-row work of the row passes.
__device__ __forceinline__ void bs_row_env(const BtStepArgs& a, int row, int lane, float* wsm) {
  bt_env_row<float>(row, lane, *reinterpret_cast<BtEnvSmem*>(wsm), a.em, a.nlist, a.cw, a.type,
                    a.cell_of, a.cell_start, a.cell_atoms, a.avg, a.std_, a.fr, a.sec, a.rcut,
                    a.rcut_smth, a.status);
}

template <int NC, bool COH>
__device__ __forceinline__ void bs_row_fwd(const BtStepArgs& a, int row, int lane, float* wsm) {
  desc_fwd_atom<BS_CH, NC, COH>(row, lane, wsm, a.xyz, a.D, a.drow, a.em, a.tt, a.M, a.naxis,
                                a.inv_nnei);
}

template <int NC>
__device__ __forceinline__ void bs_row_bwd(const BtStepArgs& a, int row, int lane, float* wsm) {
  desc_bwd_atom<BS_CH, NC>(row, lane, wsm, a.net_deriv, a.dD, a.drow, a.xyz, a.em, a.tt, a.M,
                           a.naxis, a.inv_nnei);
}

template <bool COH>
__device__ __forceinline__ void bs_row_force(const BtStepArgs& a, int row, int lane) {
  bt_force_row<float, COH>(row, lane, a.force, a.virial, a.net_deriv, a.cw, a.type, a.std_,
                           a.nlist, a.fr, a.sec.ntypes, a.sec.nnei, a.rcut, a.rcut_smth);
}

template <int MODE>
__device__ __forceinline__ void bs_gemm(const BtStepArgs& a, int l, unsigned char* smem,
                                     GemmBars& bars, uint32_t tmem) {
  gemm_run<CfgBS, MODE, true>(a.maps[l], a.shp[l], a.epi[l], a.status, smem, bars, tmem);
}

template <int NC>
__global__ void __launch_bounds__(BS_THREADS, 1) k_bt_step(const __grid_constant__ BtStepArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ GemmBars bars[BS_PASSES];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_ok, s_item;
  __shared__ double s_part[BS_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 1) tmem_alloc_all(&tmem_slot);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const int nrows = a.nrows, F = a.fr.nframes;
  const int gthreads = gridDim.x * BS_THREADS, gtid = blockIdx.x * BS_THREADS + threadIdx.x;
  float* wsm = reinterpret_cast<float*>(smem) + (size_t)warp * a.wsm_floats;
  unsigned k = 0;
  bs_stamp(a, 0);

  // ---- P0: accumulators, cells
  for (int q = gtid; q < 3 * nrows; q += gthreads) a.force[q] = 0.;
  for (int q = gtid; q < 9 * F; q += gthreads) a.virial[q] = 0.;
  for (int q = gtid; q < nrows; q += gthreads) a.e_rows[q] = 0.f;
  for (int f = bs_next_frame(a.sync + 5, &s_item); f < F; f = bs_next_frame(a.sync + 5, &s_item))
    bt_cells_frame(f, a.cw, a.cell_of, a.cell_start, a.cell_atoms, a.coord, a.fr,
                   reinterpret_cast<int*>(smem));
  bool ok = bs_sync(a, ++k, &s_ok);
  bs_stamp(a, k);

  // ---- P1: env rows + descriptor forward
  if (ok) {
    for (int row = bs_next_row(a.sync + 1, lane); row < nrows;
         row = bs_next_row(a.sync + 1, lane)) {
      bs_row_env(a, row, lane, wsm);
      __syncwarp();
      if (!a.split_rows) {
        bs_row_fwd<NC, true>(a, row, lane, wsm);
        __syncwarp();
      }
    }
    if (a.split_rows) {
      ok = bs_sync(a, ++k, &s_ok);
      bs_stamp(a, k);
      if (ok)
        for (int row = bs_next_row(a.sync + 2, lane); row < nrows;
             row = bs_next_row(a.sync + 2, lane)) {
          bs_row_fwd<NC, false>(a, row, lane, wsm);
          __syncwarp();
        }
    }
    bs_smem_switch();
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }

  // ---- P2-P7: the fitting GEMMs
  if (ok) {
    bs_gemm<EPI_TANH>(a, 0, smem, bars[0], tmem);
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }
  if (ok) {
    bs_gemm<EPI_RES_DT>(a, 1, smem, bars[1], tmem);
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }
  if (ok) {
    bs_gemm<EPI_LAST>(a, 2, smem, bars[2], tmem);
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }
  if (ok) {
    bs_gemm<EPI_BWD_DT>(a, 3, smem, bars[3], tmem);
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }
  if (ok) {
    bs_gemm<EPI_BWD_RES>(a, 4, smem, bars[4], tmem);
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }
  if (ok) {
    bs_gemm<EPI_STORE>(a, 5, smem, bars[5], tmem);
    bs_smem_switch();
    ok = bs_sync(a, ++k, &s_ok);
    bs_stamp(a, k);
  }

  // ---- P8: energies, descriptor backward + forces
  if (ok) {
    for (int f = blockIdx.x; f < F; f += gridDim.x) {
      bt_energy_frame<float>(f, a.energy, a.e_rows, a.drow, a.e_const, a.fr, s_part);
      __syncthreads();
    }
    for (int row = bs_next_row(a.sync + 3, lane); row < nrows;
         row = bs_next_row(a.sync + 3, lane)) {
      bs_row_bwd<NC>(a, row, lane, wsm);
      __syncwarp();
      if (!a.split_rows) {
        bs_row_force<true>(a, row, lane);
        __syncwarp();
      }
    }
    if (a.split_rows) {
      ok = bs_sync(a, ++k, &s_ok);
      bs_stamp(a, k);
      if (ok)
        for (int row = bs_next_row(a.sync + 4, lane); row < nrows;
             row = bs_next_row(a.sync + 4, lane)) {
          bs_row_force<false>(a, row, lane);
          __syncwarp();
        }
    }
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (ok && a.pass_ns != nullptr && threadIdx.x == 0) {
    // the end of the last pass: when the last CTA finishes it
    __threadfence();
    if (atomicAdd(a.sync, 1u) == (k + 1) * gridDim.x - 1) a.pass_ns[k + 1] = bs_clock();
  }
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tmem_free_all(tmem);
  }
}

struct BtStepPlan {
  BtStepArgs a;
  int nc;
  int grid;
  size_t smem;
};


}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_bt_step_create(void** plan, const dpb_bt_step_desc* d) {
  if (plan == nullptr || d == nullptr) {
    set_error("bt_step: plan and description required");
    return DPB_ERR_INVALID;
  }
  *plan = nullptr;
  BtStepArgs a{};
  int rc = bt_frames(a.fr, d->atom_off, d->cell_off, d->box, d->ncell, d->row_frame,
                     d->nframes);
  if (rc) return rc;
  if (d->sec == nullptr || d->nsec < 2 || d->nsec - 1 > BT_MAXT || d->sec[0] != 0 ||
      d->sec[d->nsec - 1] > BT_NMAX || d->status == nullptr || d->sync == nullptr ||
      d->nrows <= 0) {
    set_error("bt_step: need 1..%d types, sum(sel) <= %d, rows, a status word and a barrier "
              "word", BT_MAXT, BT_NMAX);
    return DPB_ERR_INVALID;
  }
  a.sec.ntypes = d->nsec - 1;
  a.sec.nnei = d->sec[d->nsec - 1];
  for (int q = 0; q < d->nsec; ++q) a.sec.sec[q] = d->sec[q];
  if (d->table_degree != 3 && d->table_degree != 5) {
    set_error("bt_step: table_degree must be 3 or 5");
    return DPB_ERR_INVALID;
  }
  if ((rc = make_tables(a.tt, d->tables, d->table_info, d->sec, d->nsec, d->M,
                        d->table_degree == 3)))
    return rc;
  if (d->naxis <= 0 || d->naxis > MAXAX || d->naxis > d->M) {
    set_error("bt_step: axis_neuron must be in [1, %d] and at most M", MAXAX);
    return DPB_ERR_INVALID;
  }
  const int nnei = a.sec.nnei;
  size_t wf = std::max(fwd_smem_floats(d->M, nnei), bwd_smem_floats(d->M, nnei, d->naxis));
  wf = std::max(wf, (sizeof(BtEnvSmem) + 3) / 4);
  wf = (wf + 3) / 4 * 4;
  const size_t smem = std::max({(size_t)CfgBS::SMEM, wf * 4 * BS_WARPS + 1024,
                                (size_t)4 * (BT_MAXCELLS + 1) + 1024});
  if (smem + 4096 > 232448) {
    set_error("bt_step: the per-warp descriptor staging (%zu B) does not fit", wf * 4);
    return DPB_ERR_INVALID;
  }
  // the six fitting GEMMs, in the order and with the epilogues of the step
  static const int modes[BS_PASSES] = {EPI_TANH, EPI_RES_DT, EPI_LAST,
                                       EPI_BWD_DT, EPI_BWD_RES, EPI_STORE};
  // chunked accumulation as the fit_kchunk* knobs ask (at least one chunk
  // per tile: the 80-column passes always drain through the chunk sums)
  const int cross_first = tune_value("fit_kchunk_cross_first", 0) != 0;
  int P = tune_value("fit_kchunk", 8);
  if (cross_first) P = std::min(P, std::min(CfgBS::STAGES, CfgBS::ASLOTS));
  if (P <= 0) P = 1 << 20;  // one chunk per tile
  for (int l = 0; l < BS_PASSES; ++l) {
    const dpb_gemm_layer& g = d->fit[l];
    if (g.mode != modes[l] || g.b_lo == nullptr) {
      set_error("bt_step: fitting GEMM %d must have epilogue %d and pre-split weights", l,
                modes[l]);
      return DPB_ERR_INVALID;
    }
    int bn = 0;
    rc = gemm_prepare(g.A, d->nrows, g.K, g.b_hi, g.b_lo, g.N, d->type_rows, d->ntypes,
                      g.mode, g.out0, g.out1, g.aux0, g.aux1, g.bias, g.idt, g.w, d->e_rows,
                      CfgBS::BN, a.maps[l], a.shp[l], a.epi[l], bn);
    if (rc) return rc;
    a.shp[l].kchunk = P;
    a.shp[l].cross_first = cross_first && P <= CfgBS::STAGES;
  }
  a.cw = d->cw;
  a.cell_of = d->cell_of;
  a.cell_start = d->cell_start;
  a.cell_atoms = d->cell_atoms;
  a.coord = d->coord;
  a.type = d->type;
  a.avg = d->avg;
  a.std_ = d->std_;
  a.em = d->em;
  a.nlist = d->nlist;
  a.drow = d->drow;
  a.xyz = d->xyz;
  a.D = d->descrpt;
  a.dD = d->d_descrpt;
  a.net_deriv = d->net_deriv;
  a.e_rows = d->e_rows;
  a.e_const = d->e_const;
  a.energy = d->energy;
  a.force = d->force;
  a.virial = d->virial;
  a.sync = d->sync;
  a.status = d->status;
  a.pass_ns = d->pass_ns;
  a.split_rows = tune_value("batch_fused_split", 0) != 0;
  a.nrows = d->nrows;
  a.M = d->M;
  a.naxis = d->naxis;
  a.wsm_floats = (int)wf;
  a.inv_nnei = 1.f / (float)nnei;
  a.rcut = d->rcut;
  a.rcut_smth = d->rcut_smth;
  if (!a.cw || !a.cell_of || !a.cell_start || !a.cell_atoms || !a.coord || !a.type || !a.avg ||
      !a.std_ || !a.em || !a.nlist || !a.drow || !a.xyz || !a.D || !a.dD || !a.net_deriv ||
      !a.e_rows || !a.e_const || !a.energy || !a.force || !a.virial) {
    set_error("bt_step: a device buffer of the description is NULL");
    return DPB_ERR_INVALID;
  }
  const int nc = d->table_degree + 1;
  const void* fn = nc == 4 ? (const void*)k_bt_step<4> : (const void*)k_bt_step<6>;
  DPB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
           "bt_step");
  // the smallest shared-memory carve-out that holds it: the rest is L1
  const int pct = (int)std::min<size_t>(100, ((smem + 4096) * 100 + 233471) / 233472);
  DPB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct),
           "bt_step");
  int per_sm = 0;
  DPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, BS_THREADS, smem),
           "bt_step");
  if (per_sm < 1) {
    set_error("bt_step: the step kernel does not fit on an SM");
    return DPB_ERR_INVALID;
  }
  BtStepPlan* p = new BtStepPlan;
  p->a = a;
  p->nc = nc;
  p->grid = sm_count();
  p->smem = smem;
  *plan = p;
  return DPB_OK;
}

int dpb_bt_step_launch(const void* plan, dpb_stream_t stream) {
  if (plan == nullptr) {
    set_error("bt_step: no plan");
    return DPB_ERR_INVALID;
  }
  const BtStepPlan* p = static_cast<const BtStepPlan*>(plan);
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(cudaMemsetAsync(p->a.sync, 0, 8 * sizeof(unsigned), st), "bt_step");
  void* args[] = {(void*)&p->a};
  const void* fn = p->nc == 4 ? (const void*)k_bt_step<4> : (const void*)k_bt_step<6>;
  DPB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(p->grid), dim3(BS_THREADS), args, p->smem, st),
           "bt_step");
  return DPB_OK;
}

void dpb_bt_step_destroy(void* plan) { delete static_cast<BtStepPlan*>(plan); }

long long dpb_bt_step_desc_layout(int which) {
  switch (which) {
    case 0: return (long long)sizeof(dpb_bt_step_desc);
    case 1: return (long long)offsetof(dpb_bt_step_desc, fit);
    case 2: return (long long)offsetof(dpb_bt_step_desc, status);
    case 3: return (long long)sizeof(dpb_gemm_layer);
    case 4: return (long long)offsetof(dpb_gemm_layer, w);
    default: return -1;
  }
}

}  // extern "C"
