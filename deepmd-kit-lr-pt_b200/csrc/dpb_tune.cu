// Tile-shape knobs read by the launchers (atoms per CTA, rows per group,
// GEMM N tile). Process-wide values, set by the autotuner (autotune.py) or
// the caller before a step is launched or captured; a captured CUDA graph
// keeps the shapes it was captured with.
#include <cstring>

#include "dpb_common.cuh"

namespace dpb {

struct Knob {
  const char* name;
  int value;
  int nopt;
  int options[6];
};

static Knob g_knobs[] = {
    // warps (one center atom each) per CTA of the fused descriptor kernels
    {"desc_atoms_per_cta", 4, 3, {2, 4, 8}},
    // L1 policy of the table-coefficient loads in the fused descriptor
    // kernels: 0 default, 1 no_allocate, 2 evict_first, 3 evict_last (measured
    // fastest on 12,288-atom water: rows near the switch cutoff are shared),
    // 4 evict_last in L1 and L2
    {"desc_coef_l1", 3, 5, {0, 1, 2, 3, 4}},
    // widest tensor-core tile of the fitting GEMMs (a width is used where it
    // divides N; 240 only for K <= 512)
    {"fit_n_tile", 160, 3, {80, 160, 240}},
    // fitting GEMM weights: 0 pre-split TF32 hi / lo read from L2, 1 FP32
    // read and split in shared memory by four dedicated warps (half the
    // weight bytes; 14% slower on the 12,288-atom water step: the GEMMs are
    // not limited by the weight bytes)
    {"fit_split_b", 0, 2, {0, 1}},
    // TF32 products per k step of the fitting GEMM: 3 (Ah Bh + Al Bh + Ah Bl)
    // or 4 (with Al Bl, 2^-22 of a product: measured to change no output
    // beyond FP32 accumulation noise, at 4% more fitting time)
    {"fit_terms", 3, 2, {3, 4}},
    // k-blocks (32 wide) per accumulator chunk of the fitting GEMM, 0 for one
    // accumulator per output tile: the tensor cores' FP32 accumulation loses
    // up to an ulp of the running sum per instruction, always in the same
    // direction, so long sums over rows that are alike drift
    // (measured, 12,288-atom water fitting stage / worst Cu-frame energy
    // error: 0 298 us / 1.4e-6 eV/atom; 8 k-block order 302 us / 2.3e-7;
    // 4 k-block order 320 us / 1.1e-7; 4 cross first 345 us / 3.1e-8)
    {"fit_kchunk", 8, 5, {0, 1, 2, 4, 8}},
    // order inside a chunk: 1 the cross products of all its k-blocks first
    // (the chunk's stages stay resident until its Ah Bh products are issued;
    // at most 4 k-blocks per chunk), 0 k-block by k-block
    {"fit_kchunk_cross_first", 0, 2, {0, 1}},
    // chunked accumulation only for K at least this (shorter sums drift less)
    {"fit_kchunk_min_k", 0, 2, {0, 512}},
    // warps (one center atom each) per CTA of the batched env / force kernels
    {"batch_atoms_per_cta", 4, 3, {2, 4, 8}},
    // batched-frames step: 1 one persistent cooperative launch
    // (dpb_bt_step_launch), 0 one launch per stage
    {"batch_fused", 0, 2, {0, 1}},
    // knots of the cubic re-interpolated tables every this many fine strides
    // of the reference's table (read by the host when it builds the tables)
    {"table_cubic_stride", 1, 2, {1, 2}},
    // one-launch step: 1 the env rows and the descriptor forward (the
    // descriptor backward and the forces) as separate passes, 0 back to back
    // per row in one pass
    {"batch_fused_split", 0, 2, {0, 1}},
    // neighbor rows per group in the FP32 training kernels
    {"train_rows_per_group", 8, 2, {4, 8}},
    // the same for the FP64 force-backward kernel (also the embedding
    // backward of the FP64 plain evaluation path)
    {"train_rows_per_group_f64", 8, 2, {4, 8}},
    // most warps per CTA of the training kernels (fewer when shared memory
    // does not allow them)
    {"train_warps_per_cta", 8, 4, {1, 2, 4, 8}},
    // reverse training kernel: one weight-gradient copy per block, updated
    // with shared-memory atomics, so 8 warps fit instead of 4 (measured: FP32
    // step 4.19 -> 4.01 ms, FP64 step 15.4 -> 12.8 ms, same gradients)
    {"train_rev_shared_acc", 1, 2, {0, 1}},
    // one frame's wrap / ghost copy / cell grid: 1 one cooperative launch,
    // 0 the separate kernels
    {"geometry_fused", 1, 2, {0, 1}},
    // contraction of the fused descriptor forward: 0 FP32 CUDA cores (packed
    // FMA on the table values in registers), 1 tensor cores (mma.sync
    // m16n8k8, 3xTF32; the table values are evaluated in the MMA fragment
    // layout). Measured on 12,288-atom water: 172 us (0) against 342 us (1),
    // so 1 is a tested option the autotuner does not try
    // (the kernel is bound by the table gathers, which 1 makes scalar)
    {"desc_tc", 0, 2, {0, 1}},
    // SIMT GEMMs (FP64 plain path and training, FP32 odd widths): 1 the
    // 128 x 64 tile with 8 x 4 outputs per thread where M >= 128, 0 the
    // 64 x 64 tile with 4 x 4 outputs
    {"gemm_simt_big", 1, 2, {0, 1}},
    // programmatic dependent launch between the kernels of a step: 1 on
    // (each kernel's launch overlaps the previous kernel's tail), 0 off
    {"pdl", 1, 2, {0, 1}},
};

static Knob* find_knob(const char* name) {
  if (name == nullptr) return nullptr;
  for (auto& k : g_knobs)
    if (std::strcmp(k.name, name) == 0) return &k;
  return nullptr;
}

int tune_value(const char* name, int fallback) {
  const Knob* k = find_knob(name);
  return k ? k->value : fallback;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_tune_count(void) { return (int)(sizeof(g_knobs) / sizeof(g_knobs[0])); }

const char* dpb_tune_name(int index) {
  if (index < 0 || index >= dpb_tune_count()) return nullptr;
  return g_knobs[index].name;
}

int dpb_tune_get(const char* name) {
  const Knob* k = find_knob(name);
  return k ? k->value : -1;
}

int dpb_tune_options(const char* name, int* out, int capacity) {
  const Knob* k = find_knob(name);
  if (k == nullptr) return -1;
  for (int i = 0; i < k->nopt && i < capacity && out; ++i) out[i] = k->options[i];
  return k->nopt;
}

int dpb_tune_set(const char* name, int value) {
  Knob* k = find_knob(name);
  if (k == nullptr) {
    set_error("tune: unknown knob '%s'", name ? name : "(null)");
    return DPB_ERR_INVALID;
  }
  for (int i = 0; i < k->nopt; ++i)
    if (k->options[i] == value) {
      k->value = value;
      return DPB_OK;
    }
  set_error("tune: %d is not an option of %s", value, k->name);
  return DPB_ERR_INVALID;
}

}  // extern "C"
