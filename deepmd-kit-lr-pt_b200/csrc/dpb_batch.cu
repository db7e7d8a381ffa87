// Many frames of uneven size in one pass per stage (batched workload): the
// geometry of every frame is handled by the same launch instead of one launch
// sequence per frame.
//
//  k_bt_cells  : one CTA per frame: positions wrapped into the frame's
//                orthorhombic box, atoms binned into cells of edge >= rcut
//                (counting sort in shared memory).
//  k_bt_env    : one warp per center atom of any frame: the 27 lattice cells
//                around the center, each mapped to (cell, periodic image), so
//                ghosts are never materialised; the candidate tests, keys
//                (type, float r^2, index) and slot filling of the single-frame
//                env pass (format_nlist_i_cpu order, fmt_nlist.cc:98-143), the
//                index being (local atom * 27 + image code); env rows in FP32
//                from FP64 differences (env_mat.cc:146-205).
//  k_bt_force  : one warp per center: the env derivative recomputed from the
//                packed (atom, image) index, pair forces added to the owners
//                directly (no ghost fold), the virial reduced per warp into
//                its frame's 9 components (prod_force.cc:23-72,
//                prod_virial.cc:22-69).
//  k_bt_energy : one CTA per frame: the atomic energies of its rows plus the
//                per-type constants, summed in FP64.
// Requirements checked on the host: orthorhombic boxes whose edges are all
// at least rcut (every neighbor then lies in the 27 lattice cells), at most
// 4096 cells and 600,000 atoms per frame.
#include "dpb_batch_dev.cuh"

namespace dpb {

__global__ void __launch_bounds__(256)
k_bt_cells(double* __restrict__ cw, int* __restrict__ cell_of, int* __restrict__ cell_start,
           int* __restrict__ cell_atoms, const double* __restrict__ coord, BtFrames fr) {
  __shared__ int cnt[BT_MAXCELLS + 1];
  pdl_wait();
  pdl_trigger();
  bt_cells_frame(blockIdx.x, cw, cell_of, cell_start, cell_atoms, coord, fr, cnt);
}

template <typename ET, int WP>
__global__ void __launch_bounds__(WP * 32)
k_bt_env(ET* __restrict__ em, int* __restrict__ nlist, const double* __restrict__ cw,
         const int* __restrict__ type, const int* __restrict__ cell_of,
         const int* __restrict__ cell_start, const int* __restrict__ cell_atoms,
         const ET* __restrict__ avg, const ET* __restrict__ std_, BtFrames fr, BtSec sec,
         int nrows, float rcut, float rcut_smth, int* status) {
  __shared__ BtEnvSmem smem[WP];
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WP + w;
  if (row >= nrows) return;
  bt_env_row<ET>(row, lane, smem[w], em, nlist, cw, type, cell_of, cell_start, cell_atoms, avg,
                 std_, fr, sec, rcut, rcut_smth, status);
}

template <typename ET, int WP>
__global__ void __launch_bounds__(WP * 32)
k_bt_force(double* __restrict__ force, double* __restrict__ virial,
           const ET* __restrict__ nd, const double* __restrict__ cw,
           const int* __restrict__ type, const ET* __restrict__ std_,
           const int* __restrict__ nlist, BtFrames fr, int ntypes, int nnei, int nrows,
           float rcut, float rcut_smth) {
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WP + w;
  if (row >= nrows) return;
  bt_force_row<ET>(row, lane, force, virial, nd, cw, type, std_, nlist, fr, ntypes, nnei, rcut,
                   rcut_smth);
}

template <typename ET>
__global__ void __launch_bounds__(256)
k_bt_energy(double* __restrict__ energy, const ET* __restrict__ e_rows,
            const int* __restrict__ drow, const double* __restrict__ e_const, BtFrames fr) {
  __shared__ double part[8];
  pdl_wait();
  pdl_trigger();
  bt_energy_frame<ET>(blockIdx.x, energy, e_rows, drow, e_const, fr, part);
}

}  // namespace dpb

namespace dpb {

template <typename ET>
static int batch_env(ET* em, int* nlist, double* cw, int* cell_of, int* cell_start,
                     int* cell_atoms, const double* coord, const int* type, const ET* avg,
                     const ET* std_, const int* atom_off, const int* cell_off, const double* box,
                     const int* ncell, const int* row_frame, int nframes, int nrows, float rcut,
                     float rcut_smth, const int* sec, int nsec, int* status, dpb_stream_t stream) {
  BtFrames fr;
  int rc = bt_frames(fr, atom_off, cell_off, box, ncell, row_frame, nframes);
  if (rc) return rc;
  if (sec == nullptr || nsec < 2 || nsec - 1 > BT_MAXT || sec[0] != 0 ||
      sec[nsec - 1] > BT_NMAX || status == nullptr) {
    set_error("batch_env_mat_a: need 1..%d types, sum(sel) <= %d and a status word", BT_MAXT,
              BT_NMAX);
    return DPB_ERR_INVALID;
  }
  BtSec s{};
  s.ntypes = nsec - 1;
  s.nnei = sec[nsec - 1];
  for (int k = 0; k < nsec; ++k) s.sec[k] = sec[k];
  if (nrows <= 0) return DPB_OK;
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(launch_pdl(k_bt_cells, dim3(nframes), dim3(256), 0, st, cw, cell_of, cell_start,
                      cell_atoms, coord, fr),
           "batch_env_mat_a/cells");
  auto run = [&](auto kern, int wp) -> int {
    DPB_CUDA(launch_pdl(kern, dim3(ceil_div(nrows, wp)), dim3(wp * 32), 0, st, em, nlist, cw,
                        type, (const int*)cell_of, (const int*)cell_start,
                        (const int*)cell_atoms, avg, std_, fr, s, nrows, rcut, rcut_smth,
                        status),
             "batch_env_mat_a/env");
    return DPB_OK;
  };
  switch (tune_value("batch_atoms_per_cta", BT_WARPS)) {
    case 2: return run(k_bt_env<ET, 2>, 2);
    case 8: return run(k_bt_env<ET, 8>, 8);
    default: return run(k_bt_env<ET, 4>, 4);
  }
}

template <typename ET>
static int batch_force(double* force, double* virial, const ET* net_deriv, const double* cw,
                       const int* type, const ET* std_, const int* nlist, const int* atom_off,
                       const int* cell_off, const double* box, const int* ncell,
                       const int* row_frame, int nframes, int nrows, int nnei, int ntypes,
                       float rcut, float rcut_smth, dpb_stream_t stream) {
  BtFrames fr;
  int rc = bt_frames(fr, atom_off, cell_off, box, ncell, row_frame, nframes);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * 3 * (size_t)nrows, st), "batch_force");
  DPB_CUDA(cudaMemsetAsync(virial, 0, sizeof(double) * 9 * (size_t)nframes, st),
           "batch_force");
  if (nrows <= 0 || nnei <= 0) return DPB_OK;
  auto run = [&](auto kern, int wp) -> int {
    DPB_CUDA(launch_pdl(kern, dim3(ceil_div(nrows, wp)), dim3(wp * 32), 0, st, force, virial,
                        net_deriv, cw, type, std_, nlist, fr, ntypes, nnei, nrows, rcut,
                        rcut_smth),
             "batch_force_virial_a");
    return DPB_OK;
  };
  switch (tune_value("batch_atoms_per_cta", BT_WARPS)) {
    case 2: return run(k_bt_force<ET, 2>, 2);
    case 8: return run(k_bt_force<ET, 8>, 8);
    default: return run(k_bt_force<ET, 4>, 4);
  }
}

template <typename ET>
static int batch_energy(double* energy, const ET* e_rows, const int* drow, const double* e_const,
                        const int* atom_off, int nframes, dpb_stream_t stream) {
  if (nframes <= 0 || !energy || !e_rows || !drow || !e_const || !atom_off) {
    set_error("batch_energy: invalid arguments");
    return DPB_ERR_INVALID;
  }
  BtFrames fr{atom_off, nullptr, nullptr, nullptr, nullptr, nframes};
  DPB_CUDA(launch_pdl(k_bt_energy<ET>, dim3(nframes), dim3(256), 0, as_stream(stream), energy,
                      e_rows, drow, e_const, fr),
           "batch_energy");
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

#define DPB_BATCH_ENTRIES(SUF, ET)                                                              \
  int dpb_batch_env_mat_a_##SUF(ET* em, int* nlist, double* cw, int* cell_of, int* cell_start,  \
                                int* cell_atoms, const double* coord, const int* type,         \
                                const ET* avg, const ET* std_, const int* atom_off,            \
                                const int* cell_off, const double* box, const int* ncell,      \
                                const int* row_frame, int nframes, int nrows, float rcut,      \
                                float rcut_smth, const int* sec, int nsec, int* status,        \
                                dpb_stream_t stream) {                                         \
    return batch_env<ET>(em, nlist, cw, cell_of, cell_start, cell_atoms, coord, type, avg,     \
                         std_, atom_off, cell_off, box, ncell, row_frame, nframes, nrows, rcut, \
                         rcut_smth, sec, nsec, status, stream);                                \
  }

DPB_BATCH_ENTRIES(f32, float)
DPB_BATCH_ENTRIES(f64, double)

int dpb_batch_force_virial_a(double* force, double* virial, const float* net_deriv,
                             const double* cw, const int* type, const float* std_,
                             const int* nlist, const int* atom_off, const int* cell_off,
                             const double* box, const int* ncell, const int* row_frame,
                             int nframes, int nrows, int nnei, int ntypes, float rcut,
                             float rcut_smth, dpb_stream_t stream) {
  return batch_force<float>(force, virial, net_deriv, cw, type, std_, nlist, atom_off, cell_off,
                            box, ncell, row_frame, nframes, nrows, nnei, ntypes, rcut, rcut_smth,
                            stream);
}

int dpb_batch_force_virial_a_f64(double* force, double* virial, const double* net_deriv,
                                 const double* cw, const int* type, const double* std_,
                                 const int* nlist, const int* atom_off, const int* cell_off,
                                 const double* box, const int* ncell, const int* row_frame,
                                 int nframes, int nrows, int nnei, int ntypes, float rcut,
                                 float rcut_smth, dpb_stream_t stream) {
  return batch_force<double>(force, virial, net_deriv, cw, type, std_, nlist, atom_off, cell_off,
                             box, ncell, row_frame, nframes, nrows, nnei, ntypes, rcut, rcut_smth,
                             stream);
}

int dpb_batch_energy(double* energy, const float* e_rows, const int* drow,
                     const double* e_const, const int* atom_off, int nframes,
                     dpb_stream_t stream) {
  return batch_energy<float>(energy, e_rows, drow, e_const, atom_off, nframes, stream);
}

int dpb_batch_energy_f64(double* energy, const double* e_rows, const int* drow,
                         const double* e_const, const int* atom_off, int nframes,
                         dpb_stream_t stream) {
  return batch_energy<double>(energy, e_rows, drow, e_const, atom_off, nframes, stream);
}

}  // extern "C"
