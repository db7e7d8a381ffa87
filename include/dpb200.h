/* dpb200: C-ABI of the B200 (sm_100a) se_e2_a energy/force/virial kernels.
 *
 * Plain pointers and sizes only. All array arguments are DEVICE pointers
 * unless marked "host". Every call is asynchronous on `stream` (a
 * cudaStream_t; NULL = the legacy default stream) and returns a dpb_status;
 * dpb_last_error() gives the message of the last failure on this thread.
 * Nothing here allocates device memory: the caller passes every output and
 * scratch buffer (sizes from the *_scratch_bytes queries), as the reference's
 * callers do (source/lib/tests/test_env_mat_a.cc:960-964).
 *
 * Device-side conditions that the reference turns into a device trap
 * (source/lib/src/gpu/prod_env_mat.cu:92-99) are written to a caller-owned
 * device status word instead; dpb_status_check() reads it back.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project). Layouts and argument meaning follow the reference.
 */
#ifndef DPB200_H
#define DPB200_H

#ifdef __cplusplus
extern "C" {
#endif

#define DPB_API __attribute__((visibility("default")))

typedef void* dpb_stream_t;

typedef enum {
  DPB_OK = 0,
  /* capacity return code 1 of build_nlist_gpu / copy_coord_gpu
   * (source/lib/include/neighbor_list.h:255-258, coord.h:44-47) */
  DPB_ERR_CAPACITY = 1,
  DPB_ERR_INVALID = 2,        /* std::invalid_argument / deepmd_exception */
  DPB_ERR_CUDA = 3,           /* DPErrcheck failure (gpu_cuda.h:21-57) */
  DPB_ERR_OOM = 4,            /* deepmd_exception_oom (errors.h:20-25) */
  DPB_ERR_NLIST_CAPACITY = 5, /* deepmd_exception_nlist_capacity (errors.h:27-33) */
  DPB_ERR_OVERFLOW = 6        /* sort-key overflow: the reference traps here */
} dpb_status;

DPB_API const char* dpb_last_error(void);
DPB_API int dpb_abi_version(void);

/* Reads the device status word written by the kernels of earlier calls on
 * `stream` (synchronises the stream) and maps it to a dpb_status. */
DPB_API int dpb_status_check(const int* status, dpb_stream_t stream);

/* Sets `bytes` bytes at device address `dst` to zero, ordered on `stream`
 * (a memset node when the stream is being captured into a CUDA graph). Used
 * for the force / virial accumulators at the start of a step. */
DPB_API int dpb_zero_async(void* dst, long long bytes, dpb_stream_t stream);

/* ---------------------------------------------------------- coordinates -- */

/* normalize_coord_gpu (source/lib/include/coord.h:56-59; coord.cu:263-282).
 * boxt: host, 9 values, rows are the box vectors. */
DPB_API int dpb_normalize_coord_f64(double* coord, int natom,
                                    const double* boxt, dpb_stream_t stream);
DPB_API int dpb_normalize_coord_f32(float* coord, int natom, const float* boxt,
                                    dpb_stream_t stream);

/* copy_coord_gpu (source/lib/include/coord.h:72-85; coord.cu:352-414),
 * producing the same extended array as copy_coord_cpu (coord.cc:29-64):
 * locals first, then ghost images cell by cell, ascending atom index within a
 * cell. *nall is host. Returns DPB_ERR_CAPACITY when nall > mem_nall (nall is
 * still reported). Synchronises `stream` to read nall. */
DPB_API long long dpb_copy_coord_scratch_bytes(int nloc, float rcut,
                                               const double* boxt);
DPB_API int dpb_copy_coord_f64(double* out_c, int* out_t, int* mapping,
                               int* nall, void* scratch,
                               long long scratch_bytes, const double* in_c,
                               const int* in_t, int nloc, int mem_nall,
                               float rcut, const double* boxt,
                               dpb_stream_t stream);
DPB_API int dpb_copy_coord_f32(float* out_c, int* out_t, int* mapping,
                               int* nall, void* scratch,
                               long long scratch_bytes, const float* in_c,
                               const int* in_t, int nloc, int mem_nall,
                               float rcut, const float* boxt,
                               dpb_stream_t stream);

/* ---------------------------------------------------------- cell grid ---- */

/* Spatial hash of nall points into cells of edge >= rcut over their bounding
 * box, built on the device (no host round trip). Used by the neighbor search
 * below; it replaces the O(nloc*nall) pair test of build_nlist_gpu
 * (source/lib/src/gpu/neighbor_list.cu:77-113). */
DPB_API long long dpb_cell_grid_bytes(int nall);
/* A grid buffer with room, after the grid, for the atoms' positions, types
 * and indices in cell order (32 bytes per atom). dpb_geometry_cells_f64 given
 * a buffer of this size writes them, and the cell-list env kernels then read
 * the candidates contiguously from them (same results); every other builder
 * marks them absent. */
DPB_API long long dpb_cell_grid_bytes_packed(int nall);
DPB_API int dpb_cell_grid_build_f64(void* grid, long long grid_bytes,
                                    const double* coord, int nall, float rcut,
                                    dpb_stream_t stream);
DPB_API int dpb_cell_grid_build_f32(void* grid, long long grid_bytes,
                                    const float* coord, int nall, float rcut,
                                    dpb_stream_t stream);

/* ------------------------------------------------------- neighbor list -- */

/* build_nlist_gpu (source/lib/include/neighbor_list.h:260-270;
 * gpu/neighbor_list.cu:197-250): every j != i with |r_i - r_j|^2 < rc^2
 * (strict), types < 0 excluded, rows in ascending j, exactly as
 * build_nlist_cpu (neighbor_list.cc:875-928). ilist/numneigh: device [nloc*
 * nframes]; firstneigh: device array of device row pointers, each row holding
 * mem_size ints. *max_list_size is host. Returns DPB_ERR_CAPACITY when a row
 * exceeds mem_size. Synchronises `stream`. */
DPB_API long long dpb_build_nlist_scratch_bytes(int nloc, int nall);
DPB_API int dpb_build_nlist_f64(int* ilist, int* numneigh, int** firstneigh,
                                int* max_list_size, void* scratch,
                                long long scratch_bytes, const double* c_cpy,
                                int nloc, int nall, int mem_size, float rcut,
                                int nframes, const int* type,
                                dpb_stream_t stream);
DPB_API int dpb_build_nlist_f32(int* ilist, int* numneigh, int** firstneigh,
                                int* max_list_size, void* scratch,
                                long long scratch_bytes, const float* c_cpy,
                                int nloc, int nall, int mem_size, float rcut,
                                int nframes, const int* type,
                                dpb_stream_t stream);

/* ----------------------------------------------------- environment matrix -- */

/* prod_env_mat_a_gpu (source/lib/include/prod_env_mat.h:97-116;
 * gpu/prod_env_mat.cu:681-726) from an input list (ilist, numneigh,
 * firstneigh as in build_nlist). The formatted nlist equals
 * format_nlist_i_cpu's (source/lib/src/fmt_nlist.cc:98-143): per-type sel
 * slots sorted by (type, float r^2, index), padding -1. em/em_deriv/rij
 * follow env_mat_a_cpu (source/lib/src/env_mat.cc:123-209) with the
 * per-center-type avg/std normalisation of prod_env_mat.cc:104-124.
 * sec: host, nsec = ntypes + 1 (cumulative sel). status: device int. */
DPB_API int dpb_prod_env_mat_a_f64(double* em, double* em_deriv, double* rij,
                                   int* nlist, const double* coord,
                                   const int* type, int inum, const int* ilist,
                                   const int* numneigh, int* const* firstneigh,
                                   int max_nbor_size, const double* avg,
                                   const double* std_, int nloc, int nall,
                                   int nframes, float rcut, float rcut_smth,
                                   const int* sec, int nsec, int* status,
                                   dpb_stream_t stream);
DPB_API int dpb_prod_env_mat_a_f32(float* em, float* em_deriv, float* rij,
                                   int* nlist, const float* coord,
                                   const int* type, int inum, const int* ilist,
                                   const int* numneigh, int* const* firstneigh,
                                   int max_nbor_size, const float* avg,
                                   const float* std_, int nloc, int nall,
                                   int nframes, float rcut, float rcut_smth,
                                   const int* sec, int nsec, int* status,
                                   dpb_stream_t stream);

/* Mixed precision of the above (no counterpart in the reference): FP64
 * coordinates (the coordinate differences stay FP64), FP32 em / em_deriv /
 * rij; em_deriv and rij may be NULL (not written). For an input list built
 * with a skin (rcut + skin) that is reused over several steps, as an MD
 * engine passes it; the format keeps r <= rcut. */
DPB_API int dpb_prod_env_mat_a_mixed(float* em, float* em_deriv, float* rij,
                                     int* nlist, const double* coord,
                                     const int* type, int inum, const int* ilist,
                                     const int* numneigh, int* const* firstneigh,
                                     int max_nbor_size, const float* avg,
                                     const float* std_, int nloc, int nall,
                                     int nframes, float rcut, float rcut_smth,
                                     const int* sec, int nsec, int* status,
                                     dpb_stream_t stream);

/* prod_force_grad_a_gpu / prod_virial_grad_a_gpu (prod_force_grad.h:26-32,
 * prod_virial_grad.h:26-32): gradients of the force and the virial with
 * respect to net_deriv. grad_net [nframes * nloc, nnei * 4] is fully written
 * (no memset needed); grad is [nframes, nloc, 3] (force) or [9] (virial);
 * neighbor indices >= nloc are taken modulo nloc, as in the reference. */
DPB_API int dpb_prod_force_grad_a_f64(double* grad_net, const double* grad,
                                      const double* env_deriv, const int* nlist, int nloc,
                                      int nnei, int nframes, dpb_stream_t stream);
DPB_API int dpb_prod_force_grad_a_f32(float* grad_net, const float* grad,
                                      const float* env_deriv, const int* nlist, int nloc,
                                      int nnei, int nframes, dpb_stream_t stream);
DPB_API int dpb_prod_virial_grad_a_f64(double* grad_net, const double* grad,
                                       const double* env_deriv, const double* rij,
                                       const int* nlist, int nloc, int nnei,
                                       dpb_stream_t stream);
DPB_API int dpb_prod_virial_grad_a_f32(float* grad_net, const float* grad,
                                       const float* env_deriv, const float* rij,
                                       const int* nlist, int nloc, int nnei,
                                       dpb_stream_t stream);

/* Fused neighbor search + format + environment matrix over a cell grid (one
 * frame): the composition build_nlist_gpu -> prod_env_mat_a_gpu in a single
 * pass, with no intermediate list in HBM. Same outputs as
 * dpb_prod_env_mat_a_*. The _mixed variant takes FP64 coordinates (the
 * coordinate differences stay FP64) and writes FP32 em/em_deriv/rij.
 * em_deriv and rij may be NULL (not written). */
DPB_API int dpb_env_mat_a_cells_f64(double* em, double* em_deriv, double* rij,
                                    int* nlist, const double* coord,
                                    const int* type, const void* grid,
                                    const double* avg, const double* std_,
                                    int nloc, int nall, float rcut,
                                    float rcut_smth, const int* sec, int nsec,
                                    int* status, dpb_stream_t stream);
DPB_API int dpb_env_mat_a_cells_f32(float* em, float* em_deriv, float* rij,
                                    int* nlist, const float* coord,
                                    const int* type, const void* grid,
                                    const float* avg, const float* std_,
                                    int nloc, int nall, float rcut,
                                    float rcut_smth, const int* sec, int nsec,
                                    int* status, dpb_stream_t stream);
DPB_API int dpb_env_mat_a_cells_mixed(float* em, float* em_deriv, float* rij,
                                      int* nlist, const double* coord,
                                      const int* type, const void* grid,
                                      const float* avg, const float* std_,
                                      int nloc, int nall, float rcut,
                                      float rcut_smth, const int* sec,
                                      int nsec, int* status,
                                      dpb_stream_t stream);

/* ------------------------------------------------- compressed embedding -- */

/* tabulate_fusion_se_a_gpu (source/lib/include/tabulate.h:175-186;
 * gpu/tabulate.cu:1219-1264), ndescrpt = 4, se_a (two_embed = NULL), sorted
 * padding fold on. out: [nloc, 4, M]. table: [nspline, 6*M] in the reference
 * layout; table_info: host, 6 values. M = last_layer_size in [1, 1024]. */
DPB_API int dpb_tabulate_fusion_se_a_f64(double* out, const double* table,
                                         const double* table_info,
                                         const double* em_x, const double* em,
                                         int nloc, int nnei,
                                         int last_layer_size,
                                         dpb_stream_t stream);
DPB_API int dpb_tabulate_fusion_se_a_f32(float* out, const float* table,
                                         const float* table_info,
                                         const float* em_x, const float* em,
                                         int nloc, int nnei,
                                         int last_layer_size,
                                         dpb_stream_t stream);

/* tabulate_fusion_se_a_grad_gpu (tabulate.h:188-201; tabulate.cu:1266-1315):
 * dy_dem_x [nloc, nnei], dy_dem [nloc, nnei, 4] from dy [nloc, 4, M]. */
DPB_API int dpb_tabulate_fusion_se_a_grad_f64(
    double* dy_dem_x, double* dy_dem, const double* table,
    const double* table_info, const double* em_x, const double* em,
    const double* dy, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream);
DPB_API int dpb_tabulate_fusion_se_a_grad_f32(
    float* dy_dem_x, float* dy_dem, const float* table,
    const float* table_info, const float* em_x, const float* em,
    const float* dy, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream);

/* tabulate_fusion_se_a_grad_grad_gpu (tabulate.h:203-217;
 * tabulate.cu:1317-1367): dz_dy [nloc, 4, M]. */
DPB_API int dpb_tabulate_fusion_se_a_grad_grad_f64(
    double* dz_dy, const double* table, const double* table_info,
    const double* em_x, const double* em, const double* dz_dy_dem_x,
    const double* dz_dy_dem, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream);
DPB_API int dpb_tabulate_fusion_se_a_grad_grad_f32(
    float* dz_dy, const float* table, const float* table_info,
    const float* em_x, const float* em, const float* dz_dy_dem_x,
    const float* dz_dy_dem, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream);

/* ------------------------------------------------------ force and virial -- */

/* prod_force_a_gpu (source/lib/include/prod_force.h:71-79;
 * gpu/prod_force.cu:104-138): force [nframes, nall, 3] (zeroed here). */
DPB_API int dpb_prod_force_a_f64(double* force, const double* net_deriv,
                                 const double* in_deriv, const int* nlist,
                                 int nloc, int nall, int nnei, int nframes,
                                 dpb_stream_t stream);
DPB_API int dpb_prod_force_a_f32(float* force, const float* net_deriv,
                                 const float* in_deriv, const int* nlist,
                                 int nloc, int nall, int nnei, int nframes,
                                 dpb_stream_t stream);

/* prod_virial_a_gpu (source/lib/include/prod_virial.h:29-38;
 * gpu/prod_virial.cu:106-139): virial [9], atom_virial [nall, 9]. */
DPB_API int dpb_prod_virial_a_f64(double* virial, double* atom_virial,
                                  const double* net_deriv,
                                  const double* env_deriv, const double* rij,
                                  const int* nlist, int nloc, int nall,
                                  int nnei, dpb_stream_t stream);
DPB_API int dpb_prod_virial_a_f32(float* virial, float* atom_virial,
                                  const float* net_deriv,
                                  const float* env_deriv, const float* rij,
                                  const int* nlist, int nloc, int nall,
                                  int nnei, dpb_stream_t stream);

/* ------------------------------------------ fused evaluation pipeline -- */
/* These entry points have no one-to-one counterpart in the reference: they
 * fuse the calls the reference makes in sequence for one se_e2_a energy /
 * force / virial evaluation (source/op/tf/prod_env_mat_multi_device.cc:
 * 2400-2600 for the geometry, deepmd/pt/model/descriptor/se_a.py:742-859 for
 * the descriptor) and are stream-ordered with no host synchronisation, so a
 * whole step can be captured in a CUDA graph. */

/* copy_coord without the host read-back: the extended size is written to the
 * device int *nall_dev; arrays are sized for mem_nall (ghosts beyond it are
 * not written, and *nall_dev > mem_nall tells the caller to grow them). */
DPB_API int dpb_copy_coord_async_f64(double* out_c, int* out_t, int* mapping,
                                     int* nall_dev, void* scratch,
                                     long long scratch_bytes,
                                     const double* in_c, const int* in_t,
                                     int nloc, int mem_nall, float rcut,
                                     const double* boxt, dpb_stream_t stream);
/* Ghost positions between neighbor-list rebuilds (no counterpart in the
 * reference, whose MD engines exchange ghosts themselves): at a rebuild,
 * shift[j] = cext[j] - coord[mapping[j]] for the first *nall_dev (or mem_nall
 * when nall_dev is NULL) extended atoms; at later steps
 * cext[j] = coord[mapping[j]] + shift[j], so every ghost keeps its periodic
 * image while the atoms move. All arrays FP64 [n, 3] on the device. */
DPB_API int dpb_ghost_shift_f64(double* shift, const double* cext, const double* coord,
                                const int* mapping, const int* nall_dev, int mem_nall,
                                dpb_stream_t stream);
DPB_API int dpb_ghost_refresh_f64(double* cext, const double* shift, const double* coord,
                                  const int* mapping, const int* nall_dev, int mem_nall,
                                  dpb_stream_t stream);
/* cell grid over the first *nall_dev of mem_nall points (grid sized by
 * dpb_cell_grid_bytes(mem_nall); pass mem_nall as nall to the env kernels). */
DPB_API int dpb_cell_grid_build_async_f64(void* grid, long long grid_bytes,
                                          const double* coord, int mem_nall,
                                          const int* nall_dev, float rcut,
                                          dpb_stream_t stream);
/* One frame's normalize_coord (coord.cc:14-27) + copy_coord (coord.cc:29-64)
 * + cell grid in one call, replacing dpb_normalize_coord_f64 on a copy of
 * `coord`, dpb_copy_coord_async_f64 and dpb_cell_grid_build_async_f64 (the
 * same cext / atype_ext / mapping / *nall_dev, bit for bit, and the same grid;
 * `coord` is read only). Runs as one cooperative launch with grid-wide
 * barriers when the copy grid's cells fit (nloc_cells + next_cells <= 32766),
 * else as the separate kernels. mem_nall >= nloc; scratch of
 * dpb_geometry_scratch_bytes(nloc, rcut, box); grid of
 * dpb_cell_grid_bytes(mem_nall); status: device int (a barrier that timed
 * out sets a bit there and leaves an empty grid). Knob geometry_fused = 0
 * forces the separate kernels. */
DPB_API long long dpb_geometry_scratch_bytes(int nloc, float rcut, const double* boxt);
DPB_API int dpb_geometry_cells_f64(double* cext, int* atype_ext, int* mapping, int* nall_dev,
                                   void* grid, long long grid_bytes, void* scratch,
                                   long long scratch_bytes, const double* coord,
                                   const int* atype, int nloc, int mem_nall, float rcut,
                                   const double* boxt, int* status, dpb_stream_t stream);

/* Batched frames (no counterpart in the reference, which evaluates frames of
 * different sizes one call at a time): many frames of uneven atom counts in
 * one launch per stage. Rows (atoms) of all frames are concatenated; the
 * frame table is on the device: atom_off [F + 1], cell_off [F + 1] (frame f
 * owns ncell_f + 1 cell_start entries from cell_off[f]), box [F, 3]
 * (orthorhombic edges, each >= rcut), ncell [F, 3] (cells per edge, each >= 1
 * with box / ncell >= rcut; at most 4096 cells and 600,000 atoms per frame),
 * row_frame [N]. Neighbors are periodic images found through the frame's own
 * cell list; nlist holds (frame-local atom * 27 + image code) per slot, with
 * the image code (sx + 1) * 9 + (sy + 1) * 3 + (sz + 1) for shifts in
 * {-1, 0, 1} box edges. Scratch: cw [N, 3] FP64 (wrapped positions),
 * cell_of [N], cell_atoms [N], cell_start [cell_off[F]]. em is FP32 from FP64
 * differences (as dpb_env_mat_a_cells_mixed); sec: host, status: device. */
DPB_API int dpb_batch_env_mat_a_f32(float* em, int* nlist, double* cw, int* cell_of,
                                    int* cell_start, int* cell_atoms, const double* coord,
                                    const int* type, const float* avg, const float* std_,
                                    const int* atom_off, const int* cell_off,
                                    const double* box, const int* ncell, const int* row_frame,
                                    int nframes, int nrows, float rcut, float rcut_smth,
                                    const int* sec, int nsec, int* status,
                                    dpb_stream_t stream);
/* The same in FP64 throughout (env rows from FP64 differences, FP64 avg/std). */
DPB_API int dpb_batch_env_mat_a_f64(double* em, int* nlist, double* cw, int* cell_of,
                                    int* cell_start, int* cell_atoms, const double* coord,
                                    const int* type, const double* avg, const double* std_,
                                    const int* atom_off, const int* cell_off,
                                    const double* box, const int* ncell, const int* row_frame,
                                    int nframes, int nrows, float rcut, float rcut_smth,
                                    const int* sec, int nsec, int* status,
                                    dpb_stream_t stream);
/* Force [N, 3] and per-frame virial [F, 9] (FP64) of the batched frames from
 * net_deriv [N, nnei * 4] (FP32), the wrapped positions cw and the packed
 * nlist of dpb_batch_env_mat_a_f32; the env derivative is recomputed. */
DPB_API int dpb_batch_force_virial_a(double* force, double* virial, const float* net_deriv,
                                     const double* cw, const int* type, const float* std_,
                                     const int* nlist, const int* atom_off,
                                     const int* cell_off, const double* box,
                                     const int* ncell, const int* row_frame, int nframes,
                                     int nrows, int nnei, int ntypes, float rcut,
                                     float rcut_smth, dpb_stream_t stream);
DPB_API int dpb_batch_force_virial_a_f64(double* force, double* virial,
                                         const double* net_deriv, const double* cw,
                                         const int* type, const double* std_,
                                         const int* nlist, const int* atom_off,
                                         const int* cell_off, const double* box,
                                         const int* ncell, const int* row_frame, int nframes,
                                         int nrows, int nnei, int ntypes, float rcut,
                                         float rcut_smth, dpb_stream_t stream);
/* Per-frame energy [F] (FP64): e_const[f] + sum over the frame's rows r of
 * e_rows[drow[r]] (the atomic energies of the fitting, in fitting-row order). */
DPB_API int dpb_batch_energy(double* energy, const float* e_rows, const int* drow,
                             const double* e_const, const int* atom_off, int nframes,
                             dpb_stream_t stream);
DPB_API int dpb_batch_energy_f64(double* energy, const double* e_rows, const int* drow,
                                 const double* e_const, const int* atom_off, int nframes,
                                 dpb_stream_t stream);

/* ------------------------------------- batched step as one persistent launch -- */

/* One fitting GEMM of the step (the arguments of dpb_gemm_tf32x3_f32 that
 * differ per layer). b_hi / b_lo / bias / idt / w are host arrays of ntypes
 * device pointers (bias / idt / w may be NULL); b_lo is required. */
typedef struct {
  const float* A;
  int K;
  const float* const* b_hi;
  const float* const* b_lo;
  int N;
  int mode;
  float* out0;
  float* out1;
  const float* aux0;
  const float* aux1;
  const float* const* bias;
  const float* const* idt;
  const float* const* w;
} dpb_gemm_layer;

/* Everything one batched-frames step touches (device buffers unless noted):
 * the frame table and geometry scratch of dpb_batch_env_mat_a_f32, the
 * descriptor tables and buffers of dpb_se_a_descriptor_{fwd,bwd}[_cubic]_f32
 * (tables: host array of device pointers, table_info: host, 6 per type,
 * table_degree 5 or 3), the six fitting GEMMs in the order layer 1..3
 * forward (epilogues 1, 2, 3) and layer 3..1 backward (4, 5, 0), the
 * per-frame energy constants and the outputs. sync: eight device words (grid
 * barrier and work counters, zeroed by each launch); status: the device
 * status word; pass_ns: NULL, or 12 device words that receive the global
 * timer (ns) at the start and after each of the 11 passes. */
typedef struct {
  int nframes;
  int nrows;
  const int* atom_off;
  const int* cell_off;
  const double* box;
  const int* ncell;
  const int* row_frame;
  const double* coord;
  const int* type;
  double* cw;
  int* cell_of;
  int* cell_start;
  int* cell_atoms;
  const float* avg;
  const float* std_;
  float rcut;
  float rcut_smth;
  const int* sec;
  int nsec;
  float* em;
  int* nlist;
  const float* const* tables;
  const float* table_info;
  int table_degree;
  int M;
  int naxis;
  const int* drow;
  float* xyz;
  float* descrpt;
  float* d_descrpt;
  float* net_deriv;
  const int* type_rows;
  int ntypes;
  dpb_gemm_layer fit[6];
  float* e_rows;
  const double* e_const;
  double* energy;
  double* force;
  double* virial;
  unsigned* sync;
  int* status;
  unsigned long long* pass_ns;
} dpb_bt_step_desc;

/* Checks the description and prepares the launch (tensor maps of the six
 * GEMMs, table descriptors); *plan is freed by dpb_bt_step_destroy. The
 * buffers must stay allocated while the plan is used. */
DPB_API int dpb_bt_step_create(void** plan, const dpb_bt_step_desc* desc);
/* One step: env, descriptor, fitting, descriptor backward, forces, virials
 * and energies of every frame in ONE cooperative launch (one CTA per SM),
 * preceded by a 32-byte memset of the barrier and work counters. */
DPB_API int dpb_bt_step_launch(const void* plan, dpb_stream_t stream);
DPB_API void dpb_bt_step_destroy(void* plan);
/* Layout of the description structs as this library was compiled: which = 0
 * sizeof(dpb_bt_step_desc), 1 offsetof(fit), 2 offsetof(status),
 * 3 sizeof(dpb_gemm_layer), 4 offsetof(dpb_gemm_layer, w); -1 otherwise. */
DPB_API long long dpb_bt_step_desc_layout(int which);

/* FP64 compression table of one se_a embedding net, built on the device
 * (the reference builds it on the host: deepmd/utils/tabulate.py:275-371).
 * xx: device [npoints] grid, steps: device [nspline] interval widths
 * (npoints >= nspline + 1); W[l] / b[l]: host arrays of device pointers to the
 * FP64 layer weights [widths[l], widths[l+1]] (row-major) and biases, widths:
 * host [nlayers + 1] with widths[0] = 1, each width <= 512, nlayers <= 8.
 * table: device [nspline, 6 * M] in the tabulate layout (M = widths[nlayers]).
 * scratch: device, dpb_se_a_build_table_scratch_bytes(npoints, M) bytes. */
DPB_API long long dpb_se_a_build_table_scratch_bytes(int npoints, int M);
DPB_API int dpb_se_a_build_table_f64(double* table, const double* xx, const double* steps,
                                     int npoints, int nspline, const double* const* W,
                                     const double* const* b, const int* widths, int nlayers,
                                     void* scratch, long long scratch_bytes,
                                     dpb_stream_t stream);

/* Repacks one compression table from the tabulate layout [nrow][M][6]
 * (source/lib/src/tabulate.cc:190-197) into the layout the fused descriptor
 * kernels below read, [nrow][6][M] (coefficient-major: a warp's loads of one
 * coefficient of a row are contiguous). out and table must not overlap.
 * No counterpart in the reference (its pipeline calls the tabulate op). */
DPB_API int dpb_se_a_pack_table_f32(float* out, const float* table, int nrow, int M,
                                    dpb_stream_t stream);

/* Compressed descriptor forward over all neighbor types: tables[t] (a HOST
 * array of device pointers, one [nspline_t, 6, M] FP32 table per neighbor
 * type in the dpb_se_a_pack_table_f32 layout), table_info: host [ntypes * 6]. em: [nloc, nnei, 4] FP32 from the env
 * kernels. Writes xyz [nloc, 4, M] (= sum_t G_t^T R_t / nnei) and the
 * descriptor row of atom i at descrpt + descrpt_row[i] * M * axis_neuron.
 * M <= 128, axis_neuron <= 16, ntypes <= 8. */
DPB_API int dpb_se_a_descriptor_fwd_f32(float* xyz, float* descrpt,
                                        const int* descrpt_row, const float* em,
                                        const float* const* tables,
                                        const float* table_info, const int* sec,
                                        int nsec, int nloc, int last_layer_size,
                                        int axis_neuron, dpb_stream_t stream);
/* Adjoint of the above: net_deriv [nloc, nnei * 4] = dE/d(em) from the
 * descriptor gradient d_descrpt (rows at descrpt_row[i]) and xyz. */
DPB_API int dpb_se_a_descriptor_bwd_f32(float* net_deriv, const float* d_descrpt,
                                        const int* descrpt_row, const float* xyz,
                                        const float* em,
                                        const float* const* tables,
                                        const float* table_info, const int* sec,
                                        int nsec, int nloc, int last_layer_size,
                                        int axis_neuron, dpb_stream_t stream);
/* The same two passes on the cubic re-interpolation of the tables (no
 * counterpart in the reference): tables [K + 1, 4, M] FP32 per neighbor type,
 * coefficient-major rows of a cubic Hermite on the fine stride everywhere
 * (the reference's quintic rows give the value and slope at every knot; row K
 * is a guard row [y(max), y'(max), 0, 0]); table_info [lower, max, max,
 * stride, stride, K] per type. Four coefficients per channel instead of six
 * cut the table bytes each neighbor slot gathers by a third; the cubic
 * differs from the quintic by its Hermite remainder, h^4 / 384 times the
 * fourth derivative of the embedding net. */
DPB_API int dpb_se_a_descriptor_fwd_cubic_f32(float* xyz, float* descrpt,
                                              const int* descrpt_row, const float* em,
                                              const float* const* tables,
                                              const float* table_info, const int* sec,
                                              int nsec, int nloc, int last_layer_size,
                                              int axis_neuron, dpb_stream_t stream);
DPB_API int dpb_se_a_descriptor_bwd_cubic_f32(float* net_deriv, const float* d_descrpt,
                                              const int* descrpt_row, const float* xyz,
                                              const float* em, const float* const* tables,
                                              const float* table_info, const int* sec,
                                              int nsec, int nloc, int last_layer_size,
                                              int axis_neuron, dpb_stream_t stream);
/* prod_force_a + prod_virial_a in one pass with FP64 accumulation; ghost
 * forces are added to their owner mapping[j] (force: [nforce, 3], nforce =
 * nloc with a mapping, nall without). atom_virial [nall, 9] may be NULL. */
DPB_API int dpb_force_virial_a_f32(double* force, double* virial,
                                   double* atom_virial, const float* net_deriv,
                                   const float* env_deriv, const float* rij,
                                   const int* nlist, const int* mapping,
                                   int nloc, int nforce, int nall, int nnei,
                                   dpb_stream_t stream);
DPB_API int dpb_force_virial_a_f64(double* force, double* virial,
                                   double* atom_virial, const double* net_deriv,
                                   const double* env_deriv, const double* rij,
                                   const int* nlist, const int* mapping,
                                   int nloc, int nforce, int nall, int nnei,
                                   dpb_stream_t stream);

/* The same force and virial with em_deriv and rij recomputed from the
 * extended coordinates and the neighbor list (so the forward pass need not
 * store them): coord [nall, 3] FP64, type [nall], std_ the env-mat
 * normalisation [ntypes, nnei * 4] used in the forward. _mixed: FP32
 * net_deriv/std with the env-mat derivative in FP32 from FP64 differences. */
DPB_API int dpb_force_virial_a_env_mixed(double* force, double* virial,
                                         const float* net_deriv,
                                         const double* coord, const int* type,
                                         const float* std_, const int* nlist,
                                         const int* mapping, int nloc, int nforce,
                                         int nnei, int ntypes, float rcut,
                                         float rcut_smth, dpb_stream_t stream);
/* As dpb_force_virial_a_env_mixed, adding into force / virial instead of
 * overwriting them (the caller zeroes them, e.g. earlier in the step, so no
 * memset sits between this kernel and the one before it). */
DPB_API int dpb_force_virial_a_env_mixed_acc(double* force, double* virial,
                                             const float* net_deriv, const double* coord,
                                             const int* type, const float* std_,
                                             const int* nlist, const int* mapping, int nloc,
                                             int nforce, int nnei, int ntypes, float rcut,
                                             float rcut_smth, dpb_stream_t stream);
DPB_API int dpb_force_virial_a_env_f64(double* force, double* virial,
                                       const double* net_deriv,
                                       const double* coord, const int* type,
                                       const double* std_, const int* nlist,
                                       const int* mapping, int nloc, int nforce,
                                       int nnei, int ntypes, float rcut,
                                       float rcut_smth, dpb_stream_t stream);

/* FP32-accurate (3xTF32) GEMM on the sm_100a tensor cores for the per-type
 * fitting networks (deepmd/pt/model/task/ener.py; layer math of
 * deepmd/dpmodel/utils/network.py:282-330): C = A B^T with A [M, K] FP32
 * row-major (rows grouped by type, type_rows[t] rows of type t) and, per
 * type, B [N, K] given pre-split into TF32 hi/lo parts (b_hi/b_lo: HOST
 * arrays of device pointers) or, with b_lo = NULL, in FP32 in b_hi and split
 * in the kernel (half the weight bytes read). mode selects the fused epilogue (0 store,
 * 1 tanh(acc+bias), 2 tanh+timestep residual, 3 last layer + energy and its
 * first gradient, 4/5 backward of the residual layers); bias/idt/w are HOST
 * arrays of per-type device vectors [N]. N must be a multiple of 80; K*4
 * and the row pitch must be multiples of 16 bytes. */
DPB_API int dpb_gemm_tf32x3_f32(const float* A, int M, int K,
                                const float* const* b_hi,
                                const float* const* b_lo, int N,
                                const int* type_rows, int ntypes, int mode,
                                float* out0, float* out1, const float* aux0,
                                const float* aux1, const float* const* bias,
                                const float* const* idt, const float* const* w,
                                float* e, int* status, dpb_stream_t stream);
/* energy[0] = e_const + sum of e[0, n) in FP64 (fixed summation order), then
 * e[0, n) = 0: the per-row energies the mode-3 epilogue accumulates, reduced
 * and cleared for the next step's accumulation. work: device buffer of
 * dpb_fit_energy_sum_work_bytes(), zeroed once by the caller (the call leaves
 * it ready for the next one); calls sharing a work buffer must not overlap. */
DPB_API long long dpb_fit_energy_sum_work_bytes(void);
DPB_API int dpb_fit_energy_sum_f32(double* energy, float* e, int n, double e_const, void* work,
                                   dpb_stream_t stream);

/* ------------------------------------------------- training step ----- */
/* Energy, force and virial of the uncompressed se_e2_a model together with
 * the gradient of a loss L(E, F, V) w.r.t. every embedding and fitting
 * weight. The reference gets this gradient from torch autograd with
 * create_graph=True through its PyTorch model (deepmd/pt/model/model/
 * transform_output.py:70-101, deepmd/pt/model/descriptor/se_a.py:742-859,
 * loss deepmd/pt/loss/ener.py:219-340); here it is hand-written: since the
 * force depends on the weights only through g = dE/d(em), dL/dtheta is the
 * energy term plus d/dtheta <u, g> with u = dL/dg, a tangent pass of the
 * network along u followed by one reverse pass over primal and tangent.
 *
 * Shared arguments: nlist / type / drow / geometry as dpb_batch_env_mat_a_*
 * (packed (atom * 27 + image) neighbors, -1 padding; drow [N] = the atom's
 * row in the type-grouped descriptor); W / b: host arrays [ntypes * 3] of
 * device pointers to the embedding layers of neighbor type t, layer l at
 * index t * 3 + l (W row-major [n_in, n_out]); widths: host [1, n1, n2, n3]
 * with 3 <= n1 <= 32, n2 <= 64, n3 <= 128 (a layer that keeps or doubles its
 * width adds the residual); axis <= 32; sec: host section offsets; fold:
 * host [ntypes * ntypes] flags, fold[ti * ntypes + t] = 1 when every padded
 * slot of section t of a type-ti center has the same avg/std (padded slots
 * are then evaluated once with their multiplicity), or NULL.
 *
 * fwd: xyz [N, 4, n3] (atom order), descrpt [N, n3 * axis] (drow order) from
 *      em [N, nnei, 4].
 * bwd: net_deriv = dE/d(em) [N, nnei, 4] (zero on padded slots) from
 *      d_descrpt = dE/dD (drow order); scratch: device [N, 4, n3].
 * tan: tangent of xyz and D along u, u recomputed from the coordinates (cw,
 *      FP64), avg/std [ntypes, nnei * 4], force_bar = dL/dF [N, 3] and
 *      virial_bar = dL/dV [F, 9] (FP64): u = (d em / d r_i) . (Fbar_j -
 *      Fbar_i + Vbar r_ij) per slot.
 * rev: adds to gW / gb (host arrays of device pointers laid out as W / b)
 *      the embedding gradient of J = <Dbar_J, D> + <Ddbar, D'> continued
 *      through xyz, xyz' and the embedding: d_descrpt / d_descrpt_t are the
 *      adjoints of D and D' from the fitting's reverse pass; scratch: device
 *      [2, N, 4, n3]. */
/* float */
DPB_API int dpb_se_a_train_fwd_f32(float* xyz, float* descrpt, const float* em, const int* nlist,
                                   const int* type, const int* drow, const float* const* W,
                                   const float* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, const unsigned char* fold,
                                   dpb_stream_t stream);
DPB_API int dpb_se_a_train_bwd_f32(float* net_deriv, float* scratch, const float* em,
                                   const float* xyz, const float* d_descrpt, const int* nlist,
                                   const int* type, const int* drow, const float* const* W,
                                   const float* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, dpb_stream_t stream);
DPB_API int dpb_se_a_train_tan_f32(float* xyz_t, float* descrpt_t, const float* xyz,
                                   const float* avg, const float* std_, const double* force_bar,
                                   const double* virial_bar, const double* cw, const int* nlist,
                                   const int* type, const int* drow, const int* atom_off,
                                   const double* box, const int* row_frame, int nframes,
                                   const float* const* W, const float* const* b, const int* widths,
                                   const int* sec, int nsec, int nrows, int axis, float rcut,
                                   float rcut_smth, dpb_stream_t stream);
DPB_API int dpb_se_a_train_rev_f32(float* const* gW, float* const* gb, float* scratch,
                                   const float* xyz, const float* xyz_t, const float* d_descrpt,
                                   const float* d_descrpt_t, const float* avg, const float* std_,
                                   const double* force_bar, const double* virial_bar,
                                   const double* cw, const int* nlist, const int* type,
                                   const int* drow, const int* atom_off, const double* box,
                                   const int* row_frame, int nframes, const float* const* W,
                                   const float* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, const unsigned char* fold,
                                   float rcut, float rcut_smth, dpb_stream_t stream);
/* fitting layer (deepmd/dpmodel/utils/network.py:282-330) around a library GEMM:
 * act: Y holds Z = H_in W + b on entry; Y = tanh(Z), H = res(H_in) + d * Y (d may be
 * NULL); tan: Hd = res(Hd_in) + d (1 - Y^2) Zd; bwd: Zb = G d (1 - Y^2); rev: reverse
 * over tangent, Zbd = d Ad q, Zb = (d A - 2 Y Zd d Ad) q with q = 1 - Y^2, gb +=
 * column sums of Zb, gd += column sums of A Y + Ad q Zd (gd may be NULL); res_adj:
 * out += adjoint of the residual; out: e = H . Wo + bo + ebias; out_adj: A = lam Wo,
 * Ad = Wo, gWo += sum lam H + Hd, gbo += sum lam (lam NULL = 1; Ad, Hd, gWo/gbo may be
 * NULL); lam: lam[drow[r]] = gE[row_frame[r]]. */
DPB_API int dpb_fit_act_f32(float* Y, float* H, const float* Hin, const float* d, int n, int w_out,
                            int w_in, dpb_stream_t stream);
DPB_API int dpb_fit_tan_f32(float* Hd, const float* Zd, const float* Hdin, const float* Y,
                            const float* d, int n, int w_out, int w_in, dpb_stream_t stream);
DPB_API int dpb_fit_bwd_f32(float* Zb, const float* G, const float* Y, const float* d, int n, int w,
                            dpb_stream_t stream);
DPB_API int dpb_fit_rev_f32(float* Zb, float* Zbd, float* gb, float* gd, const float* A,
                            const float* Ad, const float* Y, const float* Zd, const float* d, int n,
                            int w, dpb_stream_t stream);
DPB_API int dpb_fit_res_adj_f32(float* out, const float* G, int n, int w_out, int w_in,
                                dpb_stream_t stream);
DPB_API int dpb_fit_out_f32(float* e, const float* H, const float* Wo, const float* bo,
                            double ebias, int n, int w, dpb_stream_t stream);
DPB_API int dpb_fit_out_adj_f32(float* A, float* Ad, float* gWo, float* gbo, const float* H,
                                const float* Hd, const float* Wo, const float* lam, int n, int w,
                                dpb_stream_t stream);
DPB_API int dpb_train_lam_f32(float* lam, const double* gE, const int* drow, const int* row_frame,
                              int n, dpb_stream_t stream);
/* Adam step as torch.optim.Adam (no weight decay, no amsgrad); hp: device
 * {lr, 1 - beta1^step, sqrt(1 - beta2^step)} (read at run time, so a captured step
 * follows the schedule). */
DPB_API int dpb_adam_f32(float* p, const float* g, float* m, float* v, long long n,
                         const double* hp, double beta1, double beta2, double eps,
                         dpb_stream_t stream);

/* double */
DPB_API int dpb_se_a_train_fwd_f64(double* xyz, double* descrpt, const double* em, const int* nlist,
                                   const int* type, const int* drow, const double* const* W,
                                   const double* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, const unsigned char* fold,
                                   dpb_stream_t stream);
DPB_API int dpb_se_a_train_bwd_f64(double* net_deriv, double* scratch, const double* em,
                                   const double* xyz, const double* d_descrpt, const int* nlist,
                                   const int* type, const int* drow, const double* const* W,
                                   const double* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, dpb_stream_t stream);
DPB_API int dpb_se_a_train_tan_f64(double* xyz_t, double* descrpt_t, const double* xyz,
                                   const double* avg, const double* std_, const double* force_bar,
                                   const double* virial_bar, const double* cw, const int* nlist,
                                   const int* type, const int* drow, const int* atom_off,
                                   const double* box, const int* row_frame, int nframes,
                                   const double* const* W, const double* const* b,
                                   const int* widths, const int* sec, int nsec, int nrows, int axis,
                                   float rcut, float rcut_smth, dpb_stream_t stream);
DPB_API int dpb_se_a_train_rev_f64(double* const* gW, double* const* gb, double* scratch,
                                   const double* xyz, const double* xyz_t, const double* d_descrpt,
                                   const double* d_descrpt_t, const double* avg, const double* std_,
                                   const double* force_bar, const double* virial_bar,
                                   const double* cw, const int* nlist, const int* type,
                                   const int* drow, const int* atom_off, const double* box,
                                   const int* row_frame, int nframes, const double* const* W,
                                   const double* const* b, const int* widths, const int* sec,
                                   int nsec, int nrows, int axis, const unsigned char* fold,
                                   float rcut, float rcut_smth, dpb_stream_t stream);
DPB_API int dpb_fit_act_f64(double* Y, double* H, const double* Hin, const double* d, int n,
                            int w_out, int w_in, dpb_stream_t stream);
DPB_API int dpb_fit_tan_f64(double* Hd, const double* Zd, const double* Hdin, const double* Y,
                            const double* d, int n, int w_out, int w_in, dpb_stream_t stream);
DPB_API int dpb_fit_bwd_f64(double* Zb, const double* G, const double* Y, const double* d, int n,
                            int w, dpb_stream_t stream);
DPB_API int dpb_fit_rev_f64(double* Zb, double* Zbd, double* gb, double* gd, const double* A,
                            const double* Ad, const double* Y, const double* Zd, const double* d,
                            int n, int w, dpb_stream_t stream);
DPB_API int dpb_fit_res_adj_f64(double* out, const double* G, int n, int w_out, int w_in,
                                dpb_stream_t stream);
DPB_API int dpb_fit_out_f64(double* e, const double* H, const double* Wo, const double* bo,
                            double ebias, int n, int w, dpb_stream_t stream);
DPB_API int dpb_fit_out_adj_f64(double* A, double* Ad, double* gWo, double* gbo, const double* H,
                                const double* Hd, const double* Wo, const double* lam, int n, int w,
                                dpb_stream_t stream);
DPB_API int dpb_train_lam_f64(double* lam, const double* gE, const int* drow, const int* row_frame,
                              int n, dpb_stream_t stream);
DPB_API int dpb_adam_f64(double* p, const double* g, double* m, double* v, long long n,
                         const double* hp, double beta1, double beta2, double eps,
                         dpb_stream_t stream);


/* ------------------------------------------------- tile-shape knobs ---- */
/* No counterpart in the reference (its kernels have fixed launch shapes).
 * Process-wide knobs read when a launcher runs (a captured CUDA graph keeps
 * the shapes it was captured with): desc_atoms_per_cta {2, 4, 8} (fused
 * descriptor kernels), desc_coef_l1 {0, 1, 2, 3, 4} (cache policy of their
 * table loads: default, L1 no_allocate, L1 evict_first, L1 evict_last, L1 and L2
 * evict_last), fit_n_tile {80, 160, 240} (widest fitting GEMM N tile; a
 * width is used where it divides N, 240 only for K <= 512), fit_split_b {0, 1} (weights pre-split or split in the
 * GEMM), batch_atoms_per_cta {2, 4, 8} (batched env / force),
 * train_rows_per_group {4, 8} (FP32 training kernels, standard net),
 * train_warps_per_cta {1, 2, 4, 8}, geometry_fused {0, 1} (one cooperative
 * geometry launch or the separate kernels). The autotuner (autotune.py) times the
 * options on the caller's own step and sets the fastest. */
DPB_API int dpb_tune_count(void);
DPB_API const char* dpb_tune_name(int index);
DPB_API int dpb_tune_get(const char* name);
DPB_API int dpb_tune_options(const char* name, int* out, int capacity);
DPB_API int dpb_tune_set(const char* name, int value);

/* FP64 GEMM of the fitting network (FP64 plain path, FP64 training):
 * C[M, N] = op(A) op(B) (+ bias[N]) (+ C when accumulate), row-major, op(X)
 * = X^T when trans_* is set; lda / ldb / ldc are the row strides of the
 * stored A, B, C. The layer algebra of deepmd/dpmodel/utils/network.py:
 * 282-330 (y = x W + b, g_in = g W^T, gW += x^T g). */
DPB_API int dpb_gemm_f64(double* C, const double* A, const double* B, const double* bias,
                         int M, int N, int K, int lda, int ldb, int ldc, int trans_a,
                         int trans_b, int accumulate, dpb_stream_t stream);

/* The same in FP32 (the FP32 training step's layers whose widths the
 * tensor-core GEMM does not take). */
DPB_API int dpb_gemm_f32(float* C, const float* A, const float* B, const float* bias, int M,
                         int N, int K, int lda, int ldb, int ldc, int trans_a, int trans_b,
                         int accumulate, dpb_stream_t stream);
/* out[c * ld_out + r] = in[r * ld_in + c] (r < rows, c < cols) and zero for
 * rows <= r < out_rows: the transposed operands of the tensor-core GEMM in
 * the training step (weights W^T for x W; activations and adjoints for the
 * weight gradient x^T g, concatenated along K). */
DPB_API int dpb_transpose_f32(float* out, const float* in, int rows, int cols, int ld_in,
                              int ld_out, int out_rows, dpb_stream_t stream);

/* ----------------------------------------- engine-facing list helpers ---- */
/* copy_coord_gpu (source/lib/include/coord.h:72-85) takes the cell
 * decomposition its caller computed with compute_cell_info
 * (source/lib/src/coord.cc:69-108) instead of rcut: `cell_info` is that
 * 23-int host array (ncell at [3..5], ngcell at [12..14], loc_cellnum at
 * [21], total_cellnum at [22]); `boxt` the host box. Ghosts come out in the
 * order of copy_coord_cpu. Returns DPB_ERR_CAPACITY with *nall set when nall
 * exceeds mem_nall. Synchronises `stream` (nall is read back). */
DPB_API long long dpb_copy_coord_cells_scratch_bytes(int nloc, const int* cell_info);
DPB_API int dpb_copy_coord_cells_f64(double* out_c, int* out_t, int* mapping, int* nall,
                                     void* scratch, long long scratch_bytes,
                                     const double* in_c, const int* in_t, int nloc,
                                     int mem_nall, const int* cell_info, const double* boxt,
                                     dpb_stream_t stream);
DPB_API int dpb_copy_coord_cells_f32(float* out_c, int* out_t, int* mapping, int* nall,
                                     void* scratch, long long scratch_bytes,
                                     const float* in_c, const int* in_t, int nloc,
                                     int mem_nall, const int* cell_info, const float* boxt,
                                     dpb_stream_t stream);
/* use_nlist_map (source/lib/include/neighbor_list.h:225-228): every entry of
 * nlist [nloc, nnei] that is not -1 replaced by nlist_map[entry]. */
DPB_API int dpb_use_nlist_map(int* nlist, const int* nlist_map, int nloc, int nnei,
                              dpb_stream_t stream);
/* convert_nlist_gpu_device (source/lib/include/neighbor_list.h:201-218): a
 * host neighbor list (ilist, numneigh, firstneigh rows) into caller device
 * arrays: d_ilist / d_numneigh [inum], d_firstneigh [inum] pointers into
 * d_rows [inum, width] (only the first numneigh[ii] entries of each row are
 * written). One packed host-to-device copy plus one scatter kernel, using
 * d_scratch (dpb_nlist_rows_scratch_bytes); a row longer than width gives
 * DPB_ERR_NLIST_CAPACITY before any device work. Synchronises `stream`. */
DPB_API long long dpb_nlist_rows_scratch_bytes(const int* numneigh, int inum);
DPB_API int dpb_nlist_rows_to_device(int* d_ilist, int* d_numneigh, int** d_firstneigh,
                                     int* d_rows, int width, const int* ilist,
                                     const int* numneigh, const int* const* firstneigh,
                                     int inum, void* d_scratch, long long scratch_bytes,
                                     dpb_stream_t stream);

/* ------------------------------------------- allocation-free variant ---- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc,
 * e.g. an MD engine's force callback that runs inside the engine's own
 * device-memory pool and may not allocate during a step: the same neighbor
 * list as dpb_build_nlist_f64 (same arguments and results) without the
 * caller scratch. Its working memory is a 4 MiB file-scope device array in
 * the library (held by every GPU that loads it until exit), which limits nall
 * to what fits (dpb_cell_grid_bytes(nall) + 256 <= 4 MiB, i.e. nall <= 209,670
 * extended atoms); larger sizes are rejected with DPB_ERR_INVALID. The first
 * call on a device looks up the array's device address and caches it for the
 * life of the device's context (call it before any stream capture; after a
 * cudaDeviceReset do not call it on that device again). All calls share the
 * array: calls that overlap on the same GPU race. */
DPB_API long long dpb_build_nlist_noalloc_max_bytes(void);
DPB_API int dpb_build_nlist_noalloc_f64(int* ilist, int* numneigh,
                                        int** firstneigh, int* max_list_size,
                                        const double* c_cpy, int nloc, int nall,
                                        int mem_size, float rcut, int nframes,
                                        const int* type, dpb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* DPB200_H */
