/* Test infrastructure only: a plain-C restatement of the reference DeePMD-kit
 * CPU algorithms on the se_e2_a path. It is the checker for the CUDA
 * implementation and is never linked into the product.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the reference project root). The restatement is single-threaded and meant
 * for small cases (seconds), not for speed.
 */
#ifndef DP_ORACLE_H
#define DP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* rec_boxt = inverse-transpose of boxt via cofactors / |det|
 * (source/lib/include/SimulationRegion_Impl.h:429-480, region.cc:38-90). */
void orc_rec_boxt(double* rec_boxt, double* volume, const double* boxt);

/* Wrap coordinates into [0,1) in box units (source/lib/src/coord.cc:14-27). */
void orc_normalize_coord(double* coord, int natom, const double* boxt);

/* 23 ints: nat_stt[3], ncell[3], ext_stt[3], ext_end[3], ngcell[3],
 * cell_shift[3], cell_iter[3], loc_cellnum, total_cellnum
 * (source/lib/src/coord.cc:66-107). */
int orc_compute_cell_info(int* cell_info, float rcut, const double* boxt);

/* Ghost-image copy (source/lib/src/coord.cc:29-64 ->
 * source/lib/src/neighbor_list.cc:43-148,730-849). Returns 1 if nall >
 * mem_nall (nall is still reported). */
int orc_copy_coord(double* out_c, int* out_t, int* mapping, int* nall,
                   const double* in_c, const int* in_t, int nloc, int mem_nall,
                   float rcut, const double* boxt);

/* Brute-force neighbor list, ascending j, strict r^2 < rc^2
 * (source/lib/src/neighbor_list.cc:875-928). rowbuf is [nframes*nloc,
 * mem_size]. Returns 1 when a row exceeds mem_size. */
int orc_build_nlist_f64(int* ilist, int* numneigh, int* rowbuf,
                        int* max_list_size, const double* c_cpy, int nloc,
                        int nall, int mem_size, float rcut, int nframes,
                        const int* type);
int orc_build_nlist_f32(int* ilist, int* numneigh, int* rowbuf,
                        int* max_list_size, const float* c_cpy, int nloc,
                        int nall, int mem_size, float rcut, int nframes,
                        const int* type);

/* Per-type sel slots sorted by (type, float r^2, index)
 * (source/lib/src/fmt_nlist.cc:98-143). Returns the overflowed type or -1. */
int orc_format_nlist_i_f64(int* fmt, const double* posi, const int* type,
                           int i_idx, const int* cand, int ncand, float rcut,
                           const int* sec, int nsec);
int orc_format_nlist_i_f32(int* fmt, const float* posi, const int* type,
                           int i_idx, const int* cand, int ncand, float rcut,
                           const int* sec, int nsec);

/* prod_env_mat_a (source/lib/src/prod_env_mat.cc:14-133 with env_mat_a_cpu,
 * source/lib/src/env_mat.cc:123-209). The input list is flat: ilist[inum],
 * numneigh[inum], rowbuf[inum, stride]. */
int orc_prod_env_mat_a_f64(double* em, double* em_deriv, double* rij,
                           int* nlist, const double* coord, const int* type,
                           int inum, const int* ilist, const int* numneigh,
                           const int* rowbuf, int stride, const double* avg,
                           const double* std_, int nloc, int nall, int nframes,
                           float rcut, float rcut_smth, const int* sec,
                           int nsec);
int orc_prod_env_mat_a_f32(float* em, float* em_deriv, float* rij, int* nlist,
                           const float* coord, const int* type, int inum,
                           const int* ilist, const int* numneigh,
                           const int* rowbuf, int stride, const float* avg,
                           const float* std_, int nloc, int nall, int nframes,
                           float rcut, float rcut_smth, const int* sec,
                           int nsec);

/* tabulate_fusion_se_a and its gradients, ndescrpt = 4, sorted padding fold
 * (source/lib/src/tabulate.cc:21-73,116-232,234-341,343-449). */
int orc_tabulate_fusion_se_a_f64(double* out, const double* table,
                                 const double* info, const double* em_x,
                                 const double* em, int nloc, int nnei,
                                 int last_layer_size);
int orc_tabulate_fusion_se_a_grad_f64(double* dy_dem_x, double* dy_dem,
                                      const double* table, const double* info,
                                      const double* em_x, const double* em,
                                      const double* dy, int nloc, int nnei,
                                      int last_layer_size);
int orc_tabulate_fusion_se_a_grad_grad_f64(double* dz_dy, const double* table,
                                           const double* info,
                                           const double* em_x,
                                           const double* em,
                                           const double* dz_dy_dem_x,
                                           const double* dz_dy_dem, int nloc,
                                           int nnei, int last_layer_size);
int orc_tabulate_fusion_se_a_f32(float* out, const float* table,
                                 const float* info, const float* em_x,
                                 const float* em, int nloc, int nnei,
                                 int last_layer_size);
int orc_tabulate_fusion_se_a_grad_f32(float* dy_dem_x, float* dy_dem,
                                      const float* table, const float* info,
                                      const float* em_x, const float* em,
                                      const float* dy, int nloc, int nnei,
                                      int last_layer_size);
int orc_tabulate_fusion_se_a_grad_grad_f32(float* dz_dy, const float* table,
                                           const float* info,
                                           const float* em_x, const float* em,
                                           const float* dz_dy_dem_x,
                                           const float* dz_dy_dem, int nloc,
                                           int nnei, int last_layer_size);

/* prod_force_a (source/lib/src/prod_force.cc:23-87) and prod_virial_a
 * (source/lib/src/prod_virial.cc:22-69). */
int orc_prod_force_a_f64(double* force, const double* net_deriv,
                         const double* env_deriv, const int* nlist, int nloc,
                         int nall, int nnei, int nframes);
int orc_prod_force_a_f32(float* force, const float* net_deriv,
                         const float* env_deriv, const int* nlist, int nloc,
                         int nall, int nnei, int nframes);
int orc_prod_virial_a_f64(double* virial, double* atom_virial,
                          const double* net_deriv, const double* env_deriv,
                          const double* rij, const int* nlist, int nloc,
                          int nall, int nnei);
int orc_prod_virial_a_f32(float* virial, float* atom_virial,
                          const float* net_deriv, const float* env_deriv,
                          const float* rij, const int* nlist, int nloc,
                          int nall, int nnei);

/* prod_force_grad_a (source/lib/src/prod_force_grad.cc:22-70) and
 * prod_virial_grad_a (source/lib/src/prod_virial_grad.cc:21-62). */
int orc_prod_force_grad_a_f64(double* grad_net, const double* grad,
                              const double* env_deriv, const int* nlist,
                              int nloc, int nnei, int nframes);
int orc_prod_force_grad_a_f32(float* grad_net, const float* grad,
                              const float* env_deriv, const int* nlist,
                              int nloc, int nnei, int nframes);
int orc_prod_virial_grad_a_f64(double* grad_net, const double* grad,
                               const double* env_deriv, const double* rij,
                               const int* nlist, int nloc, int nnei);
int orc_prod_virial_grad_a_f32(float* grad_net, const float* grad,
                               const float* env_deriv, const float* rij,
                               const int* nlist, int nloc, int nnei);

#ifdef __cplusplus
}
#endif
#endif
