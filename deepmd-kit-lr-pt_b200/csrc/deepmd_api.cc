// deepmd:: C++ drop-in over the C-ABI (see include/deepmd_b200/deepmd_api.h).
//
// Same function templates and explicit float/double instantiations as the
// reference (source/lib/src/gpu/{neighbor_list,prod_env_mat,tabulate,
// prod_force,prod_virial}.cu), hence the same mangled symbols. Calls run on
// the legacy default stream and end with a device synchronisation, as the
// reference's do; failures throw the reference's exception types.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/dpb200.h"
#include "../../include/deepmd_b200/deepmd_api.h"

namespace {

void raise(int code, const char* what) {
  if (code == DPB_OK) return;
  std::string msg = std::string(what) + ": " + dpb_last_error();
  if (code == DPB_ERR_OOM) throw deepmd::deepmd_exception_oom(msg);
  if (code == DPB_ERR_NLIST_CAPACITY) throw deepmd::deepmd_exception_nlist_capacity(msg);
  throw deepmd::deepmd_exception(msg);
}

void sync(const char* what) {
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess)
    throw deepmd::deepmd_exception(std::string(what) + ": " + cudaGetErrorString(e));
}

void se_a_only(const void* two_embed, bool is_sorted, int ndescrpt, const char* what) {
  if (two_embed != nullptr)
    throw deepmd::deepmd_exception(std::string(what) +
                                   ": two_embed (se_atten) is not supported by this library");
  if (!is_sorted)
    throw deepmd::deepmd_exception(std::string(what) + ": only the sorted-padding mode is supported");
  if (ndescrpt != 4)
    throw deepmd::deepmd_exception(std::string(what) +
                                   ": the environment basis dimension must be 4 for se_a, got " +
                                   std::to_string(ndescrpt));
}

// overloads selecting the C-ABI precision
int c_tab(float* o, const float* t, const float* i, const float* x, const float* e, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_f32(o, t, i, x, e, a, b, m, nullptr);
}
int c_tab(double* o, const double* t, const double* i, const double* x, const double* e, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_f64(o, t, i, x, e, a, b, m, nullptr);
}
int c_tab_g(float* dx, float* de, const float* t, const float* i, const float* x, const float* e,
            const float* dy, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_grad_f32(dx, de, t, i, x, e, dy, a, b, m, nullptr);
}
int c_tab_g(double* dx, double* de, const double* t, const double* i, const double* x,
            const double* e, const double* dy, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_grad_f64(dx, de, t, i, x, e, dy, a, b, m, nullptr);
}
int c_tab_gg(float* o, const float* t, const float* i, const float* x, const float* e,
             const float* zx, const float* ze, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_grad_grad_f32(o, t, i, x, e, zx, ze, a, b, m, nullptr);
}
int c_tab_gg(double* o, const double* t, const double* i, const double* x, const double* e,
             const double* zx, const double* ze, int a, int b, int m) {
  return dpb_tabulate_fusion_se_a_grad_grad_f64(o, t, i, x, e, zx, ze, a, b, m, nullptr);
}
int c_force(float* f, const float* nd, const float* ed, const int* nl, int a, int b, int c, int d) {
  return dpb_prod_force_a_f32(f, nd, ed, nl, a, b, c, d, nullptr);
}
int c_force(double* f, const double* nd, const double* ed, const int* nl, int a, int b, int c, int d) {
  return dpb_prod_force_a_f64(f, nd, ed, nl, a, b, c, d, nullptr);
}
int c_virial(float* v, float* av, const float* nd, const float* ed, const float* r, const int* nl,
             int a, int b, int c) {
  return dpb_prod_virial_a_f32(v, av, nd, ed, r, nl, a, b, c, nullptr);
}
int c_virial(double* v, double* av, const double* nd, const double* ed, const double* r,
             const int* nl, int a, int b, int c) {
  return dpb_prod_virial_a_f64(v, av, nd, ed, r, nl, a, b, c, nullptr);
}
int c_force_grad(float* g, const float* gr, const float* ed, const int* nl, int a, int b,
                 int c) {
  return dpb_prod_force_grad_a_f32(g, gr, ed, nl, a, b, c, nullptr);
}
int c_force_grad(double* g, const double* gr, const double* ed, const int* nl, int a, int b,
                 int c) {
  return dpb_prod_force_grad_a_f64(g, gr, ed, nl, a, b, c, nullptr);
}
int c_virial_grad(float* g, const float* gr, const float* ed, const float* r, const int* nl,
                  int a, int b) {
  return dpb_prod_virial_grad_a_f32(g, gr, ed, r, nl, a, b, nullptr);
}
int c_virial_grad(double* g, const double* gr, const double* ed, const double* r,
                  const int* nl, int a, int b) {
  return dpb_prod_virial_grad_a_f64(g, gr, ed, r, nl, a, b, nullptr);
}
int c_env(float* em, float* ed, float* r, int* nl, const float* c, const int* t, int inum,
          const int* il, const int* nn, int* const* fn, int mx, const float* av, const float* sd,
          int nloc, int nall, int nf, float rc, float rs, const int* sec, int nsec, int* st) {
  return dpb_prod_env_mat_a_f32(em, ed, r, nl, c, t, inum, il, nn, fn, mx, av, sd, nloc, nall, nf,
                                rc, rs, sec, nsec, st, nullptr);
}
int c_env(double* em, double* ed, double* r, int* nl, const double* c, const int* t, int inum,
          const int* il, const int* nn, int* const* fn, int mx, const double* av,
          const double* sd, int nloc, int nall, int nf, float rc, float rs, const int* sec,
          int nsec, int* st) {
  return dpb_prod_env_mat_a_f64(em, ed, r, nl, c, t, inum, il, nn, fn, mx, av, sd, nloc, nall,
                                nf, rc, rs, sec, nsec, st, nullptr);
}
int c_nlist(int* il, int* nn, int** fn, int* mx, void* s, long long sb, const float* c, int nloc,
            int nall, int mem, float rc, int nf, const int* t) {
  return dpb_build_nlist_f32(il, nn, fn, mx, s, sb, c, nloc, nall, mem, rc, nf, t, nullptr);
}
int c_nlist(int* il, int* nn, int** fn, int* mx, void* s, long long sb, const double* c, int nloc,
            int nall, int mem, float rc, int nf, const int* t) {
  return dpb_build_nlist_f64(il, nn, fn, mx, s, sb, c, nloc, nall, mem, rc, nf, t, nullptr);
}

int c_normalize(float* c, int n, const float* b) {
  return dpb_normalize_coord_f32(c, n, b, nullptr);
}
int c_normalize(double* c, int n, const double* b) {
  return dpb_normalize_coord_f64(c, n, b, nullptr);
}
int c_copy_cells(float* oc, int* ot, int* m, int* nall, void* s, long long sb, const float* ic,
                 const int* it, int nloc, int mem, const int* ci, const float* b) {
  return dpb_copy_coord_cells_f32(oc, ot, m, nall, s, sb, ic, it, nloc, mem, ci, b, nullptr);
}
int c_copy_cells(double* oc, int* ot, int* m, int* nall, void* s, long long sb, const double* ic,
                 const int* it, int nloc, int mem, const int* ci, const double* b) {
  return dpb_copy_coord_cells_f64(oc, ot, m, nall, s, sb, ic, it, nloc, mem, ci, b, nullptr);
}

template <typename T>
void d2h(T* dst, const T* src, size_t n, const char* what) {
  cudaError_t e = cudaMemcpy(dst, src, sizeof(T) * n, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess)
    throw deepmd::deepmd_exception(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
void dev_alloc(T*& p, size_t n, const char* what) {
  p = nullptr;
  cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * (n > 0 ? n : 1));
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    throw deepmd::deepmd_exception_oom(std::string(what) + ": cudaMalloc failed");
  }
  if (e != cudaSuccess)
    throw deepmd::deepmd_exception(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

namespace deepmd {

template <typename FPTYPE>
void normalize_coord_gpu(FPTYPE* coord, const int natom, const Region<FPTYPE>& region) {
  sync("normalize_coord_gpu");
  FPTYPE box[9];
  d2h(box, region.boxt, 9, "normalize_coord_gpu");
  raise(c_normalize(coord, natom, box), "normalize_coord_gpu");
  sync("normalize_coord_gpu");
}

template <typename FPTYPE>
int copy_coord_gpu(FPTYPE* out_c, int* out_t, int* mapping, int* nall, int* int_data,
                   const FPTYPE* in_c, const int* in_t, const int& nloc, const int& mem_nall,
                   const int& loc_cellnum, const int& total_cellnum, const int* cell_info,
                   const Region<FPTYPE>& region) {
  sync("copy_coord_gpu");
  int ci[23];
  FPTYPE box[9];
  d2h(ci, cell_info, 23, "copy_coord_gpu");
  d2h(box, region.boxt, 9, "copy_coord_gpu");
  if (ci[21] != loc_cellnum || ci[22] != total_cellnum)
    throw deepmd_exception("copy_coord_gpu: loc_cellnum / total_cellnum disagree with cell_info");
  // the int_data the reference's callers allocate
  // (op/tf/prod_env_mat_multi_device.cc:2428-2430, less the 23 cell_info ints)
  const long long have =
      (4LL * nloc + 2LL * loc_cellnum + 7LL * total_cellnum + 2) * (long long)sizeof(int);
  int code = c_copy_cells(out_c, out_t, mapping, nall, int_data, have, in_c, in_t, nloc,
                          mem_nall, ci, box);
  if (code == DPB_ERR_CAPACITY) return 1;
  raise(code, "copy_coord_gpu");
  sync("copy_coord_gpu");
  return 0;
}

void convert_nlist_gpu_device(InputNlist& gpu_nlist, InputNlist& cpu_nlist, int*& gpu_memory,
                              const int& max_nbor_size) {
  // every row is checked before gpu_nlist is touched (neighbor_list.cc:993-1016)
  for (int ii = 0; ii < cpu_nlist.inum; ++ii) {
    if (cpu_nlist.numneigh[ii] > max_nbor_size)
      throw deepmd_exception_nlist_capacity(
          "Neighbor list row " + std::to_string(ii) + " contains " +
          std::to_string(cpu_nlist.numneigh[ii]) +
          " neighbors, exceeding the allocated GPU row capacity " +
          std::to_string(max_nbor_size));
  }
  const int inum = cpu_nlist.inum;
  gpu_nlist.inum = inum;
  dev_alloc(gpu_nlist.ilist, inum, "convert_nlist_gpu_device");
  dev_alloc(gpu_nlist.numneigh, inum, "convert_nlist_gpu_device");
  dev_alloc(gpu_nlist.firstneigh, inum, "convert_nlist_gpu_device");
  const long long sb = dpb_nlist_rows_scratch_bytes(cpu_nlist.numneigh, inum);
  unsigned char* scratch = nullptr;
  dev_alloc(scratch, (size_t)sb, "convert_nlist_gpu_device");
  int code = dpb_nlist_rows_to_device(gpu_nlist.ilist, gpu_nlist.numneigh, gpu_nlist.firstneigh,
                                      gpu_memory, max_nbor_size, cpu_nlist.ilist,
                                      cpu_nlist.numneigh, cpu_nlist.firstneigh, inum, scratch,
                                      sb, nullptr);
  cudaFree(scratch);
  raise(code, "convert_nlist_gpu_device");
  sync("convert_nlist_gpu_device");
}

void free_nlist_gpu_device(InputNlist& gpu_nlist) {
  for (void* p : {(void*)gpu_nlist.ilist, (void*)gpu_nlist.numneigh,
                  (void*)gpu_nlist.firstneigh}) {
    if (p != nullptr) {
      cudaError_t e = cudaFree(p);
      if (e != cudaSuccess)
        throw deepmd_exception(std::string("free_nlist_gpu_device: ") + cudaGetErrorString(e));
    }
  }
  gpu_nlist.ilist = nullptr;
  gpu_nlist.numneigh = nullptr;
  gpu_nlist.firstneigh = nullptr;
}

void use_nlist_map(int* nlist, const int* nlist_map, const int nloc, const int nnei) {
  sync("use_nlist_map");
  raise(dpb_use_nlist_map(nlist, nlist_map, nloc, nnei, nullptr), "use_nlist_map");
  sync("use_nlist_map");
}

template <typename FPTYPE>
int build_nlist_gpu(InputNlist& nlist, int* max_list_size, int* nlist_data,
                    const FPTYPE* c_cpy, const int& nloc, const int& nall,
                    const int& mem_size, const float& rcut, const int& nframes,
                    const int* type) {
  // neighbor_list.cu:207-210: the row buffers must be able to hold nall
  if (mem_size < nall) return 1;
  // nlist_data: >= 2 * nframes * nloc * mem_size ints of caller scratch
  // (neighbor_list.h:236-238); the cell grid needs far less.
  long long have = 2LL * nframes * nloc * mem_size * (long long)sizeof(int);
  long long need = dpb_build_nlist_scratch_bytes(nloc, nall);
  if (have < need)
    throw deepmd_exception("build_nlist_gpu: nlist_data is smaller than " +
                           std::to_string(need) + " bytes");
  nlist.inum = nframes * nloc;
  int code = c_nlist(nlist.ilist, nlist.numneigh, nlist.firstneigh, max_list_size, nlist_data,
                     have, c_cpy, nloc, nall, mem_size, rcut, nframes, type);
  if (code == DPB_ERR_CAPACITY) return 1;
  raise(code, "build_nlist_gpu");
  sync("build_nlist_gpu");
  return 0;
}

template <typename FPTYPE>
void prod_env_mat_a_gpu(FPTYPE* em, FPTYPE* em_deriv, FPTYPE* rij, int* nlist,
                        const FPTYPE* coord, const int* type,
                        const InputNlist& gpu_inlist, int* array_int,
                        unsigned long long* array_longlong, const int max_nbor_size,
                        const FPTYPE* avg, const FPTYPE* std, const int nloc,
                        const int nall, const int nframes, const float rcut,
                        const float rcut_smth, const std::vector<int> sec,
                        const int* f_type) {
  (void)array_longlong;
  if (f_type != nullptr && f_type != type)
    throw deepmd_exception("prod_env_mat_a_gpu: a separate f_type is not supported");
  if (cudaMemsetAsync(array_int, 0, sizeof(int), nullptr) != cudaSuccess)
    throw deepmd_exception("prod_env_mat_a_gpu: cannot reset the status word");
  raise(c_env(em, em_deriv, rij, nlist, coord, type, gpu_inlist.inum, gpu_inlist.ilist,
              gpu_inlist.numneigh, gpu_inlist.firstneigh, max_nbor_size, avg, std, nloc, nall,
              nframes, rcut, rcut_smth, sec.data(), (int)sec.size(), array_int),
        "prod_env_mat_a_gpu");
  raise(dpb_status_check(array_int, nullptr), "prod_env_mat_a_gpu");
  sync("prod_env_mat_a_gpu");
}

template <typename FPTYPE>
void tabulate_fusion_se_a_gpu(FPTYPE* out, const FPTYPE* table, const FPTYPE* table_info,
                              const FPTYPE* em_x, const FPTYPE* em, const FPTYPE* two_embed,
                              const int nloc, const int nnei, const int last_layer_size,
                              const bool is_sorted, const int ndescrpt) {
  se_a_only(two_embed, is_sorted, ndescrpt, "tabulate_fusion_se_a_gpu");
  raise(c_tab(out, table, table_info, em_x, em, nloc, nnei, last_layer_size),
        "tabulate_fusion_se_a_gpu");
  sync("tabulate_fusion_se_a_gpu");
}

template <typename FPTYPE>
void tabulate_fusion_se_a_grad_gpu(FPTYPE* dy_dem_x, FPTYPE* dy_dem, FPTYPE* dy_dtwo,
                                   const FPTYPE* table, const FPTYPE* table_info,
                                   const FPTYPE* em_x, const FPTYPE* em,
                                   const FPTYPE* two_embed, const FPTYPE* dy, const int nloc,
                                   const int nnei, const int last_layer_size,
                                   const bool is_sorted, const int ndescrpt) {
  (void)dy_dtwo;
  se_a_only(two_embed, is_sorted, ndescrpt, "tabulate_fusion_se_a_grad_gpu");
  raise(c_tab_g(dy_dem_x, dy_dem, table, table_info, em_x, em, dy, nloc, nnei, last_layer_size),
        "tabulate_fusion_se_a_grad_gpu");
  sync("tabulate_fusion_se_a_grad_gpu");
}

template <typename FPTYPE>
void tabulate_fusion_se_a_grad_grad_gpu(FPTYPE* dz_dy, const FPTYPE* table,
                                        const FPTYPE* table_info, const FPTYPE* em_x,
                                        const FPTYPE* em, const FPTYPE* two_embed,
                                        const FPTYPE* dz_dy_dem_x, const FPTYPE* dz_dy_dem,
                                        const FPTYPE* dz_dy_dtwo, const int nloc,
                                        const int nnei, const int last_layer_size,
                                        const bool is_sorted, const int ndescrpt) {
  (void)dz_dy_dtwo;
  se_a_only(two_embed, is_sorted, ndescrpt, "tabulate_fusion_se_a_grad_grad_gpu");
  raise(c_tab_gg(dz_dy, table, table_info, em_x, em, dz_dy_dem_x, dz_dy_dem, nloc, nnei,
                 last_layer_size),
        "tabulate_fusion_se_a_grad_grad_gpu");
  sync("tabulate_fusion_se_a_grad_grad_gpu");
}

template <typename FPTYPE>
void prod_force_a_gpu(FPTYPE* force, const FPTYPE* net_deriv, const FPTYPE* in_deriv,
                      const int* nlist, const int nloc, const int nall, const int nnei,
                      const int nframes) {
  raise(c_force(force, net_deriv, in_deriv, nlist, nloc, nall, nnei, nframes), "prod_force_a_gpu");
  sync("prod_force_a_gpu");
}

template <typename FPTYPE>
void prod_virial_a_gpu(FPTYPE* virial, FPTYPE* atom_virial, const FPTYPE* net_deriv,
                       const FPTYPE* env_deriv, const FPTYPE* rij, const int* nlist,
                       const int nloc, const int nall, const int nnei) {
  raise(c_virial(virial, atom_virial, net_deriv, env_deriv, rij, nlist, nloc, nall, nnei),
        "prod_virial_a_gpu");
  sync("prod_virial_a_gpu");
}

template <typename FPTYPE>
void prod_force_grad_a_gpu(FPTYPE* grad_net, const FPTYPE* grad, const FPTYPE* env_deriv,
                           const int* nlist, const int nloc, const int nnei,
                           const int nframes) {
  raise(c_force_grad(grad_net, grad, env_deriv, nlist, nloc, nnei, nframes),
        "prod_force_grad_a_gpu");
  sync("prod_force_grad_a_gpu");
}

template <typename FPTYPE>
void prod_virial_grad_a_gpu(FPTYPE* grad_net, const FPTYPE* grad, const FPTYPE* env_deriv,
                            const FPTYPE* rij, const int* nlist, const int nloc,
                            const int nnei) {
  raise(c_virial_grad(grad_net, grad, env_deriv, rij, nlist, nloc, nnei),
        "prod_virial_grad_a_gpu");
  sync("prod_virial_grad_a_gpu");
}

#define DPB_INSTANTIATE(T)                                                                   \
  template void normalize_coord_gpu<T>(T*, const int, const Region<T>&);                     \
  template int copy_coord_gpu<T>(T*, int*, int*, int*, int*, const T*, const int*,           \
                                 const int&, const int&, const int&, const int&, const int*, \
                                 const Region<T>&);                                          \
  template int build_nlist_gpu<T>(InputNlist&, int*, int*, const T*, const int&, const int&, \
                                  const int&, const float&, const int&, const int*);         \
  template void prod_env_mat_a_gpu<T>(T*, T*, T*, int*, const T*, const int*,                \
                                      const InputNlist&, int*, unsigned long long*, const int, \
                                      const T*, const T*, const int, const int, const int,    \
                                      const float, const float, const std::vector<int>,       \
                                      const int*);                                            \
  template void tabulate_fusion_se_a_gpu<T>(T*, const T*, const T*, const T*, const T*,      \
                                            const T*, const int, const int, const int,       \
                                            const bool, const int);                          \
  template void tabulate_fusion_se_a_grad_gpu<T>(T*, T*, T*, const T*, const T*, const T*,   \
                                                 const T*, const T*, const T*, const int,    \
                                                 const int, const int, const bool,           \
                                                 const int);                                 \
  template void tabulate_fusion_se_a_grad_grad_gpu<T>(                                       \
      T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*,    \
      const int, const int, const int, const bool, const int);                               \
  template void prod_force_a_gpu<T>(T*, const T*, const T*, const int*, const int,           \
                                    const int, const int, const int);                        \
  template void prod_virial_a_gpu<T>(T*, T*, const T*, const T*, const T*, const int*,       \
                                     const int, const int, const int);                       \
  template void prod_force_grad_a_gpu<T>(T*, const T*, const T*, const int*, const int,      \
                                         const int, const int);                              \
  template void prod_virial_grad_a_gpu<T>(T*, const T*, const T*, const T*, const int*,      \
                                          const int, const int);

DPB_INSTANTIATE(float)
DPB_INSTANTIATE(double)

}  // namespace deepmd
