// Test infrastructure only: a C-ABI shim over the reference DeePMD-kit CUDA
// library (source/lib/src/gpu/*.cu), compiled for sm_100a from the reference
// sources into oracle/_ref/libdpref_gpu.so by oracle/Makefile. Only the GPU
// tests load it, to compare the reference's own device kernels with this
// package's drop-ins on the same inputs (results and CUDA-event times); the
// product never does.
//
// Each entry point forwards to the deepmd:: GPU template named beside it and
// keeps that function's argument meaning. The reference functions run on the
// legacy default stream and synchronise the device before and after their
// kernels. firstneigh is a DEVICE array of device row pointers, as the
// reference's convert_nlist_gpu_device produces (neighbor_list.cc:1010-1033).
// Returns 0, or 1 when the reference raised.
#include <exception>
#include <vector>

#include "neighbor_list.h"
#include "prod_env_mat.h"
#include "prod_force.h"
#include "prod_virial.h"
#include "tabulate.h"

#define REFGPU_API extern "C" __attribute__((visibility("default")))

// source/lib/src/gpu/neighbor_list.cu:197-250 (build_nlist_gpu<double>);
// returns 2 when mem_size < nall (the reference's return value 1)
REFGPU_API int refgpu_build_nlist_f64(int* ilist, int* numneigh, int** firstneigh,
                                      int* max_list_size, int* nlist_data,
                                      const double* c_cpy, int nloc, int nall,
                                      int mem_size, float rcut) {
  try {
    deepmd::InputNlist nl(nloc, ilist, numneigh, firstneigh);
    const int r = deepmd::build_nlist_gpu<double>(nl, max_list_size, nlist_data, c_cpy, nloc,
                                                  nall, mem_size, rcut);
    return r == 0 ? 0 : 2;
  } catch (const std::exception&) {
    return 1;
  }
}

// source/lib/src/gpu/prod_env_mat.cu:681-726 (prod_env_mat_a_gpu)
template <typename T>
static int env_mat(T* em, T* em_deriv, T* rij, int* nlist, const T* coord, const int* type,
                   int inum, int* ilist, int* numneigh, int** firstneigh, int* array_int,
                   unsigned long long* array_longlong, int max_nbor, const T* avg,
                   const T* std_, int nloc, int nall, float rcut, float rcut_smth,
                   const int* sec, int nsec) {
  try {
    deepmd::InputNlist nl(inum, ilist, numneigh, firstneigh);
    std::vector<int> s(sec, sec + nsec);
    deepmd::prod_env_mat_a_gpu<T>(em, em_deriv, rij, nlist, coord, type, nl, array_int,
                                  array_longlong, max_nbor, avg, std_, nloc, nall, rcut,
                                  rcut_smth, s);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

REFGPU_API int refgpu_prod_env_mat_a_f64(double* em, double* em_deriv, double* rij, int* nlist,
                                         const double* coord, const int* type, int inum,
                                         int* ilist, int* numneigh, int** firstneigh,
                                         int* array_int, unsigned long long* array_longlong,
                                         int max_nbor, const double* avg, const double* std_,
                                         int nloc, int nall, float rcut, float rcut_smth,
                                         const int* sec, int nsec) {
  return env_mat<double>(em, em_deriv, rij, nlist, coord, type, inum, ilist, numneigh,
                         firstneigh, array_int, array_longlong, max_nbor, avg, std_, nloc, nall,
                         rcut, rcut_smth, sec, nsec);
}

REFGPU_API int refgpu_prod_env_mat_a_f32(float* em, float* em_deriv, float* rij, int* nlist,
                                         const float* coord, const int* type, int inum,
                                         int* ilist, int* numneigh, int** firstneigh,
                                         int* array_int, unsigned long long* array_longlong,
                                         int max_nbor, const float* avg, const float* std_,
                                         int nloc, int nall, float rcut, float rcut_smth,
                                         const int* sec, int nsec) {
  return env_mat<float>(em, em_deriv, rij, nlist, coord, type, inum, ilist, numneigh,
                        firstneigh, array_int, array_longlong, max_nbor, avg, std_, nloc, nall,
                        rcut, rcut_smth, sec, nsec);
}

// source/lib/src/gpu/tabulate.cu:1219-1264 (tabulate_fusion_se_a_gpu); table_info
// is a HOST array, as in the reference op
template <typename T>
static int tab_fwd(T* out, const T* table, const T* info, const T* em_x, const T* em, int nloc,
                   int nnei, int M) {
  try {
    deepmd::tabulate_fusion_se_a_gpu<T>(out, table, info, em_x, em, nullptr, nloc, nnei, M);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}
REFGPU_API int refgpu_tabulate_fusion_se_a_f64(double* out, const double* table,
                                               const double* info, const double* em_x,
                                               const double* em, int nloc, int nnei, int M) {
  return tab_fwd<double>(out, table, info, em_x, em, nloc, nnei, M);
}
REFGPU_API int refgpu_tabulate_fusion_se_a_f32(float* out, const float* table,
                                               const float* info, const float* em_x,
                                               const float* em, int nloc, int nnei, int M) {
  return tab_fwd<float>(out, table, info, em_x, em, nloc, nnei, M);
}

// source/lib/src/gpu/tabulate.cu:1266-1315 (tabulate_fusion_se_a_grad_gpu)
template <typename T>
static int tab_grad(T* dy_dem_x, T* dy_dem, const T* table, const T* info, const T* em_x,
                    const T* em, const T* dy, int nloc, int nnei, int M) {
  try {
    deepmd::tabulate_fusion_se_a_grad_gpu<T>(dy_dem_x, dy_dem, nullptr, table, info, em_x, em,
                                             nullptr, dy, nloc, nnei, M);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}
REFGPU_API int refgpu_tabulate_fusion_se_a_grad_f64(double* dy_dem_x, double* dy_dem,
                                                    const double* table, const double* info,
                                                    const double* em_x, const double* em,
                                                    const double* dy, int nloc, int nnei,
                                                    int M) {
  return tab_grad<double>(dy_dem_x, dy_dem, table, info, em_x, em, dy, nloc, nnei, M);
}
REFGPU_API int refgpu_tabulate_fusion_se_a_grad_f32(float* dy_dem_x, float* dy_dem,
                                                    const float* table, const float* info,
                                                    const float* em_x, const float* em,
                                                    const float* dy, int nloc, int nnei, int M) {
  return tab_grad<float>(dy_dem_x, dy_dem, table, info, em_x, em, dy, nloc, nnei, M);
}

// source/lib/src/gpu/prod_force.cu:104-138 (prod_force_a_gpu, one frame)
template <typename T>
static int force(T* f, const T* nd, const T* ed, const int* nlist, int nloc, int nall,
                 int nnei) {
  try {
    deepmd::prod_force_a_gpu<T>(f, nd, ed, nlist, nloc, nall, nnei, 1);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}
REFGPU_API int refgpu_prod_force_a_f64(double* f, const double* nd, const double* ed,
                                       const int* nlist, int nloc, int nall, int nnei) {
  return force<double>(f, nd, ed, nlist, nloc, nall, nnei);
}
REFGPU_API int refgpu_prod_force_a_f32(float* f, const float* nd, const float* ed,
                                       const int* nlist, int nloc, int nall, int nnei) {
  return force<float>(f, nd, ed, nlist, nloc, nall, nnei);
}

// source/lib/src/gpu/prod_virial.cu:106-139 (prod_virial_a_gpu)
template <typename T>
static int virial(T* v, T* av, const T* nd, const T* ed, const T* rij, const int* nlist,
                  int nloc, int nall, int nnei) {
  try {
    deepmd::prod_virial_a_gpu<T>(v, av, nd, ed, rij, nlist, nloc, nall, nnei);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}
REFGPU_API int refgpu_prod_virial_a_f64(double* v, double* av, const double* nd,
                                        const double* ed, const double* rij, const int* nlist,
                                        int nloc, int nall, int nnei) {
  return virial<double>(v, av, nd, ed, rij, nlist, nloc, nall, nnei);
}
REFGPU_API int refgpu_prod_virial_a_f32(float* v, float* av, const float* nd, const float* ed,
                                        const float* rij, const int* nlist, int nloc, int nall,
                                        int nnei) {
  return virial<float>(v, av, nd, ed, rij, nlist, nloc, nall, nnei);
}
