// Test infrastructure only: a C-ABI shim over the reference DeePMD-kit CPU
// library (source/lib/src/*.cc), compiled from the reference sources into
// oracle/_ref/libdpref.so by oracle/Makefile. Only tests, the smoke check and
// the CPU-baseline leg of bench.py load it; the product never does.
//
// Each entry point forwards to the deepmd:: CPU template named beside it and
// keeps that function's argument meaning. The InputNlist is passed flat:
// ilist[inum], numneigh[inum] and a dense row buffer firstneigh_rows
// [inum, row_stride] (row r starts at firstneigh_rows + r * row_stride).
#include <cstring>
#include <exception>
#include <vector>

#include "coord.h"
#include "env_mat.h"
#include "fmt_nlist.h"
#include "neighbor_list.h"
#include "prod_env_mat.h"
#include "prod_force.h"
#include "prod_force_grad.h"
#include "prod_virial.h"
#include "prod_virial_grad.h"
#include "region.h"
#include "tabulate.h"

namespace {

struct FlatNlist {
  std::vector<int*> rows;
  deepmd::InputNlist nl;
  FlatNlist(int inum, int* ilist, int* numneigh, int* rowbuf, int stride)
      : rows(inum > 0 ? inum : 1) {
    for (int ii = 0; ii < inum; ++ii) {
      rows[ii] = rowbuf + static_cast<size_t>(ii) * stride;
    }
    nl = deepmd::InputNlist(inum, ilist, numneigh, rows.data());
  }
};

}  // namespace

extern "C" {

// source/lib/src/coord.cc:14-27 (normalize_coord_cpu)
int dpref_normalize_coord_f64(double* coord, int natom, const double* boxt) {
  try {
    deepmd::Region<double> region;
    deepmd::init_region_cpu(region, boxt);
    deepmd::normalize_coord_cpu(coord, natom, region);
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// source/lib/src/coord.cc:29-64 (copy_coord_cpu); returns 1 when nall > mem_nall
int dpref_copy_coord_f64(double* out_c, int* out_t, int* mapping, int* nall,
                         const double* in_c, const int* in_t, int nloc,
                         int mem_nall, float rcut, const double* boxt) {
  try {
    deepmd::Region<double> region;
    deepmd::init_region_cpu(region, boxt);
    return deepmd::copy_coord_cpu(out_c, out_t, mapping, nall, in_c, in_t,
                                  nloc, mem_nall, rcut, region);
  } catch (const std::exception&) {
    return 2;
  }
}

// source/lib/src/coord.cc:66-107 (compute_cell_info), 23 ints
int dpref_compute_cell_info_f64(int* cell_info, float rcut,
                                const double* boxt) {
  try {
    deepmd::Region<double> region;
    deepmd::init_region_cpu(region, boxt);
    deepmd::compute_cell_info(cell_info, rcut, region);
  } catch (const std::exception&) {
    return 2;
  }
  return 0;
}

// source/lib/src/neighbor_list.cc:875-928 (build_nlist_cpu)
int dpref_build_nlist_f64(int* ilist, int* numneigh, int* rowbuf,
                          int* max_list_size, const double* c_cpy, int nloc,
                          int nall, int mem_size, float rcut, int nframes,
                          const int* type) {
  FlatNlist f(nframes * nloc, ilist, numneigh, rowbuf, mem_size);
  return deepmd::build_nlist_cpu(f.nl, max_list_size, c_cpy, nloc, nall,
                                 mem_size, rcut, nframes, type);
}

int dpref_build_nlist_f32(int* ilist, int* numneigh, int* rowbuf,
                          int* max_list_size, const float* c_cpy, int nloc,
                          int nall, int mem_size, float rcut, int nframes,
                          const int* type) {
  FlatNlist f(nframes * nloc, ilist, numneigh, rowbuf, mem_size);
  return deepmd::build_nlist_cpu(f.nl, max_list_size, c_cpy, nloc, nall,
                                 mem_size, rcut, nframes, type);
}

// source/lib/src/fmt_nlist.cc:98-143 (format_nlist_i_cpu) over all rows
int dpref_format_nlist_f64(int* nlist, const double* coord, const int* type,
                           int nloc, int nall, const int* ilist,
                           const int* numneigh, const int* rowbuf, int stride,
                           float rcut, const int* sec, int nsec) {
  std::vector<double> posi(coord, coord + static_cast<size_t>(nall) * 3);
  std::vector<int> atype(type, type + nall);
  std::vector<int> sec_a(sec, sec + nsec);
  int nnei = sec_a.back();
  int ret = -1;
  for (int ii = 0; ii < nloc; ++ii) {
    int i_idx = ilist[ii];
    std::vector<int> cand(rowbuf + static_cast<size_t>(ii) * stride,
                          rowbuf + static_cast<size_t>(ii) * stride +
                              numneigh[ii]);
    std::vector<int> fmt;
    int r = format_nlist_i_cpu<double>(fmt, posi, atype, i_idx, cand, rcut,
                                       sec_a);
    if (r != -1) ret = r;
    std::memcpy(nlist + static_cast<size_t>(i_idx) * nnei, fmt.data(),
                sizeof(int) * nnei);
  }
  return ret;
}

#define DPREF_ENV(T, SUF)                                                     \
  int dpref_prod_env_mat_a_##SUF(                                             \
      T* em, T* em_deriv, T* rij, int* nlist, const T* coord,                 \
      const int* type, int inum, int* ilist, int* numneigh, int* rowbuf,      \
      int stride, const T* avg, const T* std_, int nloc, int nall,            \
      int nframes, float rcut, float rcut_smth, const int* sec, int nsec) {   \
    try {                                                                     \
      FlatNlist f(inum, ilist, numneigh, rowbuf, stride);                     \
      std::vector<int> s(sec, sec + nsec);                                    \
      deepmd::prod_env_mat_a_cpu(em, em_deriv, rij, nlist, coord, type, f.nl, \
                                 stride, avg, std_, nloc, nall, nframes,      \
                                 rcut, rcut_smth, s);                         \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_tabulate_fusion_se_a_##SUF(                                       \
      T* out, const T* table, const T* info, const T* em_x, const T* em,      \
      int nloc, int nnei, int last_layer_size) {                              \
    try {                                                                     \
      deepmd::tabulate_fusion_se_a_cpu<T>(out, table, info, em_x, em,         \
                                          nullptr, nloc, nnei,                \
                                          last_layer_size, true, 4);          \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_tabulate_fusion_se_a_grad_##SUF(                                  \
      T* dy_dem_x, T* dy_dem, const T* table, const T* info, const T* em_x,   \
      const T* em, const T* dy, int nloc, int nnei, int last_layer_size) {    \
    try {                                                                     \
      deepmd::tabulate_fusion_se_a_grad_cpu<T>(                               \
          dy_dem_x, dy_dem, nullptr, table, info, em_x, em, nullptr, dy,      \
          nloc, nnei, last_layer_size, true, 4);                              \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_tabulate_fusion_se_a_grad_grad_##SUF(                             \
      T* dz_dy, const T* table, const T* info, const T* em_x, const T* em,    \
      const T* dz_dy_dem_x, const T* dz_dy_dem, int nloc, int nnei,           \
      int last_layer_size) {                                                  \
    try {                                                                     \
      deepmd::tabulate_fusion_se_a_grad_grad_cpu<T>(                          \
          dz_dy, table, info, em_x, em, nullptr, dz_dy_dem_x, dz_dy_dem,      \
          nullptr, nloc, nnei, last_layer_size, true, 4);                     \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_prod_force_a_##SUF(T* force, const T* net_deriv,                  \
                               const T* env_deriv, const int* nlist,          \
                               int nloc, int nall, int nnei, int nframes) {   \
    try {                                                                     \
      deepmd::prod_force_a_cpu<T>(force, net_deriv, env_deriv, nlist, nloc,   \
                                  nall, nnei, nframes);                       \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_prod_virial_a_##SUF(T* virial, T* atom_virial,                    \
                                const T* net_deriv, const T* env_deriv,       \
                                const T* rij, const int* nlist, int nloc,     \
                                int nall, int nnei) {                         \
    try {                                                                     \
      deepmd::prod_virial_a_cpu<T>(virial, atom_virial, net_deriv, env_deriv, \
                                   rij, nlist, nloc, nall, nnei);             \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_prod_force_grad_a_##SUF(T* grad_net, const T* grad,               \
                                    const T* env_deriv, const int* nlist,     \
                                    int nloc, int nnei, int nframes) {        \
    try {                                                                     \
      deepmd::prod_force_grad_a_cpu<T>(grad_net, grad, env_deriv, nlist,      \
                                       nloc, nnei, nframes);                  \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }                                                                           \
  int dpref_prod_virial_grad_a_##SUF(T* grad_net, const T* grad,              \
                                     const T* env_deriv, const T* rij,        \
                                     const int* nlist, int nloc, int nnei) {  \
    try {                                                                     \
      deepmd::prod_virial_grad_a_cpu<T>(grad_net, grad, env_deriv, rij,       \
                                        nlist, nloc, nnei);                   \
    } catch (const std::exception&) {                                         \
      return 2;                                                               \
    }                                                                         \
    return 0;                                                                 \
  }

DPREF_ENV(double, f64)
DPREF_ENV(float, f32)

}  // extern "C"
