// C++ drop-in for the reference's deepmd:: GPU functions on the se_e2_a path.
//
// libdpb200.so defines these templates for float and double with the same
// names, parameter lists and namespaces as the reference's
// source/lib/include/{neighbor_list,prod_env_mat,tabulate,prod_force,
// prod_virial,coord}.h, so the mangled symbols of the reference's explicit
// instantiations resolve to this library. Each forwards to the C-ABI in
// ../dpb200.h and, like the reference, synchronises the device and throws a
// deepmd::deepmd_exception (or _oom / _nlist_capacity) on failure.
//
// InputNlist has the reference's member layout (neighbor_list.h:20-119) so an
// object built by the reference's callers can be passed as is; only inum,
// ilist, numneigh and firstneigh are read here.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#define DPB_CXX_API __attribute__((visibility("default")))

namespace deepmd {

// source/lib/include/errors.h:9-33
struct deepmd_exception : public std::runtime_error {
 public:
  deepmd_exception() : runtime_error("DeePMD-kit Error!") {}
  deepmd_exception(const std::string& msg)
      : runtime_error(std::string("DeePMD-kit Error: ") + msg) {}
};
struct deepmd_exception_oom : public deepmd_exception {
 public:
  deepmd_exception_oom() : deepmd_exception("DeePMD-kit OOM!") {}
  deepmd_exception_oom(const std::string& msg)
      : deepmd_exception(std::string("DeePMD-kit OOM: ") + msg) {}
};
struct deepmd_exception_nlist_capacity : public deepmd_exception {
 public:
  using deepmd_exception::deepmd_exception;
};

// source/lib/include/neighbor_list.h:20-119 (member order is the ABI)
struct InputNlist {
  int inum;
  int* ilist;
  int* numneigh;
  int** firstneigh;
  int nswap;
  int* sendnum;
  int* recvnum;
  int* firstrecv;
  int** sendlist;
  int* sendproc;
  int* recvproc;
  void* world;
  int mask = 0xFFFFFFFF;
  int* mapping = nullptr;
  int nprocs = 1;
  InputNlist()
      : inum(0), ilist(nullptr), numneigh(nullptr), firstneigh(nullptr),
        nswap(0), sendnum(nullptr), recvnum(nullptr), firstrecv(nullptr),
        sendlist(nullptr), sendproc(nullptr), recvproc(nullptr),
        world(nullptr) {}
  InputNlist(int inum_, int* ilist_, int* numneigh_, int** firstneigh_)
      : inum(inum_), ilist(ilist_), numneigh(numneigh_),
        firstneigh(firstneigh_), nswap(0), sendnum(nullptr), recvnum(nullptr),
        firstrecv(nullptr), sendlist(nullptr), sendproc(nullptr),
        recvproc(nullptr), world(nullptr) {}
};

// source/lib/include/region.h:6-16 (member layout). Its constructors and
// destructor are the reference's own (source/lib/src/region.cc); the
// functions below only read boxt and rec_boxt, which point to device memory
// as the reference's GPU callers set them up
// (op/tf/prod_env_mat_multi_device.cc:2417-2442).
template <typename FPTYPE>
struct Region {
  FPTYPE* boxt;
  FPTYPE* rec_boxt;
  Region();
  Region(FPTYPE* extern_boxt, FPTYPE* extern_rec_boxt);
  ~Region();

 private:
  bool self_allocated;
};

// source/lib/include/coord.h:56-59: wrap natom device coordinates into the
// box (the box is read from region.boxt on the device).
template <typename FPTYPE>
DPB_CXX_API void normalize_coord_gpu(FPTYPE* coord, const int natom,
                                     const Region<FPTYPE>& region);

// source/lib/include/coord.h:72-85: ghost copy on the caller's cell
// decomposition (cell_info, 23 device ints from compute_cell_info); int_data
// is the caller's scratch of 4 nloc + 2 loc_cellnum + 7 total_cellnum + 2
// ints (what the reference's callers allocate). Returns 1 when nall exceeds
// mem_nall. Ghost order: that of copy_coord_cpu.
template <typename FPTYPE>
DPB_CXX_API int copy_coord_gpu(FPTYPE* out_c, int* out_t, int* mapping, int* nall,
                               int* int_data, const FPTYPE* in_c, const int* in_t,
                               const int& nloc, const int& mem_nall, const int& loc_cellnum,
                               const int& total_cellnum, const int* cell_info,
                               const Region<FPTYPE>& region);

// source/lib/include/neighbor_list.h:201-228
DPB_CXX_API void convert_nlist_gpu_device(InputNlist& gpu_nlist, InputNlist& cpu_nlist,
                                          int*& gpu_memory, const int& max_nbor_size);
DPB_CXX_API void free_nlist_gpu_device(InputNlist& gpu_nlist);
DPB_CXX_API void use_nlist_map(int* nlist, const int* nlist_map, const int nloc,
                               const int nnei);

// source/lib/include/neighbor_list.h:260-270
template <typename FPTYPE>
DPB_CXX_API int build_nlist_gpu(InputNlist& nlist, int* max_list_size,
                                int* nlist_data, const FPTYPE* c_cpy,
                                const int& nloc, const int& nall,
                                const int& mem_size, const float& rcut,
                                const int& nframes = 1,
                                const int* type = nullptr);

// source/lib/include/prod_env_mat.h:97-116 (array_longlong is not needed:
// the sort runs in shared memory; array_int[0] is used as the status word)
template <typename FPTYPE>
DPB_CXX_API void prod_env_mat_a_gpu(
    FPTYPE* em, FPTYPE* em_deriv, FPTYPE* rij, int* nlist, const FPTYPE* coord,
    const int* type, const InputNlist& gpu_inlist, int* array_int,
    unsigned long long* array_longlong, const int max_nbor_size,
    const FPTYPE* avg, const FPTYPE* std, const int nloc, const int nall,
    const int nframes, const float rcut, const float rcut_smth,
    const std::vector<int> sec, const int* f_type = nullptr);

// source/lib/include/tabulate.h:175-217
template <typename FPTYPE>
DPB_CXX_API void tabulate_fusion_se_a_gpu(
    FPTYPE* out, const FPTYPE* table, const FPTYPE* table_info,
    const FPTYPE* em_x, const FPTYPE* em, const FPTYPE* two_embed,
    const int nloc, const int nnei, const int last_layer_size,
    const bool is_sorted = true, const int ndescrpt = 4);

template <typename FPTYPE>
DPB_CXX_API void tabulate_fusion_se_a_grad_gpu(
    FPTYPE* dy_dem_x, FPTYPE* dy_dem, FPTYPE* dy_dtwo, const FPTYPE* table,
    const FPTYPE* table_info, const FPTYPE* em_x, const FPTYPE* em,
    const FPTYPE* two_embed, const FPTYPE* dy, const int nloc, const int nnei,
    const int last_layer_size, const bool is_sorted = true,
    const int ndescrpt = 4);

template <typename FPTYPE>
DPB_CXX_API void tabulate_fusion_se_a_grad_grad_gpu(
    FPTYPE* dz_dy, const FPTYPE* table, const FPTYPE* table_info,
    const FPTYPE* em_x, const FPTYPE* em, const FPTYPE* two_embed,
    const FPTYPE* dz_dy_dem_x, const FPTYPE* dz_dy_dem,
    const FPTYPE* dz_dy_dtwo, const int nloc, const int nnei,
    const int last_layer_size, const bool is_sorted = true,
    const int ndescrpt = 4);

// source/lib/include/prod_force.h:71-79
template <typename FPTYPE>
DPB_CXX_API void prod_force_a_gpu(FPTYPE* force, const FPTYPE* net_deriv,
                                  const FPTYPE* in_deriv, const int* nlist,
                                  const int nloc, const int nall,
                                  const int nnei, const int nframes);

// source/lib/include/prod_virial.h:29-38
template <typename FPTYPE>
DPB_CXX_API void prod_virial_a_gpu(FPTYPE* virial, FPTYPE* atom_virial,
                                   const FPTYPE* net_deriv,
                                   const FPTYPE* env_deriv, const FPTYPE* rij,
                                   const int* nlist, const int nloc,
                                   const int nall, const int nnei);

// source/lib/include/prod_force_grad.h:26-32
template <typename FPTYPE>
DPB_CXX_API void prod_force_grad_a_gpu(FPTYPE* grad_net, const FPTYPE* grad,
                                       const FPTYPE* env_deriv, const int* nlist,
                                       const int nloc, const int nnei,
                                       const int nframes);

// source/lib/include/prod_virial_grad.h:26-32
template <typename FPTYPE>
DPB_CXX_API void prod_virial_grad_a_gpu(FPTYPE* grad_net, const FPTYPE* grad,
                                        const FPTYPE* env_deriv, const FPTYPE* rij,
                                        const int* nlist, const int nloc,
                                        const int nnei);

}  // namespace deepmd
