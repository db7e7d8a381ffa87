// Internal structures shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>

namespace dpb {

// Box data computed on the host once per call (passed by value to kernels).
struct HostRegion {
  double box[9];     // rows are the box vectors
  double rec[9];     // cofactor inverse, SimulationRegion_Impl.h:455-480
  double inv_nc[3];  // 1 / ncell (build_clist cell size in box units)
  double volume;
  int nc[3];         // local cells per dimension
  int ng[3];         // ghost cell layers per dimension
  int nloc_cells;
  int next_cells;    // prod(nc + 2 ng)
};

void host_region(HostRegion& r, const double* boxt, float rcut);

// Cell grid over a point set (device memory, carved from a caller buffer).
struct GridHeader {
  unsigned long long kmin[3], kmax[3];  // order-preserving bbox keys
  double origin[3];
  double inv_cs[3];
  int dims[3];
  int ncells;
  int natoms;
  int packed;  // 1: cell_pos holds this grid's atoms in cell order (fused builder)
  int pad[2];
};

struct GridView {
  GridHeader* h;
  int* cell_start;  // [ncells + 1]
  int* fill;        // [ncells]
  int* cell_of;     // [natoms]
  int* cell_atoms;  // [natoms], atoms sorted by cell
  int* redo;        // [natoms + 1]: count, then atoms deferred to a larger buffer
  // [natoms] in cell order: x, y, z and (type << 32 | atom index) as the
  // bits of the fourth double. Its storage follows the grid in buffers of
  // grid_bytes_packed(nall) bytes; valid only while h->packed == 1
  double4* cell_pos;
  int max_cells;
  int cap_atoms;
};

long long grid_bytes(int nall);
// a grid buffer with room for the cell-ordered positions after the grid
long long grid_bytes_packed(int nall);
GridView carve_grid(void* p, int nall);
template <typename T>
int grid_build(void* grid, long long bytes, const T* coord, int nall,
               const int* nall_dev, float rcut, cudaStream_t st);
template <typename T>
int copy_coord_async(T* out_c, int* out_t, int* mapping, int* nall_dev,
                     void* scratch, long long scratch_bytes, const T* in_c,
                     const int* in_t, int nloc, int mem_nall, float rcut,
                     const double* boxt, cudaStream_t st);
long long copy_coord_scratch_bytes(int nloc, float rcut, const double* boxt);
template <typename T>
int build_nlist(int* ilist, int* numneigh, int** firstneigh, int* max_list_size,
                void* scratch, long long scratch_bytes, const T* c_cpy, int nloc,
                int nall, int mem_size, float rcut, int nframes, const int* type,
                cudaStream_t st);

}  // namespace dpb
