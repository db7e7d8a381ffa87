// Frame table and packed neighbor indices shared by the batched-frames
// kernels (geometry, force/virial) and the training kernels that recompute
// the environment rows from the same packed neighbor list.
//
// A packed neighbor is (local atom j of the frame) * 27 + image code, the
// code being (sx + 1) * 9 + (sy + 1) * 3 + (sz + 1) for the lattice shift
// (sx, sy, sz) in {-1, 0, 1}^3 of the orthorhombic box.
#pragma once

#include "dpb_common.cuh"

namespace dpb {

constexpr int BT_MAXCELLS = 4096;
constexpr int BT_CAP = 256;     // in-range candidates per center
constexpr int BT_MAXT = 8;      // neighbor types
constexpr int BT_NMAX = 512;    // sum(sel)
constexpr int BT_WARPS = 4;

struct BtFrames {
  const int* atom_off;   // [F + 1]
  const int* cell_off;   // [F + 1] (each frame: ncell + 1 entries)
  const double* box;     // [F, 3] orthorhombic edge lengths
  const int* ncell;      // [F, 3] cells per edge (>= 1)
  const int* row_frame;  // [N]
  int nframes;
};

struct BtSec {
  int ntypes, nnei;
  int sec[BT_MAXT + 1];
};

__device__ __forceinline__ int bt_wrap_cell(double x, double L, int n) {
  int c = (int)(x / L * n);
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__device__ __forceinline__ unsigned bt_lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ void bt_unpack(int packed, int& j, double s[3]) {
  j = packed / 27;
  const int code = packed - j * 27;
  s[0] = (double)(code / 9 - 1);
  s[1] = (double)((code / 3) % 3 - 1);
  s[2] = (double)(code % 3 - 1);
}

// r = r_j(image) - r_i in T from FP64 wrapped coordinates of the frame
template <typename T>
__device__ __forceinline__ void bt_rij(T r[3], const double* fc, int packed, const double xi[3],
                                       const double L[3]) {
  int j;
  double s[3];
  bt_unpack(packed, j, s);
#pragma unroll
  for (int d = 0; d < 3; ++d) r[d] = (T)((fc[3 * j + d] + s[d] * L[d]) - xi[d]);
}

static inline int bt_frames(BtFrames& fr, const int* atom_off, const int* cell_off,
                            const double* box, const int* ncell, const int* row_frame,
                            int nframes) {
  if (nframes <= 0 || !atom_off || !cell_off || !box || !ncell || !row_frame) {
    set_error("batched frames: invalid frame table (nframes=%d)", nframes);
    return DPB_ERR_INVALID;
  }
  fr = BtFrames{atom_off, cell_off, box, ncell, row_frame, nframes};
  return DPB_OK;
}

}  // namespace dpb
