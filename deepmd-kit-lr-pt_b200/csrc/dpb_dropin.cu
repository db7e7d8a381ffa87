// Neighbor-list helpers of the reference's device API that the engines call
// around the se_e2_a path:
//
//  dpb_use_nlist_map        : nlist[i, k] = map[nlist[i, k]] for every entry
//                             that is not -1 (map_nlist / use_nlist_map,
//                             source/lib/src/gpu/neighbor_list.cu:132-146,
//                             252-264): an engine's own atom order applied to
//                             a formatted list.
//  dpb_nlist_rows_to_device : a host InputNlist (ilist, numneigh, the
//                             firstneigh rows) moved into device rows of fixed
//                             width (convert_nlist_gpu_device, source/lib/src/
//                             neighbor_list.cc:1010-1033). The reference issues
//                             one host-to-device copy per row; here the rows are
//                             packed back to back on the host, moved by one
//                             copy, and scattered into the padded device rows
//                             (and firstneigh filled) by one kernel. Only the
//                             first numneigh[ii] entries of each row are written,
//                             as in the reference.
#include <vector>

#include "dpb_common.cuh"

namespace dpb {

__global__ void k_nlist_map(int* __restrict__ nlist, const int* __restrict__ map,
                            long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int j = nlist[i];
    if (j != -1) nlist[i] = map[j];
  }
}

// One warp per row: the packed row (offset off[ii], numneigh[ii] entries) to
// rows + ii * width, and firstneigh[ii] pointing there.
__global__ void k_rows_scatter(int* __restrict__ rows, int** __restrict__ firstneigh,
                               const int* __restrict__ packed, const long long* __restrict__ off,
                               int inum, int width) {
  const int lane = threadIdx.x & 31;
  for (int ii = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ii < inum;
       ii += (gridDim.x * blockDim.x) >> 5) {
    int* dst = rows + (long long)ii * width;
    const long long a = off[ii], n = off[ii + 1] - a;
    for (long long k = lane; k < n; k += 32) dst[k] = packed[a + k];
    if (lane == 0) firstneigh[ii] = dst;
  }
}

}  // namespace dpb

using namespace dpb;

extern "C" {

int dpb_use_nlist_map(int* nlist, const int* nlist_map, int nloc, int nnei,
                      dpb_stream_t stream) {
  if (nloc < 0 || nnei < 0 || (nloc > 0 && nnei > 0 && (!nlist || !nlist_map))) {
    set_error("use_nlist_map: invalid arguments (nloc=%d nnei=%d)", nloc, nnei);
    return DPB_ERR_INVALID;
  }
  const long long n = (long long)nloc * nnei;
  if (n == 0) return DPB_OK;
  k_nlist_map<<<grid_stride_blocks(n, 256), 256, 0, as_stream(stream)>>>(nlist, nlist_map, n);
  DPB_CHECK_LAUNCH("use_nlist_map");
  return DPB_OK;
}

long long dpb_nlist_rows_scratch_bytes(const int* numneigh, int inum) {
  if (inum < 0 || (inum > 0 && !numneigh)) return -1;
  long long total = 0;
  for (int ii = 0; ii < inum; ++ii) total += numneigh[ii] > 0 ? numneigh[ii] : 0;
  return (long long)(inum + 1) * (long long)sizeof(long long) + total * (long long)sizeof(int);
}

int dpb_nlist_rows_to_device(int* d_ilist, int* d_numneigh, int** d_firstneigh, int* d_rows,
                             int width, const int* ilist, const int* numneigh,
                             const int* const* firstneigh, int inum, void* d_scratch,
                             long long scratch_bytes, dpb_stream_t stream) {
  if (inum < 0 || width < 0) {
    set_error("nlist_rows_to_device: invalid sizes (inum=%d width=%d)", inum, width);
    return DPB_ERR_INVALID;
  }
  if (inum == 0) return DPB_OK;
  if (!d_ilist || !d_numneigh || !d_firstneigh || !d_rows || !ilist || !numneigh ||
      !firstneigh) {
    set_error("nlist_rows_to_device: null pointer argument");
    return DPB_ERR_INVALID;
  }
  // host side: row offsets, then the rows back to back (rows are validated
  // before anything is written to the device)
  std::vector<long long> off(inum + 1, 0);
  for (int ii = 0; ii < inum; ++ii) {
    const int n = numneigh[ii];
    if (n < 0 || n > width) {
      set_error("nlist_rows_to_device: row %d contains %d neighbors, exceeding the allocated "
                "GPU row capacity %d", ii, n, width);
      return DPB_ERR_NLIST_CAPACITY;
    }
    if (n > 0 && firstneigh[ii] == nullptr) {
      set_error("nlist_rows_to_device: row %d has no neighbor array", ii);
      return DPB_ERR_INVALID;
    }
    off[ii + 1] = off[ii] + n;
  }
  const long long total = off[inum];
  const long long need = (long long)(inum + 1) * (long long)sizeof(long long) +
                         total * (long long)sizeof(int);
  if (!d_scratch || scratch_bytes < need) {
    set_error("nlist_rows_to_device: scratch too small (%lld < %lld bytes)", scratch_bytes,
              need);
    return DPB_ERR_INVALID;
  }
  std::vector<int> packed((size_t)(total > 0 ? total : 1));
  for (int ii = 0; ii < inum; ++ii)
    for (int k = 0; k < numneigh[ii]; ++k) packed[(size_t)(off[ii] + k)] = firstneigh[ii][k];
  cudaStream_t st = as_stream(stream);
  long long* d_off = (long long*)d_scratch;
  int* d_packed = (int*)(d_off + inum + 1);
  // pageable sources: each copy returns once its source has been staged, so
  // the host vectors may go out of scope afterwards
  DPB_CUDA(cudaMemcpyAsync(d_ilist, ilist, sizeof(int) * inum, cudaMemcpyHostToDevice, st),
           "nlist_rows_to_device");
  DPB_CUDA(cudaMemcpyAsync(d_numneigh, numneigh, sizeof(int) * inum, cudaMemcpyHostToDevice, st),
           "nlist_rows_to_device");
  DPB_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * (inum + 1),
                           cudaMemcpyHostToDevice, st),
           "nlist_rows_to_device");
  if (total > 0)
    DPB_CUDA(cudaMemcpyAsync(d_packed, packed.data(), sizeof(int) * total,
                             cudaMemcpyHostToDevice, st),
             "nlist_rows_to_device");
  k_rows_scatter<<<grid_stride_blocks((long long)inum * 32, 256), 256, 0, st>>>(
      d_rows, d_firstneigh, d_packed, d_off, inum, width);
  DPB_CHECK_LAUNCH("nlist_rows_to_device");
  // the staged host buffers are consumed; wait so that the caller may reuse
  // or free the scratch as soon as this returns
  DPB_CUDA(cudaStreamSynchronize(st), "nlist_rows_to_device");
  return DPB_OK;
}

}  // extern "C"
