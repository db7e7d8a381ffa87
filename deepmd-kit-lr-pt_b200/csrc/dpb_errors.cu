// Error reporting and the device status word read-back.
#include <stdarg.h>
#include <stdio.h>

#include "dpb_common.cuh"

namespace dpb {

static thread_local char g_msg[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
  set_error("CUDA error in %s: %s", where, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? DPB_ERR_OOM : DPB_ERR_CUDA;
}

}  // namespace dpb

extern "C" {

const char* dpb_last_error(void) { return dpb::g_msg; }

int dpb_abi_version(void) { return 1; }

int dpb_zero_async(void* dst, long long bytes, dpb_stream_t stream) {
  if (bytes == 0) return DPB_OK;
  if (dst == nullptr || bytes < 0) {
    dpb::set_error("dpb_zero_async: null destination or negative size (%lld bytes)", bytes);
    return DPB_ERR_INVALID;
  }
  DPB_CUDA(cudaMemsetAsync(dst, 0, (size_t)bytes, dpb::as_stream(stream)), "dpb_zero_async");
  return DPB_OK;
}

int dpb_status_check(const int* status, dpb_stream_t stream) {
  if (status == nullptr) return DPB_OK;
  int h = 0;
  cudaStream_t s = dpb::as_stream(stream);
  DPB_CUDA(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, s),
           "dpb_status_check");
  DPB_CUDA(cudaStreamSynchronize(s), "dpb_status_check");
  if (h == 0) return DPB_OK;
  if (h & dpb::ST_KEY_OVERFLOW) {
    dpb::set_error(
        "neighbor sort key overflow: a type >= 128 or an atom index >= 2^24 "
        "(status 0x%x)", h);
    return DPB_ERR_OVERFLOW;
  }
  if (h & (dpb::ST_NLIST_CAPACITY | dpb::ST_ROW_CAPACITY)) {
    dpb::set_error(
        "neighbor row capacity exceeded: more in-range candidates than the "
        "row buffer holds (status 0x%x)", h);
    return DPB_ERR_NLIST_CAPACITY;
  }
  if (h & dpb::ST_SYNC_TIMEOUT) {
    dpb::set_error("a grid-wide barrier of the geometry pass timed out (status 0x%x)", h);
    return DPB_ERR_CUDA;
  }
  if (h & (1 << 8)) {
    dpb::set_error("a tensor-core GEMM timed out waiting on its pipeline (status 0x%x)", h);
    return DPB_ERR_CUDA;
  }
  if (h & dpb::ST_TYPE_RANGE) {
    dpb::set_error("an atom type is >= ntypes = len(sec) - 1 (status 0x%x)", h);
    return DPB_ERR_INVALID;
  }
  if (h & dpb::ST_CELL_RANGE) {
    dpb::set_error("cell index outside the cell grid (status 0x%x)", h);
    return DPB_ERR_INVALID;
  }
  // ST_SEL_OVERFLOW alone is not an error: the reference drops the farthest
  // neighbors of an overflowing type (fmt_nlist.cc:132-141).
  return DPB_OK;
}

}  // extern "C"
