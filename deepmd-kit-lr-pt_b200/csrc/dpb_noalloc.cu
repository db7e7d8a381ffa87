// Neighbor-list build for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: for example an MD
// engine's force callback that runs inside the engine's own device-memory
// pool and is not allowed to allocate during a time step, or a loop where the
// device-wide synchronisation and unpredictable latency of an allocation are
// not acceptable. dpb_build_nlist_noalloc_f64 serves them: the caller passes
// only inputs and outputs, and the working memory of the cell grid lives in
// the file-scope device array below (DPB_NOALLOC_SCRATCH_BYTES, 4 MiB). Every
// GPU that loads the library holds that array until the process exits.
//
// The array holds the cell grid of nall extended atoms plus two status words:
// dpb_cell_grid_bytes(nall) + 256 <= 4 MiB, i.e. nall <= 209,670 (about 20
// bytes per extended atom); larger calls are rejected before any GPU work.
//
// The device address of the array is looked up with cudaGetSymbolAddress the
// first time the entry point runs on a device (with that device current) and
// cached per device for the life of the process; make that first call before
// any stream capture. The cached address belongs to the device's current
// context: a process that destroys it (cudaDeviceReset) must not call this
// entry point on that device again. Every call shares the one array per
// device and leaves its contents behind; the parts that must start at zero
// (status words, cell counters, bounding box) are reset by each call. Two
// calls whose work overlaps on the same GPU (e.g. from two host threads on
// different streams) race on the array and must not be issued.
#include <mutex>

#include "dpb_common.cuh"
#include "dpb_internal.cuh"

#define DPB_NOALLOC_SCRATCH_BYTES (4ll << 20)

static __device__ __align__(256) unsigned char g_nlist_scratch[DPB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

// Device address of g_nlist_scratch on the current device. The name of the
// array in host code is only a host-side stand-in, never a device address.
int scratch_address(void** out) {
  int dev = -1;
  DPB_CUDA(cudaGetDevice(&dev), "build_nlist_noalloc");
  if (dev < 0 || dev >= kMaxDevices) {
    dpb::set_error("build_nlist_noalloc: device ordinal %d is out of range", dev);
    return DPB_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[dev] == nullptr) {
    void* p = nullptr;
    DPB_CUDA(cudaGetSymbolAddress(&p, g_nlist_scratch), "build_nlist_noalloc");
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return DPB_OK;
}

}  // namespace

extern "C" {

long long dpb_build_nlist_noalloc_max_bytes(void) { return DPB_NOALLOC_SCRATCH_BYTES; }

int dpb_build_nlist_noalloc_f64(int* ilist, int* numneigh, int** firstneigh,
                                int* max_list_size, const double* c_cpy, int nloc,
                                int nall, int mem_size, float rcut, int nframes,
                                const int* type, dpb_stream_t stream) {
  const long long need = dpb::grid_bytes(nall) + 256;
  if (need > DPB_NOALLOC_SCRATCH_BYTES) {
    dpb::set_error(
        "build_nlist_noalloc: nall=%d needs %lld bytes of working memory, more than the "
        "%lld-byte built-in array; use dpb_build_nlist_f64 with caller scratch",
        nall, need, (long long)DPB_NOALLOC_SCRATCH_BYTES);
    return DPB_ERR_INVALID;
  }
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != DPB_OK) return rc;
  return dpb::build_nlist<double>(ilist, numneigh, firstneigh, max_list_size, scratch,
                                  DPB_NOALLOC_SCRATCH_BYTES, c_cpy, nloc, nall, mem_size,
                                  rcut, nframes, type, dpb::as_stream(stream));
}

}  // extern "C"
