// Shared device/host helpers for the se_e2_a kernels (sm_100a).
//
// Error model: every C-ABI entry point returns a dpb_status code and records a
// message readable through dpb_last_error(). Kernels never trap: conditions
// the reference turns into a device trap or assert (sort-key overflow in
// source/lib/src/gpu/prod_env_mat.cu:92-99, max_nbor_size assert at :640-642)
// are written to a caller-visible device status word instead.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dpb200.h"

namespace dpb {

// Device status word bits (OR-ed together by kernels; 0 = fine).
enum : int {
  ST_NLIST_CAPACITY = 1 << 0,  // more in-range candidates than the row buffer
  ST_KEY_OVERFLOW = 1 << 1,    // type >= 128 or index >= 2^24 in a sort key
  ST_SEL_OVERFLOW = 1 << 2,    // more neighbors of a type than sel (dropped)
  ST_ROW_CAPACITY = 1 << 3,    // build_nlist row longer than mem_size
  ST_CELL_RANGE = 1 << 4,      // ghost/cell index outside the cell grid
  ST_TYPE_RANGE = 1 << 5,      // center type >= ntypes (no avg/std row)
  ST_SYNC_TIMEOUT = 1 << 6,    // a grid-wide barrier of a cooperative kernel timed out
};

void set_error(const char* fmt, ...);
// current value of a tile-shape knob (csrc/dpb_tune.cc), fallback if unknown
int tune_value(const char* name, int fallback);
int cuda_status(cudaError_t e, const char* where);

inline cudaStream_t as_stream(dpb_stream_t s) {
  return reinterpret_cast<cudaStream_t>(s);
}

#define DPB_CHECK_LAUNCH(where)                                  \
  do {                                                           \
    cudaError_t _e = cudaGetLastError();                         \
    if (_e != cudaSuccess) return ::dpb::cuda_status(_e, where); \
  } while (0)

#define DPB_CUDA(call, where)                                    \
  do {                                                           \
    cudaError_t _e = (call);                                     \
    if (_e != cudaSuccess) return ::dpb::cuda_status(_e, where); \
  } while (0)

// ---- correctly rounded, never-contracted arithmetic -----------------------
// The CPU oracle is compiled with -ffp-contract=off, so quantities that feed
// integer decisions (cutoff tests, sort keys, cell indices) are computed here
// with explicit round-to-nearest intrinsics that the compiler cannot fuse.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// r0*r0 + r1*r1 + r2*r2 evaluated left to right without fusion
// (source/lib/include/utilities.h:24-26).
template <typename T>
__device__ __forceinline__ T dot3_rn(T a, T b, T c) {
  return add_rn(add_rn(mul_rn(a, a), mul_rn(b, b)), mul_rn(c, c));
}

// Warp-level inclusive sum.
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void atomic_add(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(float* p, float v) { atomicAdd(p, v); }

// Adds the nine per-lane partial sums vs of every warp of the block to
// out[0..8] with one atomic per component and block: a warp butterfly, then
// the NW warps' sums through shared memory. Every thread of the block must
// call it (it synchronises the block).
template <int NW, typename T>
__device__ __forceinline__ void block_add9(const T (&vs)[9], T* out) {
  __shared__ T s9[NW][9];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const T s = warp_sum(vs[k]);
    if (lane == 0) s9[w][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    T t = (T)0.;
#pragma unroll
    for (int q = 0; q < NW; ++q) t += s9[q][threadIdx.x];
    atomic_add(&out[threadIdx.x], t);
  }
}

// SM count of the current device (looked up once per process)
inline int sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    sms = n;
  }
  return sms;
}

// Blocks for a grid-stride kernel of `per_block` items per block pass: the
// item count, capped at 8 blocks per SM.
inline int grid_stride_blocks(long long items, int per_block) {
  const int sms = sm_count();
  const long long need = (items + per_block - 1) / per_block;
  return (int)(need < (long long)sms * 8 ? need : (long long)sms * 8);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---- programmatic dependent launch -----------------------------------------
// Kernels launched by launch_pdl may be scheduled while the previous kernel of
// the stream drains (its CTAs have all started and triggered): their launch
// latency and set-up overlap that kernel's tail. Such a kernel calls
// pdl_wait() before it touches global memory: the wait returns once the
// previous kernel has completed and its writes are visible (immediately when
// the kernel was launched without the attribute). pdl_trigger() lets the next
// kernel be scheduled once every CTA of this one has called it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launch of a kernel that starts with pdl_wait(); the attribute is dropped
// when the pdl knob is 0.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = tune_value("pdl", 1) != 0 ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace dpb
