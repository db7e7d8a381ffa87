// Compressed se_a embedding: the quintic table G_m(x) fused with the
// contraction over neighbors (tabulate_fusion_se_a and its two gradients).
//
// Layout: one warp per (center atom, block of up to 128 embedding channels m);
// lane l owns channels m = mb + 32c + l. A neighbor's table row is read once
// per warp as contiguous 24-byte (FP32) / 48-byte (FP64) coefficient groups,
// so a warp-wide load covers a contiguous 768 B / 1.5 KB span of the row.
// The forward and grad_grad accumulate over neighbors in registers; the
// gradient reduces over channels with a butterfly and keeps the result in the
// lane that owns the neighbor, flushing 32 neighbors per coalesced store.
//
// Semantics follow the CPU reference (source/lib/src/tabulate.cc): locate_xx
// (:45-73) with the nextafter upper bound (:21-30), linear extrapolation
// outside the table (:133-144), and the sorted-padding fold (:184-189): the
// first slot whose em_x equals the last slot's and whose em[1..3] are zero is
// weighted by (nnei - slot) and ends the loop.
#include <math.h>

#include "dpb_common.cuh"

namespace dpb {

template <typename T>
struct TabInfo {
  T lower, upper, max, s0, s1;
  int first;     // int((upper - lower) / stride0)
  int high_idx;  // locate_high_tail_xx
};

template <typename T>
static int make_info(TabInfo<T>& t, const T* info, int M) {
  if (info == nullptr) {
    set_error("table_info is required (host pointer, 6 values)");
    return DPB_ERR_INVALID;
  }
  if (M <= 0 || M > 1024) {
    set_error("last_layer_size must be between 1 and 1024 for GPU tabulation, but got %d", M);
    return DPB_ERR_INVALID;
  }
  t.lower = info[0];
  t.upper = info[1];
  t.max = info[2];
  t.s0 = info[3];
  t.s1 = info[4];
  t.first = (int)((t.upper - t.lower) / t.s0);
  T bxx = (sizeof(T) == 8) ? (T)nextafter((double)t.max, (double)t.lower)
                           : (T)nextafterf((float)t.max, (float)t.lower);
  t.high_idx = t.first + (int)((bxx - t.upper) / t.s1);
  return DPB_OK;
}

template <typename T>
__device__ __forceinline__ void locate(const TabInfo<T>& t, T x, int& idx, T& xx,
                                       T& delta) {
  delta = (T)0.;
  if (x < t.lower) {
    idx = 0;
    xx = (T)0.;
    delta = x - t.lower;
  } else if (x < t.upper) {
    idx = (int)((x - t.lower) / t.s0);
    xx = x - ((T)idx * t.s0 + t.lower);
  } else if (x < t.max) {
    idx = t.first + (int)((x - t.upper) / t.s1);
    xx = x - ((T)(idx - t.first) * t.s1 + t.upper);
  } else {
    idx = t.high_idx;
    xx = t.max - ((T)(idx - t.first) * t.s1 + t.upper);
    delta = x - t.max;
  }
}

template <typename T>
struct Coef {
  T a0, a1, a2, a3, a4, a5;
};

__device__ __forceinline__ Coef<float> load_coef(const float* p) {
  const float2* q = reinterpret_cast<const float2*>(p);
  float2 x = __ldg(q), y = __ldg(q + 1), z = __ldg(q + 2);
  return {x.x, x.y, y.x, y.y, z.x, z.y};
}
__device__ __forceinline__ Coef<double> load_coef(const double* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 x = __ldg(q), y = __ldg(q + 1), z = __ldg(q + 2);
  return {x.x, x.y, y.x, y.y, z.x, z.y};
}

// value (with extrapolation) and derivative of the quintic (tabulate.cc:116-144)
template <typename T>
__device__ __forceinline__ void poly(const Coef<T>& a, T xx, T delta, T& v, T& g) {
  g = a.a1 + ((T)2. * a.a2 + ((T)3. * a.a3 + ((T)4. * a.a4 + (T)5. * a.a5 * xx) * xx) * xx) * xx;
  v = a.a0 + (a.a1 + (a.a2 + (a.a3 + (a.a4 + a.a5 * xx) * xx) * xx) * xx) * xx;
  v = v + g * delta;
}

// First slot of the sorted padding tail, or nnei when there is none.
template <typename T>
__device__ __forceinline__ int fold_start(const T* em_x, const T* em, int nnei, int lane) {
  const T last = em_x[nnei - 1];
  for (int base = 0; base < nnei; base += 32) {
    int jj = base + lane;
    bool c = false;
    if (jj < nnei) {
      const T* e = em + (size_t)jj * 4;
      c = em_x[jj] == last && e[1] == (T)0. && e[2] == (T)0. && e[3] == (T)0.;
    }
    unsigned b = __ballot_sync(0xffffffffu, c);
    if (b) return base + __ffs(b) - 1;
  }
  return nnei;
}

constexpr int TW = 4;  // warps per block

template <typename T, int MC>
__global__ void __launch_bounds__(TW * 32)
k_tab_fwd(T* __restrict__ out, const T* __restrict__ table, TabInfo<T> ti,
          const T* __restrict__ em_x, const T* __restrict__ em, int nloc,
          int nnei, int M, const T* __restrict__ dz_dem_x,
          const T* __restrict__ dz_dem) {
  // out[i,k,m] = sum_jj w_jj * (G_m(x_jj) * em[jj,k])              (forward)
  // out[i,k,m] = sum_jj w_jj * (G_m * dz_dem[jj,k] + dz_dem_x[jj] * G'_m * em[jj,k])
  //                                                   (grad_grad, dz_* != NULL)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * TW + w;
  if (i >= nloc) return;
  const int m0 = blockIdx.y * 32 * MC;
  const bool gg = dz_dem != nullptr;
  T acc[MC][4];
#pragma unroll
  for (int c = 0; c < MC; ++c)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[c][k] = (T)0.;
  const T* ex = em_x + (size_t)i * nnei;
  const T* ee = em + (size_t)i * nnei * 4;
  const int brk = nnei > 0 ? fold_start(ex, ee, nnei, lane) : 0;
  for (int jj = 0; jj < nnei; ++jj) {
    const T x = ex[jj];
    T e[4] = {ee[jj * 4 + 0], ee[jj * 4 + 1], ee[jj * 4 + 2], ee[jj * 4 + 3]};
    T h[4] = {(T)0., (T)0., (T)0., (T)0.}, dzx = (T)0.;
    if (gg) {
      const T* hz = dz_dem + ((size_t)i * nnei + jj) * 4;
      h[0] = hz[0]; h[1] = hz[1]; h[2] = hz[2]; h[3] = hz[3];
      dzx = dz_dem_x[(size_t)i * nnei + jj];
    }
    int idx;
    T xx, delta;
    locate(ti, x, idx, xx, delta);
    const T rep = jj == brk ? (T)(nnei - jj) : (T)1.;
    const T* row = table + (size_t)idx * M * 6;
#pragma unroll
    for (int c = 0; c < MC; ++c) {
      const int m = m0 + c * 32 + lane;
      if (m < M) {
        Coef<T> a = load_coef(row + (size_t)m * 6);
        T v, g;
        poly(a, xx, delta, v, g);
        if (!gg) {
          const T sc = rep * v;
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[c][k] += sc * e[k];
        } else {
          const T dg = dzx * g;
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[c][k] += rep * (v * h[k] + dg * e[k]);
        }
      }
    }
    if (jj == brk) break;
  }
  T* o = out + (size_t)i * 4 * M;
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    const int m = m0 + c * 32 + lane;
    if (m < M) {
#pragma unroll
      for (int k = 0; k < 4; ++k) o[k * M + m] = acc[c][k];
    }
  }
}

template <typename T, int MC>
__global__ void __launch_bounds__(TW * 32)
k_tab_grad(T* __restrict__ dy_dem_x, T* __restrict__ dy_dem,
           const T* __restrict__ table, TabInfo<T> ti,
           const T* __restrict__ em_x, const T* __restrict__ em,
           const T* __restrict__ dy, int nloc, int nnei, int M) {
  // dy_dem_x[i,jj] = sum_m G'_m * sum_k em[jj,k] dy[k,m]
  // dy_dem[i,jj,k] = sum_m G_m * dy[k,m]           (tabulate.cc:234-341)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * TW + w;
  if (i >= nloc) return;
  const T* ex = em_x + (size_t)i * nnei;
  const T* ee = em + (size_t)i * nnei * 4;
  const T* dyi = dy + (size_t)i * 4 * M;
  T* ox = dy_dem_x + (size_t)i * nnei;
  T* oe = dy_dem + (size_t)i * nnei * 4;
  const int brk = fold_start(ex, ee, nnei, lane);
  const int last = brk < nnei ? brk : nnei - 1;
  const int nmb = (M + 32 * MC - 1) / (32 * MC);
  for (int mb = 0; mb < nmb; ++mb) {
    const int m0 = mb * 32 * MC;
    T dyr[MC][4];
#pragma unroll
    for (int c = 0; c < MC; ++c) {
      const int m = m0 + c * 32 + lane;
#pragma unroll
      for (int k = 0; k < 4; ++k) dyr[c][k] = m < M ? dyi[k * M + m] : (T)0.;
    }
    for (int base = 0; base <= last; base += 32) {
      T kx = (T)0., kk4[4] = {(T)0., (T)0., (T)0., (T)0.};
      const int cnt = (last + 1 - base) < 32 ? (last + 1 - base) : 32;
      for (int q = 0; q < cnt; ++q) {
        const int jj = base + q;
        const T x = ex[jj];
        T e[4] = {ee[jj * 4 + 0], ee[jj * 4 + 1], ee[jj * 4 + 2], ee[jj * 4 + 3]};
        int idx;
        T xx, delta;
        locate(ti, x, idx, xx, delta);
        const T* row = table + (size_t)idx * M * 6;
        T px = (T)0., pk[4] = {(T)0., (T)0., (T)0., (T)0.};
#pragma unroll
        for (int c = 0; c < MC; ++c) {
          const int m = m0 + c * 32 + lane;
          if (m < M) {
            Coef<T> a = load_coef(row + (size_t)m * 6);
            T v, g;
            poly(a, xx, delta, v, g);
            T dot = e[0] * dyr[c][0] + e[1] * dyr[c][1] + e[2] * dyr[c][2] + e[3] * dyr[c][3];
            px += g * dot;
#pragma unroll
            for (int k = 0; k < 4; ++k) pk[k] += v * dyr[c][k];
          }
        }
        px = warp_sum(px);
#pragma unroll
        for (int k = 0; k < 4; ++k) pk[k] = warp_sum(pk[k]);
        const T rep = jj == brk ? (T)(nnei - jj) : (T)1.;
        if (lane == q) {
          kx = px * rep;
#pragma unroll
          for (int k = 0; k < 4; ++k) kk4[k] = pk[k] * rep;
        }
      }
      const int jj = base + lane;
      if (lane < cnt) {
        if (mb == 0) {
          ox[jj] = kx;
#pragma unroll
          for (int k = 0; k < 4; ++k) oe[jj * 4 + k] = kk4[k];
        } else {
          ox[jj] += kx;
#pragma unroll
          for (int k = 0; k < 4; ++k) oe[jj * 4 + k] += kk4[k];
        }
      }
    }
  }
  // slots after the fold point keep the zero of the reference's memset
  for (int jj = last + 1 + lane; jj < nnei; jj += 32) {
    ox[jj] = (T)0.;
#pragma unroll
    for (int k = 0; k < 4; ++k) oe[jj * 4 + k] = (T)0.;
  }
}

template <typename T, int MC>
static void launch_fwd(T* out, const T* table, const TabInfo<T>& ti, const T* em_x,
                       const T* em, int nloc, int nnei, int M, const T* dzx,
                       const T* dze, cudaStream_t st) {
  dim3 grid(ceil_div(nloc, TW), ceil_div(M, 32 * MC));
  k_tab_fwd<T, MC><<<grid, TW * 32, 0, st>>>(out, table, ti, em_x, em, nloc, nnei, M,
                                             dzx, dze);
}

template <typename T>
static int tab_fwd(T* out, const T* table, const T* info, const T* em_x,
                   const T* em, int nloc, int nnei, int M, const T* dzx,
                   const T* dze, cudaStream_t st, const char* name) {
  TabInfo<T> ti;
  int rc = make_info(ti, info, M);
  if (rc) return rc;
  if (nloc < 0 || nnei < 0) {
    set_error("%s: negative sizes", name);
    return DPB_ERR_INVALID;
  }
  if (nloc == 0) return DPB_OK;
  if (nnei == 0) {
    // an empty neighbor axis is a valid empty reduction (tabulate.cc:173-179)
    DPB_CUDA(cudaMemsetAsync(out, 0, sizeof(T) * (size_t)nloc * 4 * M, st), name);
    return DPB_OK;
  }
  if (M <= 32) launch_fwd<T, 1>(out, table, ti, em_x, em, nloc, nnei, M, dzx, dze, st);
  else if (M <= 64) launch_fwd<T, 2>(out, table, ti, em_x, em, nloc, nnei, M, dzx, dze, st);
  else if (M <= 96) launch_fwd<T, 3>(out, table, ti, em_x, em, nloc, nnei, M, dzx, dze, st);
  else launch_fwd<T, 4>(out, table, ti, em_x, em, nloc, nnei, M, dzx, dze, st);
  DPB_CHECK_LAUNCH(name);
  return DPB_OK;
}

template <typename T>
static int tab_grad(T* dy_dem_x, T* dy_dem, const T* table, const T* info,
                    const T* em_x, const T* em, const T* dy, int nloc, int nnei,
                    int M, cudaStream_t st) {
  TabInfo<T> ti;
  int rc = make_info(ti, info, M);
  if (rc) return rc;
  if (nloc < 0 || nnei < 0) {
    set_error("tabulate_fusion_se_a_grad: negative sizes");
    return DPB_ERR_INVALID;
  }
  if (nloc == 0 || nnei == 0) return DPB_OK;  // tabulate.cc:251-256
  dim3 grid(ceil_div(nloc, TW));
  if (M <= 32) k_tab_grad<T, 1><<<grid, TW * 32, 0, st>>>(dy_dem_x, dy_dem, table, ti, em_x, em, dy, nloc, nnei, M);
  else if (M <= 64) k_tab_grad<T, 2><<<grid, TW * 32, 0, st>>>(dy_dem_x, dy_dem, table, ti, em_x, em, dy, nloc, nnei, M);
  else if (M <= 96) k_tab_grad<T, 3><<<grid, TW * 32, 0, st>>>(dy_dem_x, dy_dem, table, ti, em_x, em, dy, nloc, nnei, M);
  else k_tab_grad<T, 4><<<grid, TW * 32, 0, st>>>(dy_dem_x, dy_dem, table, ti, em_x, em, dy, nloc, nnei, M);
  DPB_CHECK_LAUNCH("tabulate_fusion_se_a_grad");
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_tabulate_fusion_se_a_f64(double* out, const double* table,
                                 const double* table_info, const double* em_x,
                                 const double* em, int nloc, int nnei,
                                 int last_layer_size, dpb_stream_t stream) {
  return tab_fwd<double>(out, table, table_info, em_x, em, nloc, nnei,
                         last_layer_size, nullptr, nullptr, as_stream(stream),
                         "tabulate_fusion_se_a");
}

int dpb_tabulate_fusion_se_a_f32(float* out, const float* table,
                                 const float* table_info, const float* em_x,
                                 const float* em, int nloc, int nnei,
                                 int last_layer_size, dpb_stream_t stream) {
  return tab_fwd<float>(out, table, table_info, em_x, em, nloc, nnei,
                        last_layer_size, nullptr, nullptr, as_stream(stream),
                        "tabulate_fusion_se_a");
}

int dpb_tabulate_fusion_se_a_grad_f64(double* dy_dem_x, double* dy_dem,
                                      const double* table,
                                      const double* table_info,
                                      const double* em_x, const double* em,
                                      const double* dy, int nloc, int nnei,
                                      int last_layer_size,
                                      dpb_stream_t stream) {
  return tab_grad<double>(dy_dem_x, dy_dem, table, table_info, em_x, em, dy,
                          nloc, nnei, last_layer_size, as_stream(stream));
}

int dpb_tabulate_fusion_se_a_grad_f32(float* dy_dem_x, float* dy_dem,
                                      const float* table,
                                      const float* table_info,
                                      const float* em_x, const float* em,
                                      const float* dy, int nloc, int nnei,
                                      int last_layer_size,
                                      dpb_stream_t stream) {
  return tab_grad<float>(dy_dem_x, dy_dem, table, table_info, em_x, em, dy,
                         nloc, nnei, last_layer_size, as_stream(stream));
}

int dpb_tabulate_fusion_se_a_grad_grad_f64(
    double* dz_dy, const double* table, const double* table_info,
    const double* em_x, const double* em, const double* dz_dy_dem_x,
    const double* dz_dy_dem, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream) {
  if (dz_dy_dem_x == nullptr || dz_dy_dem == nullptr) {
    set_error("tabulate_fusion_se_a_grad_grad: dz_dy_dem_x and dz_dy_dem are required");
    return DPB_ERR_INVALID;
  }
  return tab_fwd<double>(dz_dy, table, table_info, em_x, em, nloc, nnei,
                         last_layer_size, dz_dy_dem_x, dz_dy_dem,
                         as_stream(stream), "tabulate_fusion_se_a_grad_grad");
}

int dpb_tabulate_fusion_se_a_grad_grad_f32(
    float* dz_dy, const float* table, const float* table_info,
    const float* em_x, const float* em, const float* dz_dy_dem_x,
    const float* dz_dy_dem, int nloc, int nnei, int last_layer_size,
    dpb_stream_t stream) {
  if (dz_dy_dem_x == nullptr || dz_dy_dem == nullptr) {
    set_error("tabulate_fusion_se_a_grad_grad: dz_dy_dem_x and dz_dy_dem are required");
    return DPB_ERR_INVALID;
  }
  return tab_fwd<float>(dz_dy, table, table_info, em_x, em, nloc, nnei,
                        last_layer_size, dz_dy_dem_x, dz_dy_dem,
                        as_stream(stream), "tabulate_fusion_se_a_grad_grad");
}

}  // extern "C"
