// Fused se_e2_a descriptor pipeline for one energy/force/virial evaluation.
//
//  desc_fwd : for every center atom, the compressed embedding of all neighbor
//             types (one table per neighbor type, type_one_side), the sorted
//             padding fold per type block, xyz = (sum_t G_t^T R_t) / nnei, and
//             the descriptor D[m, a] = sum_k xyz[k, m] xyz[k, a], a < axis
//             (deepmd/pt/model/descriptor/se_a.py:804-851, with the table op
//             of source/lib/src/tabulate.cc:162-232 applied per type block).
//  desc_bwd : the adjoint: dD -> dxyz -> per-type table gradient
//             (tabulate.cc:234-341) -> net_deriv = dE/d(em) with the em_x
//             gradient folded into column 0 (se_a.py:823 feeds em[..., 0]
//             to the table).
//  force_virial : prod_force_a + prod_virial_a (prod_force.cc:23-72,
//             prod_virial.cc:22-69) in one pass, ghost forces folded onto
//             their owners through `mapping` (make_model.py:216-221), force and
//             virial accumulated in FP64.
//
// D rows are written at descrpt_row[i] so the caller can group atoms by type
// for the per-type fitting networks without a gather.
#include <math.h>

#include "dpb_common.cuh"
#include "dpb_internal.cuh"

namespace dpb {

constexpr int SW = 4;         // warps per block
constexpr int MAXM = 128;     // embedding width handled by one warp (4 x 32)
constexpr int MAXAX = 16;     // axis_neuron
constexpr int PMAXT = 8;      // neighbor types in the fused pipeline
constexpr int PNMAX = 512;

struct FTab {
  float lower, upper, max, s0, s1;
  int first, high_idx;
};

struct TypeTables {
  const float* table[PMAXT];
  FTab info[PMAXT];
  int sec[PMAXT + 1];
  int ntypes;
  int nnei;
};

__device__ __forceinline__ void flocate(const FTab& t, float x, int& idx, float& xx,
                                        float& delta) {
  delta = 0.f;
  if (x < t.lower) {
    idx = 0;
    xx = 0.f;
    delta = x - t.lower;
  } else if (x < t.upper) {
    idx = (int)((x - t.lower) / t.s0);
    xx = x - ((float)idx * t.s0 + t.lower);
  } else if (x < t.max) {
    idx = t.first + (int)((x - t.upper) / t.s1);
    xx = x - ((float)(idx - t.first) * t.s1 + t.upper);
  } else {
    idx = t.high_idx;
    xx = t.max - ((float)(idx - t.first) * t.s1 + t.upper);
    delta = x - t.max;
  }
}

__device__ __forceinline__ void fpoly(const float* p, float xx, float delta, float& v,
                                      float& g) {
  const float2* q = reinterpret_cast<const float2*>(p);
  float2 A = __ldg(q), B = __ldg(q + 1), C = __ldg(q + 2);
  g = A.y + (2.f * B.x + (3.f * B.y + (4.f * C.x + 5.f * C.y * xx) * xx) * xx) * xx;
  v = A.x + (A.y + (B.x + (B.y + (C.x + C.y * xx) * xx) * xx) * xx) * xx;
  v = v + g * delta;
}

// first slot q in [0, n) of a type block whose em_x equals the block's last
// and whose em[1..3] are zero; n when there is none
__device__ __forceinline__ int block_fold(const float4* e4, int n, int lane) {
  if (n <= 0) return 0;
  const float last = e4[n - 1].x;
  for (int base = 0; base < n; base += 32) {
    int q = base + lane;
    bool c = false;
    if (q < n) {
      float4 e = e4[q];
      c = e.x == last && e.y == 0.f && e.z == 0.f && e.w == 0.f;
    }
    unsigned b = __ballot_sync(0xffffffffu, c);
    if (b) return base + __ffs(b) - 1;
  }
  return n;
}

template <int MC>
__global__ void __launch_bounds__(SW * 32)
k_desc_fwd(float* __restrict__ xyz_out, float* __restrict__ D,
           const int* __restrict__ drow, const float* __restrict__ em,
           TypeTables tt, int nloc, int M, int naxis, float inv_nnei) {
  __shared__ float s_x[SW][4][MAXM];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SW + w;
  if (i >= nloc) return;
  const int nnei = tt.nnei;
  float acc[MC][4];
#pragma unroll
  for (int c = 0; c < MC; ++c)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[c][k] = 0.f;
  const float4* erow = reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4);
  for (int t = 0; t < tt.ntypes; ++t) {
    const int s0 = tt.sec[t], nt = tt.sec[t + 1] - s0;
    if (nt <= 0) continue;
    const float4* e4 = erow + s0;
    const int brk = block_fold(e4, nt, lane);
    const float* tab = tt.table[t];
    const FTab inf = tt.info[t];
    for (int q = 0; q < nt; ++q) {
      const float4 e = e4[q];
      int idx;
      float xx, delta;
      flocate(inf, e.x, idx, xx, delta);
      const float rep = q == brk ? (float)(nt - q) : 1.f;
      const float* row = tab + (size_t)idx * M * 6;
#pragma unroll
      for (int c = 0; c < MC; ++c) {
        const int m = c * 32 + lane;
        if (m < M) {
          float v, g;
          fpoly(row + m * 6, xx, delta, v, g);
          const float sc = rep * v;
          acc[c][0] += sc * e.x;
          acc[c][1] += sc * e.y;
          acc[c][2] += sc * e.z;
          acc[c][3] += sc * e.w;
        }
      }
      if (q == brk) break;
    }
  }
  float* xo = xyz_out + (size_t)i * 4 * M;
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    const int m = c * 32 + lane;
    if (m < M) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float v = acc[c][k] * inv_nnei;
        s_x[w][k][m] = v;
        xo[k * M + m] = v;
      }
    }
  }
  __syncwarp();
  float* Dr = D + (size_t)drow[i] * M * naxis;
  const int nd = M * naxis;
  for (int q = lane; q < nd; q += 32) {
    const int m = q / naxis, a = q - m * naxis;
    Dr[q] = s_x[w][0][m] * s_x[w][0][a] + s_x[w][1][m] * s_x[w][1][a] +
            s_x[w][2][m] * s_x[w][2][a] + s_x[w][3][m] * s_x[w][3][a];
  }
}

template <int MC>
__global__ void __launch_bounds__(SW * 32)
k_desc_bwd(float* __restrict__ net_deriv, const float* __restrict__ dD,
           const int* __restrict__ drow, const float* __restrict__ xyz,
           const float* __restrict__ em, TypeTables tt, int nloc, int M, int naxis,
           float inv_nnei) {
  __shared__ float s_x[SW][4][MAXM];
  __shared__ float s_d[SW][MAXM * (MAXAX + 1)];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SW + w;
  if (i >= nloc) return;
  const int nnei = tt.nnei;
  const float* xi = xyz + (size_t)i * 4 * M;
  for (int q = lane; q < 4 * M; q += 32) s_x[w][q / M][q % M] = xi[q];
  const float* dr = dD + (size_t)drow[i] * M * naxis;
  const int ldd = naxis + 1;  // padded row: conflict-free column reads
  for (int q = lane; q < M * naxis; q += 32) {
    const int m = q / naxis, a = q - m * naxis;
    s_d[w][m * ldd + a] = dr[q];
  }
  __syncwarp();
  // dxyz[k, m] = sum_a dD[m, a] x[k, a] + [m < naxis] sum_m' dD[m', m] x[k, m']
  float dyr[MC][4];
#pragma unroll
  for (int c = 0; c < MC; ++c) {
    const int m = c * 32 + lane;
    float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
    if (m < M) {
      for (int a = 0; a < naxis; ++a) {
        const float g = s_d[w][m * ldd + a];
        d0 += g * s_x[w][0][a];
        d1 += g * s_x[w][1][a];
        d2 += g * s_x[w][2][a];
        d3 += g * s_x[w][3][a];
      }
      if (m < naxis) {
        for (int mp = 0; mp < M; ++mp) {
          const float g = s_d[w][mp * ldd + m];
          d0 += g * s_x[w][0][mp];
          d1 += g * s_x[w][1][mp];
          d2 += g * s_x[w][2][mp];
          d3 += g * s_x[w][3][mp];
        }
      }
    }
    dyr[c][0] = d0 * inv_nnei;
    dyr[c][1] = d1 * inv_nnei;
    dyr[c][2] = d2 * inv_nnei;
    dyr[c][3] = d3 * inv_nnei;
  }
  const float4* erow = reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4);
  float4* nrow = reinterpret_cast<float4*>(net_deriv + (size_t)i * nnei * 4);
  for (int t = 0; t < tt.ntypes; ++t) {
    const int s0 = tt.sec[t], nt = tt.sec[t + 1] - s0;
    if (nt <= 0) continue;
    const float4* e4 = erow + s0;
    const int brk = block_fold(e4, nt, lane);
    const int last = brk < nt ? brk : nt - 1;
    const float* tab = tt.table[t];
    const FTab inf = tt.info[t];
    for (int base = 0; base < nt; base += 32) {
      float4 keep = make_float4(0.f, 0.f, 0.f, 0.f);
      const int cnt = (last + 1 - base) < 32 ? (last + 1 - base) : 32;
      for (int q = 0; q < cnt; ++q) {
        const int qq = base + q;
        const float4 e = e4[qq];
        int idx;
        float xx, delta;
        flocate(inf, e.x, idx, xx, delta);
        const float* row = tab + (size_t)idx * M * 6;
        float px = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
#pragma unroll
        for (int c = 0; c < MC; ++c) {
          const int m = c * 32 + lane;
          if (m < M) {
            float v, g;
            fpoly(row + m * 6, xx, delta, v, g);
            const float dot = e.x * dyr[c][0] + e.y * dyr[c][1] + e.z * dyr[c][2] +
                              e.w * dyr[c][3];
            px += g * dot;
            p0 += v * dyr[c][0];
            p1 += v * dyr[c][1];
            p2 += v * dyr[c][2];
            p3 += v * dyr[c][3];
          }
        }
        px = warp_sum(px);
        p0 = warp_sum(p0);
        p1 = warp_sum(p1);
        p2 = warp_sum(p2);
        p3 = warp_sum(p3);
        const float rep = qq == brk ? (float)(nt - qq) : 1.f;
        if (lane == q) keep = make_float4((p0 + px) * rep, p1 * rep, p2 * rep, p3 * rep);
      }
      const int qq = base + lane;
      if (qq < nt) nrow[s0 + qq] = keep;  // zero beyond the fold point
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(SW * 32)
k_force_virial(double* __restrict__ force, double* __restrict__ virial,
               double* __restrict__ atom_virial, const T* __restrict__ nd,
               const T* __restrict__ ed, const T* __restrict__ rij,
               const int* __restrict__ nlist, const int* __restrict__ mapping,
               int nloc, int nnei) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SW + w;
  if (i >= nloc) return;
  const T* ndr = nd + (size_t)i * nnei * 4;
  const T* edr = ed + (size_t)i * nnei * 12;
  const T* rr = rij + (size_t)i * nnei * 3;
  double c0 = 0., c1 = 0., c2 = 0.;
  double vs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vs[k] = 0.;
  for (int jj = lane; jj < nnei; jj += 32) {
    T p[3] = {(T)0., (T)0., (T)0.};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const T n = ndr[jj * 4 + a];
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += n * edr[(jj * 4 + a) * 3 + d];
    }
    const double q0 = (double)p[0], q1 = (double)p[1], q2 = (double)p[2];
    c0 += q0;
    c1 += q1;
    c2 += q2;
    const int j = nlist[(size_t)i * nnei + jj];
    if (j >= 0) {
      const int o = mapping ? mapping[j] : j;
      atomicAdd(&force[(size_t)o * 3 + 0], q0);
      atomicAdd(&force[(size_t)o * 3 + 1], q1);
      atomicAdd(&force[(size_t)o * 3 + 2], q2);
      const double r[3] = {(double)rr[jj * 3 + 0], (double)rr[jj * 3 + 1],
                           (double)rr[jj * 3 + 2]};
      const double q[3] = {q0, q1, q2};
#pragma unroll
      for (int d0 = 0; d0 < 3; ++d0)
#pragma unroll
        for (int d1 = 0; d1 < 3; ++d1) {
          const double v = q[d0] * r[d1];
          vs[d0 * 3 + d1] += v;
          if (atom_virial) atomicAdd(&atom_virial[(size_t)j * 9 + d0 * 3 + d1], v);
        }
    }
  }
  c0 = warp_sum(c0);
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  if (lane == 0) {
    atomicAdd(&force[(size_t)i * 3 + 0], -c0);
    atomicAdd(&force[(size_t)i * 3 + 1], -c1);
    atomicAdd(&force[(size_t)i * 3 + 2], -c2);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double s = warp_sum(vs[k]);
    if (lane == 0) atomicAdd(&virial[k], s);
  }
}

static int make_tables(TypeTables& tt, const float* const* tables, const float* info,
                       const int* sec, int nsec, int M) {
  if (nsec < 2 || nsec - 1 > PMAXT || tables == nullptr || info == nullptr || sec == nullptr) {
    set_error("se_a pipeline: need 1..%d neighbor types with tables, info and sec", PMAXT);
    return DPB_ERR_INVALID;
  }
  if (M <= 0 || M > MAXM) {
    set_error("se_a pipeline: last_layer_size must be in [1, %d], got %d", MAXM, M);
    return DPB_ERR_INVALID;
  }
  tt.ntypes = nsec - 1;
  for (int k = 0; k < nsec; ++k) tt.sec[k] = sec[k];
  tt.nnei = sec[nsec - 1];
  if (sec[0] != 0 || tt.nnei > PNMAX) {
    set_error("se_a pipeline: invalid sec (sec[0]=%d, sum(sel)=%d)", sec[0], tt.nnei);
    return DPB_ERR_INVALID;
  }
  for (int t = 0; t < tt.ntypes; ++t) {
    if (sec[t + 1] < sec[t]) {
      set_error("se_a pipeline: sec must be non-decreasing");
      return DPB_ERR_INVALID;
    }
    tt.table[t] = tables[t];
    const float* f = info + 6 * t;
    FTab& x = tt.info[t];
    x.lower = f[0];
    x.upper = f[1];
    x.max = f[2];
    x.s0 = f[3];
    x.s1 = f[4];
    x.first = (int)((x.upper - x.lower) / x.s0);
    x.high_idx = x.first + (int)((nextafterf(x.max, x.lower) - x.upper) / x.s1);
  }
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_copy_coord_async_f64(double* out_c, int* out_t, int* mapping, int* nall_dev,
                             void* scratch, long long scratch_bytes, const double* in_c,
                             const int* in_t, int nloc, int mem_nall, float rcut,
                             const double* boxt, dpb_stream_t stream) {
  return copy_coord_async<double>(out_c, out_t, mapping, nall_dev, scratch, scratch_bytes,
                                  in_c, in_t, nloc, mem_nall, rcut, boxt, as_stream(stream));
}

int dpb_cell_grid_build_async_f64(void* grid, long long grid_bytes_, const double* coord,
                                  int mem_nall, const int* nall_dev, float rcut,
                                  dpb_stream_t stream) {
  return grid_build<double>(grid, grid_bytes_, coord, mem_nall, nall_dev, rcut,
                            as_stream(stream));
}

int dpb_se_a_descriptor_fwd_f32(float* xyz, float* descrpt, const int* descrpt_row,
                                const float* em, const float* const* tables,
                                const float* table_info, const int* sec, int nsec,
                                int nloc, int last_layer_size, int axis_neuron,
                                dpb_stream_t stream) {
  TypeTables tt;
  int rc = make_tables(tt, tables, table_info, sec, nsec, last_layer_size);
  if (rc) return rc;
  if (axis_neuron <= 0 || axis_neuron > MAXAX || axis_neuron > last_layer_size) {
    set_error("se_a descriptor: axis_neuron must be in [1, min(%d, M)]", MAXAX);
    return DPB_ERR_INVALID;
  }
  if (nloc <= 0) return DPB_OK;
  const int M = last_layer_size;
  const float inv = tt.nnei > 0 ? 1.f / (float)tt.nnei : 0.f;
  cudaStream_t st = as_stream(stream);
  dim3 g(ceil_div(nloc, SW));
  if (M <= 32) k_desc_fwd<1><<<g, SW * 32, 0, st>>>(xyz, descrpt, descrpt_row, em, tt, nloc, M, axis_neuron, inv);
  else if (M <= 64) k_desc_fwd<2><<<g, SW * 32, 0, st>>>(xyz, descrpt, descrpt_row, em, tt, nloc, M, axis_neuron, inv);
  else if (M <= 96) k_desc_fwd<3><<<g, SW * 32, 0, st>>>(xyz, descrpt, descrpt_row, em, tt, nloc, M, axis_neuron, inv);
  else k_desc_fwd<4><<<g, SW * 32, 0, st>>>(xyz, descrpt, descrpt_row, em, tt, nloc, M, axis_neuron, inv);
  DPB_CHECK_LAUNCH("se_a_descriptor_fwd");
  return DPB_OK;
}

int dpb_se_a_descriptor_bwd_f32(float* net_deriv, const float* d_descrpt,
                                const int* descrpt_row, const float* xyz, const float* em,
                                const float* const* tables, const float* table_info,
                                const int* sec, int nsec, int nloc, int last_layer_size,
                                int axis_neuron, dpb_stream_t stream) {
  TypeTables tt;
  int rc = make_tables(tt, tables, table_info, sec, nsec, last_layer_size);
  if (rc) return rc;
  if (axis_neuron <= 0 || axis_neuron > MAXAX || axis_neuron > last_layer_size) {
    set_error("se_a descriptor: axis_neuron must be in [1, min(%d, M)]", MAXAX);
    return DPB_ERR_INVALID;
  }
  if (nloc <= 0) return DPB_OK;
  const int M = last_layer_size;
  const float inv = tt.nnei > 0 ? 1.f / (float)tt.nnei : 0.f;
  cudaStream_t st = as_stream(stream);
  dim3 g(ceil_div(nloc, SW));
  if (M <= 32) k_desc_bwd<1><<<g, SW * 32, 0, st>>>(net_deriv, d_descrpt, descrpt_row, xyz, em, tt, nloc, M, axis_neuron, inv);
  else if (M <= 64) k_desc_bwd<2><<<g, SW * 32, 0, st>>>(net_deriv, d_descrpt, descrpt_row, xyz, em, tt, nloc, M, axis_neuron, inv);
  else if (M <= 96) k_desc_bwd<3><<<g, SW * 32, 0, st>>>(net_deriv, d_descrpt, descrpt_row, xyz, em, tt, nloc, M, axis_neuron, inv);
  else k_desc_bwd<4><<<g, SW * 32, 0, st>>>(net_deriv, d_descrpt, descrpt_row, xyz, em, tt, nloc, M, axis_neuron, inv);
  DPB_CHECK_LAUNCH("se_a_descriptor_bwd");
  return DPB_OK;
}

int dpb_force_virial_a_f32(double* force, double* virial, double* atom_virial,
                           const float* net_deriv, const float* env_deriv, const float* rij,
                           const int* nlist, const int* mapping, int nloc, int nforce,
                           int nall, int nnei, dpb_stream_t stream) {
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * 3 * (size_t)nforce, st), "force_virial");
  DPB_CUDA(cudaMemsetAsync(virial, 0, sizeof(double) * 9, st), "force_virial");
  if (atom_virial)
    DPB_CUDA(cudaMemsetAsync(atom_virial, 0, sizeof(double) * 9 * (size_t)nall, st),
             "force_virial");
  if (nloc <= 0 || nnei <= 0) return DPB_OK;
  k_force_virial<float><<<ceil_div(nloc, SW), SW * 32, 0, st>>>(
      force, virial, atom_virial, net_deriv, env_deriv, rij, nlist, mapping, nloc, nnei);
  DPB_CHECK_LAUNCH("force_virial");
  return DPB_OK;
}

int dpb_force_virial_a_f64(double* force, double* virial, double* atom_virial,
                           const double* net_deriv, const double* env_deriv,
                           const double* rij, const int* nlist, const int* mapping,
                           int nloc, int nforce, int nall, int nnei, dpb_stream_t stream) {
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * 3 * (size_t)nforce, st), "force_virial");
  DPB_CUDA(cudaMemsetAsync(virial, 0, sizeof(double) * 9, st), "force_virial");
  if (atom_virial)
    DPB_CUDA(cudaMemsetAsync(atom_virial, 0, sizeof(double) * 9 * (size_t)nall, st),
             "force_virial");
  if (nloc <= 0 || nnei <= 0) return DPB_OK;
  k_force_virial<double><<<ceil_div(nloc, SW), SW * 32, 0, st>>>(
      force, virial, atom_virial, net_deriv, env_deriv, rij, nlist, mapping, nloc, nnei);
  DPB_CHECK_LAUNCH("force_virial");
  return DPB_OK;
}

}  // extern "C"
