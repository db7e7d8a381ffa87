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

#include <type_traits>

#include "dpb_common.cuh"
#include "dpb_envmath.cuh"
#include "dpb_internal.cuh"
#include "dpb_desc_dev.cuh"

namespace dpb {

template <int SWT, int CH, int NC>
__global__ void __launch_bounds__(SWT * 32, 20 / SWT)
k_desc_fwd(float* __restrict__ xyz_out, float* __restrict__ D,
           const int* __restrict__ drow, const float* __restrict__ em,
           TypeTables tt, int nloc, int M, int naxis, float inv_nnei, int warp_floats) {
  extern __shared__ float4 dsm4[];
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SWT + w;
  if (i >= nloc) return;
  float* wsm = reinterpret_cast<float*>(dsm4) + (size_t)w * warp_floats;
  desc_fwd_atom<CH, NC>(i, lane, wsm, xyz_out, D, drow, em, tt, M, naxis, inv_nnei);
}

// ---- tensor-core variant of the forward contraction (knob desc_tc = 1) ----
// The contraction xyz[k, m] = sum_s e_s[k] G_s[m] as warp-level MMAs
// (mma.sync m16n8k8, TF32 operands, 3xTF32 split for FP32-level products):
// per group of 8 slots and 16 channels, A[m][s] = G_s[m] (each lane evaluates
// the 4 table polynomials of its A-fragment positions: channels g, g + 8 of
// slots t, t + 4, g = lane / 4, t = lane % 4) and B[s][k] = e_s[k] (k < 4,
// columns 4..7 zero). Kept as a measured option next to the CUDA-core
// contraction of k_desc_fwd.
__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4],
                                         const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// G of channel c (< M) at one staged slot L (row, offset, extrapolation
// distance), times the fold multiplier
template <int NC>
__device__ __forceinline__ float g_scalar(const float* tab, size_t rs, int M, int c,
                                          const float4 L, float rep) {
  const float* r = tab + (size_t)__float_as_int(L.x) * rs + c;
  float a[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) a[k] = __ldg(r + k * M);
  const float x = L.y;
  float p = a[NC - 1], d = a[NC - 1];
#pragma unroll
  for (int k = NC - 2; k >= 1; --k) {
    p = fmaf(p, x, a[k]);
    d = fmaf(d, x, p);
  }
  const float v = fmaf(p, x, a[0]);
  return (L.z == 0.f ? v : fmaf(d, L.z, v)) * rep;
}

constexpr int TC_MT = MAXM / 16;  // channel tiles of 16

template <int SWT, int NC>
__global__ void __launch_bounds__(SWT * 32, 20 / SWT)
k_desc_fwd_tc(float* __restrict__ xyz_out, float* __restrict__ D,
              const int* __restrict__ drow, const float* __restrict__ em,
              TypeTables tt, int nloc, int M, int naxis, float inv_nnei, int warp_floats) {
  extern __shared__ float4 dsm4[];
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SWT + w;
  if (i >= nloc) return;
  const int nnei = tt.nnei;
  float* wsm = reinterpret_cast<float*>(dsm4) + (size_t)w * warp_floats;
  float4* se = reinterpret_cast<float4*>(wsm);
  float4* sl = se + nnei;
  stage_slots(se, sl, reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4), tt, lane);
  __syncwarp();
  const int g = lane >> 2, t4 = lane & 3;
  const int ntile = (M + 15) / 16;
  float acc[TC_MT][4];
#pragma unroll
  for (int mt = 0; mt < TC_MT; ++mt)
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[mt][k] = 0.f;
  for (int t = 0; t < tt.ntypes; ++t) {
    const int s0 = tt.sec[t], nt = tt.sec[t + 1] - s0;
    if (nt <= 0) continue;
    const int brk = block_fold(se + s0, nt, lane);
    const int last = brk < nt ? brk : nt - 1;
    const float* tab = tt.table[t];
    const size_t rs = (size_t)M * NC;
    for (int q0 = 0; q0 <= last; q0 += 8) {
      const int qa = q0 + t4, qb = q0 + t4 + 4;
      const bool va = qa <= last, vb = qb <= last;
      // B: e_s[k] of slots qa (row t4) and qb (row t4 + 4), column g
      float eb0 = 0.f, eb1 = 0.f;
      if (g < 4) {
        if (va) eb0 = reinterpret_cast<const float*>(se + s0 + qa)[g];
        if (vb) eb1 = reinterpret_cast<const float*>(se + s0 + qb)[g];
      }
      unsigned bh[2], bl[2];
      split_tf32(eb0, bh[0], bl[0]);
      split_tf32(eb1, bh[1], bl[1]);
      const float4 La = va ? sl[s0 + qa] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 Lb = vb ? sl[s0 + qb] : make_float4(0.f, 0.f, 0.f, 0.f);
      const float ra = qa == brk ? (float)(nt - qa) : 1.f;
      const float rb = qb == brk ? (float)(nt - qb) : 1.f;
#pragma unroll
      for (int mt = 0; mt < TC_MT; ++mt) {
        if (mt >= ntile) break;
        const int c0 = mt * 16 + g, c1 = c0 + 8;
        const float a0 = (va && c0 < M) ? g_scalar<NC>(tab, rs, M, c0, La, ra) : 0.f;
        const float a1 = (va && c1 < M) ? g_scalar<NC>(tab, rs, M, c1, La, ra) : 0.f;
        const float a2 = (vb && c0 < M) ? g_scalar<NC>(tab, rs, M, c0, Lb, rb) : 0.f;
        const float a3 = (vb && c1 < M) ? g_scalar<NC>(tab, rs, M, c1, Lb, rb) : 0.f;
        unsigned ah[4], al[4];
        split_tf32(a0, ah[0], al[0]);
        split_tf32(a1, ah[1], al[1]);
        split_tf32(a2, ah[2], al[2]);
        split_tf32(a3, ah[3], al[3]);
        mma_tf32(acc[mt], ah, bh);
        mma_tf32(acc[mt], al, bh);
        mma_tf32(acc[mt], ah, bl);
      }
    }
  }
  __syncwarp();  // the slot staging is reused for x below
  float* sx = wsm;  // [4][M]
  float* xo = xyz_out + (size_t)i * 4 * M;
  // C fragment: rows (channels) g, g + 8; columns (env components) 2 t4, 2 t4 + 1
  if (t4 < 2) {
#pragma unroll
    for (int mt = 0; mt < TC_MT; ++mt) {
      if (mt >= ntile) break;
      const int c0 = mt * 16 + g, c1 = c0 + 8;
      const int k0 = 2 * t4, k1 = 2 * t4 + 1;
      if (c0 < M) {
        sx[k0 * M + c0] = acc[mt][0] * inv_nnei;
        sx[k1 * M + c0] = acc[mt][1] * inv_nnei;
      }
      if (c1 < M) {
        sx[k0 * M + c1] = acc[mt][2] * inv_nnei;
        sx[k1 * M + c1] = acc[mt][3] * inv_nnei;
      }
    }
  }
  __syncwarp();
  for (int q = lane; q < 4 * M; q += 32) xo[q] = sx[q];
  write_descriptor(D + (size_t)drow[i] * M * naxis, sx, M, naxis, lane);
}


template <int SWT, int CH, int NC>
__global__ void __launch_bounds__(SWT * 32, 20 / SWT)
k_desc_bwd(float* __restrict__ net_deriv, const float* __restrict__ dD,
           const int* __restrict__ drow, const float* __restrict__ xyz,
           const float* __restrict__ em, TypeTables tt, int nloc, int M, int naxis,
           float inv_nnei, int warp_floats) {
  extern __shared__ float4 dsm4[];
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * SWT + w;
  if (i >= nloc) return;
  float* wsm = reinterpret_cast<float*>(dsm4) + (size_t)w * warp_floats;
  desc_bwd_atom<CH, NC>(i, lane, wsm, net_deriv, dD, drow, xyz, em, tt, M, naxis, inv_nnei);
}

template <typename T>
__global__ void __launch_bounds__(SW * 32)
k_force_virial(double* __restrict__ force, double* __restrict__ virial,
               double* __restrict__ atom_virial, const T* __restrict__ nd,
               const T* __restrict__ ed, const T* __restrict__ rij,
               const int* __restrict__ nlist, const int* __restrict__ mapping,
               int nloc, int nnei) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double vs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vs[k] = 0.;
  for (int i = blockIdx.x * SW + w; i < nloc; i += gridDim.x * SW) {
  const T* ndr = nd + (size_t)i * nnei * 4;
  const T* edr = ed + (size_t)i * nnei * 12;
  const T* rr = rij + (size_t)i * nnei * 3;
  double c0 = 0., c1 = 0., c2 = 0.;
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
  }
  block_add9<SW>(vs, virial);
}

// Force and virial with em_deriv and rij recomputed from the coordinates and
// the neighbor list instead of being read back (same formulas and precision
// as the env kernels, dpb_envmath.cuh): the forward pass then stores only em.
template <typename CT, typename OT>
__global__ void __launch_bounds__(SW * 32, sizeof(OT) == 4 ? 24 / SW : 1)
k_force_virial_rc(double* __restrict__ force, double* __restrict__ virial,
                  const OT* __restrict__ nd, const CT* __restrict__ coord,
                  const int* __restrict__ type, const OT* __restrict__ std_,
                  const int* __restrict__ nlist, const int* __restrict__ mapping, int nloc,
                  int nnei, int ntypes, float rcut, float rcut_smth) {
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const OT inv_span = (OT)1. / (OT)(rcut - rcut_smth);
  // grid-stride over center atoms (one warp each); the virial stays in
  // registers across atoms and is reduced once per block, so the nine
  // accumulators see one atomic per block instead of one per atom
  double vs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vs[k] = 0.;
  for (int i = blockIdx.x * SW + w; i < nloc; i += gridDim.x * SW) {
  const int ti = type[i];
  if (ti < 0 || ti >= ntypes) continue;  // em_deriv rows are zero (prod_env_mat.cc:117-123)
  const CT xi[3] = {coord[3 * i], coord[3 * i + 1], coord[3 * i + 2]};
  const OT* sd = std_ + (size_t)ti * nnei * 4;
  const OT* ndr = nd + (size_t)i * nnei * 4;
  double c0 = 0., c1 = 0., c2 = 0.;
  // 16-byte rows of net_deriv and std when both arrays are 16-byte aligned
  const bool vec16 = ((reinterpret_cast<uintptr_t>(ndr) | reinterpret_cast<uintptr_t>(sd)) & 15) == 0;
  const int* nl = nlist + (size_t)i * nnei;
  int jn = lane < nnei ? nl[lane] : -1;  // the next slot's neighbor, requested early
  for (int jj = lane; jj < nnei; jj += 32) {
    const int j = jn;
    jn = jj + 32 < nnei ? nl[jj + 32] : -1;
    if (j < 0) continue;  // padding: em_deriv = 0
    OT r[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[d] = (OT)(coord[3 * j + d] - xi[d]);
    OT nv[4], sv[4];
    if (sizeof(OT) == 4 && vec16) {
      const float4 n4 = *reinterpret_cast<const float4*>(ndr + jj * 4);
      const float4 s4 = *reinterpret_cast<const float4*>(sd + jj * 4);
      nv[0] = n4.x, nv[1] = n4.y, nv[2] = n4.z, nv[3] = n4.w;
      sv[0] = s4.x, sv[1] = s4.y, sv[2] = s4.z, sv[3] = s4.w;
    } else {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        nv[a] = ndr[jj * 4 + a];
        sv[a] = sd[jj * 4 + a];
      }
    }
    OT gd[12];
    env_deriv<OT>(r, rcut_smth, rcut, inv_span, gd);
    // dE/d(env) = net_deriv / std, one division per env column
    OT p[3] = {(OT)0., (OT)0., (OT)0.};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const OT ns = nv[a] / sv[a];
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += ns * gd[a * 3 + d];
    }
    const double q[3] = {(double)p[0], (double)p[1], (double)p[2]};
    c0 += q[0];
    c1 += q[1];
    c2 += q[2];
    const int o = mapping ? mapping[j] : j;
    atomicAdd(&force[(size_t)o * 3 + 0], q[0]);
    atomicAdd(&force[(size_t)o * 3 + 1], q[1]);
    atomicAdd(&force[(size_t)o * 3 + 2], q[2]);
#pragma unroll
    for (int d0 = 0; d0 < 3; ++d0)
#pragma unroll
      for (int d1 = 0; d1 < 3; ++d1) vs[d0 * 3 + d1] += q[d0] * (double)r[d1];
  }
  c0 = warp_sum(c0);
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  if (lane == 0) {
    atomicAdd(&force[(size_t)i * 3 + 0], -c0);
    atomicAdd(&force[(size_t)i * 3 + 1], -c1);
    atomicAdd(&force[(size_t)i * 3 + 2], -c2);
  }
  }
  block_add9<SW>(vs, virial);
}

template <typename CT, typename OT>
static int force_virial_rc(double* force, double* virial, const OT* nd, const CT* coord,
                           const int* type, const OT* std_, const int* nlist,
                           const int* mapping, int nloc, int nforce, int nnei, int ntypes,
                           float rcut, float rcut_smth, cudaStream_t st, bool zero = true) {
  if (nloc < 0 || nforce < 0 || nnei < 0 || ntypes <= 0) {
    set_error("force_virial_env: invalid sizes");
    return DPB_ERR_INVALID;
  }
  if (zero) {
    DPB_CUDA(cudaMemsetAsync(force, 0, sizeof(double) * 3 * (size_t)nforce, st),
             "force_virial");
    DPB_CUDA(cudaMemsetAsync(virial, 0, sizeof(double) * 9, st), "force_virial");
  }
  if (nloc == 0 || nnei == 0) return DPB_OK;
  DPB_CUDA(launch_pdl(k_force_virial_rc<CT, OT>, dim3(grid_stride_blocks(nloc, SW)),
                      dim3(SW * 32), 0, st, force, virial, nd, coord, type, std_, nlist, mapping,
                      nloc, nnei, ntypes, rcut, rcut_smth),
           "force_virial_env");
  return DPB_OK;
}

// [nrow][M][6] (reference layout) -> [nrow][6][M] (pipeline layout)
__global__ void k_pack_table(float* __restrict__ out, const float* __restrict__ in, long long n,
                             int M) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    const long long r = o / (6LL * M);
    const int rem = (int)(o - r * 6LL * M);
    const int k = rem / M, m = rem - k * M;
    out[o] = in[r * 6LL * M + (long long)m * 6 + k];
  }
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

int dpb_se_a_pack_table_f32(float* out, const float* table, int nrow, int M,
                             dpb_stream_t stream) {
  if (nrow < 0 || M <= 0 || (nrow > 0 && (out == nullptr || table == nullptr || out == table))) {
    set_error("se_a_pack_table: invalid arguments (nrow=%d M=%d, out must not alias table)",
              nrow, M);
    return DPB_ERR_INVALID;
  }
  const long long n = 6LL * M * nrow;
  if (n == 0) return DPB_OK;
  const int blocks = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
  k_pack_table<<<blocks, 256, 0, as_stream(stream)>>>(out, table, n, M);
  DPB_CHECK_LAUNCH("se_a_pack_table");
  return DPB_OK;
}

}  // extern "C"

namespace dpb {

template <int NC>
static int desc_fwd(float* xyz, float* descrpt, const int* descrpt_row, const float* em,
                    const float* const* tables, const float* table_info, const int* sec,
                    int nsec, int nloc, int last_layer_size, int axis_neuron,
                    dpb_stream_t stream) {
  TypeTables tt;
  int rc = make_tables(tt, tables, table_info, sec, nsec, last_layer_size, NC == 4);
  if (rc) return rc;
  if (axis_neuron <= 0 || axis_neuron > MAXAX || axis_neuron > last_layer_size) {
    set_error("se_a descriptor: axis_neuron must be in [1, min(%d, M)]", MAXAX);
    return DPB_ERR_INVALID;
  }
  if (nloc <= 0) return DPB_OK;
  const int M = last_layer_size;
  const float inv = tt.nnei > 0 ? 1.f / (float)tt.nnei : 0.f;
  cudaStream_t st = as_stream(stream);
  const int wf = (int)fwd_smem_floats(M, tt.nnei);
  auto run = [&](auto kern, int sw) -> int {
    const size_t smem = sizeof(float) * sw * (size_t)wf;
    DPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "se_a_descriptor_fwd");
    DPB_CUDA(launch_pdl(kern, dim3(ceil_div(nloc, sw)), dim3(sw * 32), smem, st, xyz, descrpt,
                        descrpt_row, em, tt, nloc, M, axis_neuron, inv, wf),
             "se_a_descriptor_fwd");
    return DPB_OK;
  };
  const int ch = tune_value("desc_coef_l1", 3);
  const bool tc = tune_value("desc_tc", 0) != 0;
  auto pick = [&](auto sw_tag) -> int {
    constexpr int SWV = decltype(sw_tag)::value;
    if (tc) return run(k_desc_fwd_tc<SWV, NC>, SWV);
    switch (ch) {
      case 1: return run(k_desc_fwd<SWV, 1, NC>, SWV);
      case 2: return run(k_desc_fwd<SWV, 2, NC>, SWV);
      case 3: return run(k_desc_fwd<SWV, 3, NC>, SWV);
      case 4: return run(k_desc_fwd<SWV, 4, NC>, SWV);
      default: return run(k_desc_fwd<SWV, 0, NC>, SWV);
    }
  };
  switch (tune_value("desc_atoms_per_cta", SW)) {
    case 2: return pick(std::integral_constant<int, 2>{});
    case 8: return pick(std::integral_constant<int, 8>{});
    default: return pick(std::integral_constant<int, 4>{});
  }
}

template <int NC>
static int desc_bwd(float* net_deriv, const float* d_descrpt, const int* descrpt_row,
                    const float* xyz, const float* em, const float* const* tables,
                    const float* table_info, const int* sec, int nsec, int nloc,
                    int last_layer_size, int axis_neuron, dpb_stream_t stream) {
  TypeTables tt;
  int rc = make_tables(tt, tables, table_info, sec, nsec, last_layer_size, NC == 4);
  if (rc) return rc;
  if (axis_neuron <= 0 || axis_neuron > MAXAX || axis_neuron > last_layer_size) {
    set_error("se_a descriptor: axis_neuron must be in [1, min(%d, M)]", MAXAX);
    return DPB_ERR_INVALID;
  }
  if (nloc <= 0) return DPB_OK;
  const int M = last_layer_size;
  const float inv = tt.nnei > 0 ? 1.f / (float)tt.nnei : 0.f;
  cudaStream_t st = as_stream(stream);
  const int wf = (int)bwd_smem_floats(M, tt.nnei, axis_neuron);
  auto run = [&](auto kern, int sw) -> int {
    const size_t smem = sizeof(float) * sw * (size_t)wf;
    DPB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "se_a_descriptor_bwd");
    DPB_CUDA(launch_pdl(kern, dim3(ceil_div(nloc, sw)), dim3(sw * 32), smem, st, net_deriv,
                        d_descrpt, descrpt_row, xyz, em, tt, nloc, M, axis_neuron, inv, wf),
             "se_a_descriptor_bwd");
    return DPB_OK;
  };
  const int ch = tune_value("desc_coef_l1", 3);
  auto pick = [&](auto sw_tag) -> int {
    constexpr int SWV = decltype(sw_tag)::value;
    switch (ch) {
      case 1: return run(k_desc_bwd<SWV, 1, NC>, SWV);
      case 2: return run(k_desc_bwd<SWV, 2, NC>, SWV);
      case 3: return run(k_desc_bwd<SWV, 3, NC>, SWV);
      case 4: return run(k_desc_bwd<SWV, 4, NC>, SWV);
      default: return run(k_desc_bwd<SWV, 0, NC>, SWV);
    }
  };
  switch (tune_value("desc_atoms_per_cta", SW)) {
    case 2: return pick(std::integral_constant<int, 2>{});
    case 8: return pick(std::integral_constant<int, 8>{});
    default: return pick(std::integral_constant<int, 4>{});
  }
}

}  // namespace dpb

extern "C" {

int dpb_se_a_descriptor_fwd_f32(float* xyz, float* descrpt, const int* descrpt_row,
                                const float* em, const float* const* tables,
                                const float* table_info, const int* sec, int nsec,
                                int nloc, int last_layer_size, int axis_neuron,
                                dpb_stream_t stream) {
  return desc_fwd<6>(xyz, descrpt, descrpt_row, em, tables, table_info, sec, nsec, nloc,
                     last_layer_size, axis_neuron, stream);
}

int dpb_se_a_descriptor_fwd_cubic_f32(float* xyz, float* descrpt, const int* descrpt_row,
                                      const float* em, const float* const* tables,
                                      const float* table_info, const int* sec, int nsec,
                                      int nloc, int last_layer_size, int axis_neuron,
                                      dpb_stream_t stream) {
  return desc_fwd<4>(xyz, descrpt, descrpt_row, em, tables, table_info, sec, nsec, nloc,
                     last_layer_size, axis_neuron, stream);
}

int dpb_se_a_descriptor_bwd_f32(float* net_deriv, const float* d_descrpt,
                                const int* descrpt_row, const float* xyz, const float* em,
                                const float* const* tables, const float* table_info,
                                const int* sec, int nsec, int nloc, int last_layer_size,
                                int axis_neuron, dpb_stream_t stream) {
  return desc_bwd<6>(net_deriv, d_descrpt, descrpt_row, xyz, em, tables, table_info, sec, nsec,
                     nloc, last_layer_size, axis_neuron, stream);
}

int dpb_se_a_descriptor_bwd_cubic_f32(float* net_deriv, const float* d_descrpt,
                                      const int* descrpt_row, const float* xyz, const float* em,
                                      const float* const* tables, const float* table_info,
                                      const int* sec, int nsec, int nloc, int last_layer_size,
                                      int axis_neuron, dpb_stream_t stream) {
  return desc_bwd<4>(net_deriv, d_descrpt, descrpt_row, xyz, em, tables, table_info, sec, nsec,
                     nloc, last_layer_size, axis_neuron, stream);
}

int dpb_force_virial_a_env_mixed(double* force, double* virial, const float* net_deriv,
                                 const double* coord, const int* type, const float* std_,
                                 const int* nlist, const int* mapping, int nloc, int nforce,
                                 int nnei, int ntypes, float rcut, float rcut_smth,
                                 dpb_stream_t stream) {
  return force_virial_rc<double, float>(force, virial, net_deriv, coord, type, std_, nlist,
                                        mapping, nloc, nforce, nnei, ntypes, rcut, rcut_smth,
                                        as_stream(stream));
}

int dpb_force_virial_a_env_mixed_acc(double* force, double* virial, const float* net_deriv,
                                     const double* coord, const int* type, const float* std_,
                                     const int* nlist, const int* mapping, int nloc,
                                     int nforce, int nnei, int ntypes, float rcut,
                                     float rcut_smth, dpb_stream_t stream) {
  return force_virial_rc<double, float>(force, virial, net_deriv, coord, type, std_, nlist,
                                        mapping, nloc, nforce, nnei, ntypes, rcut, rcut_smth,
                                        as_stream(stream), false);
}

int dpb_force_virial_a_env_f64(double* force, double* virial, const double* net_deriv,
                               const double* coord, const int* type, const double* std_,
                               const int* nlist, const int* mapping, int nloc, int nforce,
                               int nnei, int ntypes, float rcut, float rcut_smth,
                               dpb_stream_t stream) {
  return force_virial_rc<double, double>(force, virial, net_deriv, coord, type, std_, nlist,
                                         mapping, nloc, nforce, nnei, ntypes, rcut, rcut_smth,
                                         as_stream(stream));
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
  k_force_virial<float><<<grid_stride_blocks(nloc, SW), SW * 32, 0, st>>>(
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
  k_force_virial<double><<<grid_stride_blocks(nloc, SW), SW * 32, 0, st>>>(
      force, virial, atom_virial, net_deriv, env_deriv, rij, nlist, mapping, nloc, nnei);
  DPB_CHECK_LAUNCH("force_virial");
  return DPB_OK;
}

}  // extern "C"
