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

// first slot q in [0, n) of a type block whose em_x equals the block's last
// and whose em[1..3] are zero; n when there is none (rows staged in shared
// memory)
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

// Coefficients of 4 consecutive channels m0..m0+3 of one table row in the
// pipeline layout [row][6][M] (coefficient-major, dpb_se_a_pack_table_f32):
// q[k] holds a_k of the 4 channels, so each of the 6 loads of a warp reads one
// contiguous 4M-byte segment of the row (M % 4 == 0 keeps them 16-byte
// aligned).
// NC = 6: the reference's quintic table; NC = 4: its cubic re-interpolation
// on the fine grid (dpb_se_a_descriptor_*_cubic_f32).
template <int NC>
struct Coef4 {
  float2 lo[NC];  // a_k of channels (0, 1)
  float2 hi[NC];  // a_k of channels (2, 3)
};

// L2 cache policies: evict_first for data read once per step (env rows, x,
// dE/dD), evict_last for the table coefficients reused by every atom
__device__ __forceinline__ unsigned long long l2_policy_first() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_policy_last() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// streaming read: not allocated in L1 (keeps L1 for the table rows), first
// out of L2
__device__ __forceinline__ float4 ld_stream4(const float4* p, unsigned long long pol) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p, unsigned long long pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

// 16-byte read-only load of table coefficients with the L1 policy CH:
// 0 default, 1 L1::no_allocate, 2 L1::evict_first, 3 L1::evict_last,
// 4 L1::evict_last with the L2 evict_last policy
template <int CH>
__device__ __forceinline__ float4 ld_coef(const float* p) {
  float4 v;
  if (CH == 4)
    asm("ld.global.nc.L1::evict_last.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(l2_policy_last()));
  else if (CH == 1)
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  else if (CH == 2)
    asm("ld.global.nc.L1::evict_first.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  else if (CH == 3)
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  else
    v = __ldg(reinterpret_cast<const float4*>(p));
  return v;
}

template <int CH, int NC>
__device__ __forceinline__ Coef4<NC> load_coef4(const float* row, int M) {
  Coef4<NC> c;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const float4 v = ld_coef<CH>(row + k * M);
    c.lo[k] = make_float2(v.x, v.y);
    c.hi[k] = make_float2(v.z, v.w);
  }
  return c;
}

// Two channels per instruction with the sm_100 packed FP32 operations
// (__ffma2_rn and friends: per component exactly __fmaf_rn / __fmul_rn /
// __fadd_rn).
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// value only: a0 + (a1 + (a2 + (a3 + (a4 + a5 x) x) x) x) x  (tabulate.cc:123-130;
// degree NC - 1)
template <int NC>
__device__ __forceinline__ float2 hval2(const float2 (&c)[NC], float2 x) {
  float2 p = __ffma2_rn(c[NC - 1], x, c[NC - 2]);
#pragma unroll
  for (int k = NC - 3; k >= 0; --k) p = __ffma2_rn(p, x, c[k]);
  return p;
}

// value and derivative by the joint Horner recurrence (2 NC - 3 FMA)
template <int NC>
__device__ __forceinline__ void hvalgrad2(const float2 (&c)[NC], float2 x, float2& v, float2& g) {
  float2 p = c[NC - 1], d = c[NC - 1];
#pragma unroll
  for (int k = NC - 2; k >= 1; --k) {
    p = __ffma2_rn(p, x, c[k]);
    d = __ffma2_rn(d, x, p);
  }
  v = __ffma2_rn(p, x, c[0]);
  g = d;
}

// Per-warp staging of one center atom's neighbor slots in shared memory:
// se[s] = em row s, sl[s] = (table row as int bits, offset in the row,
// extrapolation distance, 0). The table coordinates are computed once per
// slot, lane-parallel, so the channel loops only wait on coefficient loads.
constexpr int STAGE_J = 4;  // env rows per lane requested together

__device__ __forceinline__ void stage_slots(float4* se, float4* sl, const float4* erow,
                                            const TypeTables& tt, int lane) {
  const unsigned long long pol = l2_policy_first();
  const int nnei = tt.nnei;
  // STAGE_J rows of this lane requested before the first is used
  for (int q0 = lane; q0 < nnei; q0 += 32 * STAGE_J) {
    float4 ev[STAGE_J];
#pragma unroll
    for (int j = 0; j < STAGE_J; ++j) {
      const int q = q0 + 32 * j;
      if (q < nnei) ev[j] = ld_stream4(erow + q, pol);
    }
#pragma unroll
    for (int j = 0; j < STAGE_J; ++j) {
      const int q = q0 + 32 * j;
      if (q < nnei) {
        int t = 0;
        while (t + 1 < tt.ntypes && q >= tt.sec[t + 1]) ++t;
        int idx;
        float xx, delta;
        flocate(tt.info[t], ev[j].x, idx, xx, delta);
        se[q] = ev[j];
        sl[q] = make_float4(__int_as_float(idx), xx, delta, 0.f);
      }
    }
  }
}

// shared memory of the descriptor kernels: per warp, 2 * nnei float4 of slot
// staging, or (backward) the dD / x tiles of the prologue when larger
static size_t fwd_smem_floats(int M, int nnei) {
  const size_t slots = (size_t)nnei * 8, xs = (size_t)4 * M;
  return slots > xs ? slots : xs;
}
static size_t bwd_smem_floats(int M, int nnei, int naxis) {
  const size_t slots = (size_t)nnei * 8, dd = (size_t)M * (naxis + 1);
  return (size_t)4 * M + 4 * MAXAX + (slots > dd ? slots : dd);
}

// one neighbor slot of the forward: G row of 4 channels (fold multiplier at
// the fold slot) times the env row, accumulated into acc01[k] / acc23[k]
// (channel pairs (0, 1) and (2, 3) of env column k)
template <int NC>
__device__ __forceinline__ void fwd_slot(float2 (&acc01)[4], float2 (&acc23)[4], const Coef4<NC>& c,
                                         const float4 e, const float4 L, float rep) {
  const float2 x = f2(L.y);
  float2 v01, v23;
  if (L.z == 0.f) {
    v01 = hval2<NC>(c.lo, x);
    v23 = hval2<NC>(c.hi, x);
  } else {  // linear extrapolation outside the table (tabulate.cc:133-144)
    float2 g01, g23;
    hvalgrad2<NC>(c.lo, x, v01, g01);
    hvalgrad2<NC>(c.hi, x, v23, g23);
    v01 = __ffma2_rn(g01, f2(L.z), v01);
    v23 = __ffma2_rn(g23, f2(L.z), v23);
  }
  if (rep != 1.f) {
    v01 = __fmul2_rn(v01, f2(rep));
    v23 = __fmul2_rn(v23, f2(rep));
  }
  const float ek[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    acc01[k] = __ffma2_rn(v01, f2(ek[k]), acc01[k]);
    acc23[k] = __ffma2_rn(v23, f2(ek[k]), acc23[k]);
  }
}

// D[m, a] = sum_k x[k, m] x[k, a] of one atom from x [4][M] in shared memory
__device__ __forceinline__ void write_descriptor(float* __restrict__ Dr, const float* sx, int M,
                                                 int naxis, int lane) {
  if (32 % naxis == 0) {  // fixed column a per lane, 32 / naxis rows per pass
    const int per = 32 / naxis, a = lane % naxis;
    const float x0 = sx[a], x1 = sx[M + a], x2 = sx[2 * M + a], x3 = sx[3 * M + a];
    for (int m = lane / naxis; m < M; m += per)
      Dr[m * naxis + a] = sx[m] * x0 + sx[M + m] * x1 + sx[2 * M + m] * x2 + sx[3 * M + m] * x3;
  } else {
    for (int q = lane; q < M * naxis; q += 32) {
      const int m = q / naxis, a = q - m * naxis;
      Dr[q] = sx[m] * sx[a] + sx[M + m] * sx[M + a] + sx[2 * M + m] * sx[2 * M + a] +
              sx[3 * M + m] * sx[3 * M + a];
    }
  }
}

// SWT warps (one center atom each) per CTA, about 20 warps per SM
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
  const int nnei = tt.nnei;
  float* wsm = reinterpret_cast<float*>(dsm4) + (size_t)w * warp_floats;
  float4* se = reinterpret_cast<float4*>(wsm);
  float4* sl = se + nnei;
  stage_slots(se, sl, reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4), tt, lane);
  __syncwarp();
  const int m0 = 4 * lane;
  const bool act = m0 < M;
  float2 acc01[4], acc23[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) acc01[k] = acc23[k] = make_float2(0.f, 0.f);
  for (int t = 0; t < tt.ntypes; ++t) {
    const int s0 = tt.sec[t], nt = tt.sec[t + 1] - s0;
    if (nt <= 0) continue;
    const int brk = block_fold(se + s0, nt, lane);
    const int last = brk < nt ? brk : nt - 1;
    if (!act) continue;
    const float* tab = tt.table[t] + m0;
    const size_t rs = (size_t)M * NC;
    const float4* E = se + s0;
    const float4* Ls = sl + s0;
    auto rep = [&](int q) { return q == brk ? (float)(nt - q) : 1.f; };
    auto row = [&](int q) { return tab + (size_t)__float_as_int(Ls[q].x) * rs; };
    // two coefficient buffers in turn: the next slot's row is in flight while
    // the current one is evaluated (reusing a row shared by consecutive slots
    // saves L1 traffic but costs the prefetch distance, a net loss measured
    // on 12k-atom water)
    Coef4<NC> ca = load_coef4<CH, NC>(row(0), M), cb;
    int q = 0;
    for (; q + 1 <= last; q += 2) {
      cb = load_coef4<CH, NC>(row(q + 1), M);
      fwd_slot<NC>(acc01, acc23, ca, E[q], Ls[q], rep(q));
      if (q + 2 <= last) ca = load_coef4<CH, NC>(row(q + 2), M);
      fwd_slot<NC>(acc01, acc23, cb, E[q + 1], Ls[q + 1], rep(q + 1));
    }
    if (q <= last) fwd_slot<NC>(acc01, acc23, ca, E[q], Ls[q], rep(q));
  }
  __syncwarp();  // the slot staging is reused for x below
  float* sx = wsm;  // [4][M]
  float* xo = xyz_out + (size_t)i * 4 * M;
  if (act) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float4 o = make_float4(acc01[k].x * inv_nnei, acc01[k].y * inv_nnei,
                             acc23[k].x * inv_nnei, acc23[k].y * inv_nnei);
      *reinterpret_cast<float4*>(xo + k * M + m0) = o;
      *reinterpret_cast<float4*>(sx + k * M + m0) = o;
    }
  }
  __syncwarp();
  write_descriptor(D + (size_t)drow[i] * M * naxis, sx, M, naxis, lane);
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

constexpr int GRP = 4;  // neighbors reduced together in the backward (even)

// one neighbor slot of the backward over this lane's 4 channels (times the
// fold multiplier): P[0] = sum_c G'_c (e . dyr_c) + G_c dyr_c[0] (the two
// terms of the slot's first output component), P[d] = sum_c G_c dyr_c[d] for
// d = 1..3; dyr01[d] / dyr23[d] hold dyr of channel pairs (0, 1) / (2, 3)
template <int NC>
__device__ __forceinline__ void bwd_slot(float (&P)[4], const Coef4<NC>& c, const float4 e,
                                         const float4 L, float rep, const float2 (&dyr01)[4],
                                         const float2 (&dyr23)[4]) {
  const float2 x = f2(L.y), dl = f2(L.z);
  float2 v01, g01, v23, g23;
  hvalgrad2<NC>(c.lo, x, v01, g01);
  hvalgrad2<NC>(c.hi, x, v23, g23);
  v01 = __ffma2_rn(g01, dl, v01);
  v23 = __ffma2_rn(g23, dl, v23);
  float2 d01 = __fmul2_rn(dyr01[0], f2(e.x));
  float2 d23 = __fmul2_rn(dyr23[0], f2(e.x));
  d01 = __ffma2_rn(dyr01[1], f2(e.y), d01);
  d23 = __ffma2_rn(dyr23[1], f2(e.y), d23);
  d01 = __ffma2_rn(dyr01[2], f2(e.z), d01);
  d23 = __ffma2_rn(dyr23[2], f2(e.z), d23);
  d01 = __ffma2_rn(dyr01[3], f2(e.w), d01);
  d23 = __ffma2_rn(dyr23[3], f2(e.w), d23);
  float2 p0 = __ffma2_rn(g23, d23, __fmul2_rn(g01, d01));
  p0 = __ffma2_rn(v01, dyr01[0], p0);
  p0 = __ffma2_rn(v23, dyr23[0], p0);
  P[0] = p0.x + p0.y;
#pragma unroll
  for (int d = 1; d < 4; ++d) {
    const float2 pd = __ffma2_rn(v23, dyr23[d], __fmul2_rn(v01, dyr01[d]));
    P[d] = pd.x + pd.y;
  }
  if (rep != 1.f) {
#pragma unroll
    for (int k = 0; k < 4; ++k) P[k] *= rep;
  }
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
  const int nnei = tt.nnei;
  float* wsm = reinterpret_cast<float*>(dsm4) + (size_t)w * warp_floats;
  float* s_x = wsm;                // [4][M]
  float* s_t = s_x + 4 * M;        // [4][naxis]
  float* s_d = s_t + 4 * MAXAX;    // [M][naxis + 1], later the slot staging
  const float* xi = xyz + (size_t)i * 4 * M;
  const unsigned long long pol = l2_policy_first();
  const float* dr = dD + (size_t)drow[i] * M * naxis;
  const int ldd = naxis + 1;  // padded row: conflict-free column reads
  if ((M & 3) == 0 && (naxis & 3) == 0 &&
      ((reinterpret_cast<uintptr_t>(xi) | reinterpret_cast<uintptr_t>(dr)) & 15) == 0) {
    // 16-byte loads (more loads in flight per lane) where the rows allow
    const float4* x4 = reinterpret_cast<const float4*>(xi);
    for (int q = lane; q < M; q += 32) reinterpret_cast<float4*>(s_x)[q] = ld_stream4(x4 + q, pol);
    const float4* d4 = reinterpret_cast<const float4*>(dr);
    const int per_row = naxis >> 2;
    for (int q = lane; q < (M * naxis) >> 2; q += 32) {
      const float4 v = ld_stream4(d4 + q, pol);
      const int m = q / per_row, a = (q - m * per_row) << 2;
      float* dst = s_d + m * ldd + a;
      dst[0] = v.x;
      dst[1] = v.y;
      dst[2] = v.z;
      dst[3] = v.w;
    }
  } else if (32 % naxis == 0) {
    for (int q = lane; q < 4 * M; q += 32) s_x[q] = ld_stream(xi + q, pol);
    const int per = 32 / naxis, a = lane % naxis;
    for (int m = lane / naxis; m < M; m += per) s_d[m * ldd + a] = ld_stream(dr + m * naxis + a, pol);
  } else {
    for (int q = lane; q < 4 * M; q += 32) s_x[q] = ld_stream(xi + q, pol);
    for (int q = lane; q < M * naxis; q += 32) {
      const int m = q / naxis, a = q - m * naxis;
      s_d[m * ldd + a] = ld_stream(dr + q, pol);
    }
  }
  __syncwarp();
  // second term of dxyz for the first naxis channels, spread over the warp:
  // T[k, a] = sum_m' dD[m', a] x[k, m']
  if (naxis == 16 && (M & 3) == 0) {
    // lane = (k, a) and (k + 2, a): one dD column read serves both rows of x,
    // x read four channels at a time
    const int a = lane & 15, k = lane >> 4;
    const float* xa = s_x + k * M;
    const float* xb = s_x + (k + 2) * M;
    float acc0 = 0.f, acc1 = 0.f;
    for (int mp = 0; mp < M; mp += 4) {
      const float4 u = *reinterpret_cast<const float4*>(xa + mp);
      const float4 v = *reinterpret_cast<const float4*>(xb + mp);
      const float d0 = s_d[mp * ldd + a], d1 = s_d[(mp + 1) * ldd + a];
      const float d2 = s_d[(mp + 2) * ldd + a], d3 = s_d[(mp + 3) * ldd + a];
      acc0 += d0 * u.x;
      acc1 += d0 * v.x;
      acc0 += d1 * u.y;
      acc1 += d1 * v.y;
      acc0 += d2 * u.z;
      acc1 += d2 * v.z;
      acc0 += d3 * u.w;
      acc1 += d3 * v.w;
    }
    s_t[lane] = acc0;
    s_t[lane + 32] = acc1;
  } else {
    for (int o = lane; o < 4 * naxis; o += 32) {
      const int k = o / naxis, a = o - k * naxis;
      float acc = 0.f;
      for (int mp = 0; mp < M; ++mp) acc += s_d[mp * ldd + a] * s_x[k * M + mp];
      s_t[o] = acc;
    }
  }
  __syncwarp();
  // dxyz[k, m] = sum_a dD[m, a] x[k, a] + [m < naxis] T[k, m]
  const int m0 = 4 * lane;
  const bool act = m0 < M;
  float dyr[4][4];
#pragma unroll
  for (int ch = 0; ch < 4; ++ch)
#pragma unroll
    for (int k = 0; k < 4; ++k) dyr[ch][k] = 0.f;
  if (act) {
    for (int a = 0; a < naxis; ++a) {
      const float x0 = s_x[a], x1 = s_x[M + a], x2 = s_x[2 * M + a], x3 = s_x[3 * M + a];
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const float g = s_d[(m0 + ch) * ldd + a];
        dyr[ch][0] += g * x0;
        dyr[ch][1] += g * x1;
        dyr[ch][2] += g * x2;
        dyr[ch][3] += g * x3;
      }
    }
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const int m = m0 + ch;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (m < naxis) dyr[ch][k] += s_t[k * naxis + m];
        dyr[ch][k] *= inv_nnei;
      }
    }
  }
  float2 dyr01[4], dyr23[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    dyr01[k] = make_float2(dyr[0][k], dyr[1][k]);
    dyr23[k] = make_float2(dyr[2][k], dyr[3][k]);
  }
  __syncwarp();  // dD tile dead: stage the slots in its place
  float4* se = reinterpret_cast<float4*>(s_d);
  float4* sl = se + nnei;
  stage_slots(se, sl, reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4), tt, lane);
  __syncwarp();
  float4* nrow = reinterpret_cast<float4*>(net_deriv + (size_t)i * nnei * 4);
  const int b4 = (lane >> 4) & 1, b3 = (lane >> 3) & 1;
  for (int t = 0; t < tt.ntypes; ++t) {
    const int s0 = tt.sec[t], nt = tt.sec[t + 1] - s0;
    if (nt <= 0) continue;
    const int brk = block_fold(se + s0, nt, lane);
    const int last = brk < nt ? brk : nt - 1;
    const float* tab = tt.table[t] + m0;
    const size_t rs = (size_t)M * NC;
    const float4* E = se + s0;
    const float4* Ls = sl + s0;
    auto rep = [&](int q) { return q == brk ? (float)(nt - q) : 1.f; };
    auto row = [&](int q) { return tab + (size_t)__float_as_int(Ls[q].x) * rs; };
    // two coefficient buffers in turn (GRP is even, so slot parity fixes the
    // buffer): the next slot's row is in flight while the current one is used
    Coef4<NC> ca, cb;
    if (act) ca = load_coef4<CH, NC>(row(0), M);
    for (int g0 = 0; g0 < nt; g0 += GRP) {
      if (g0 > last) {  // beyond the fold point: zero rows
        for (int qq = g0 + lane; qq < nt && qq < g0 + GRP; qq += 32)
          nrow[s0 + qq] = make_float4(0.f, 0.f, 0.f, 0.f);
        continue;
      }
      float P[GRP][4];
#pragma unroll
      for (int q = 0; q < GRP; ++q) {
#pragma unroll
        for (int k = 0; k < 4; ++k) P[q][k] = 0.f;
        const int qq = g0 + q;
        if (qq <= last && act) {  // warp-uniform apart from the idle lanes
          if ((q & 1) == 0) {
            if (qq + 1 <= last) cb = load_coef4<CH, NC>(row(qq + 1), M);
            bwd_slot<NC>(P[q], ca, E[qq], Ls[qq], rep(qq), dyr01, dyr23);
          } else {
            if (qq + 1 <= last) ca = load_coef4<CH, NC>(row(qq + 1), M);
            bwd_slot<NC>(P[q], cb, E[qq], Ls[qq], rep(qq), dyr01, dyr23);
          }
        }
      }
      // reduce-scatter of the 4 x 4 partials over the warp: after the xor-16
      // and -8 steps lane L holds neighbor q = 2*b4 + b3 summed over 8 lanes;
      // xor-4, -2 and -1 finish the sum in every lane of the group of 8.
      float R1[2][4];
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float mine = b4 ? P[2 + q][k] : P[q][k];
          const float other = b4 ? P[q][k] : P[2 + q][k];
          R1[q][k] = mine + __shfl_xor_sync(0xffffffffu, other, 16);
        }
      float R2[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float mine = b3 ? R1[1][k] : R1[0][k];
        const float other = b3 ? R1[0][k] : R1[1][k];
        R2[k] = mine + __shfl_xor_sync(0xffffffffu, other, 8);
        R2[k] += __shfl_xor_sync(0xffffffffu, R2[k], 4);
        R2[k] += __shfl_xor_sync(0xffffffffu, R2[k], 2);
        R2[k] += __shfl_xor_sync(0xffffffffu, R2[k], 1);
      }
      const int qq = g0 + 2 * b4 + b3;
      if ((lane & 7) == 0 && qq < nt)  // zero beyond the fold point
        nrow[s0 + qq] = make_float4(R2[0], R2[1], R2[2], R2[3]);
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
    OT v[4], gd[12];
    env_row<OT>(r, rcut_smth, rcut, v, gd);
    OT p[3] = {(OT)0., (OT)0., (OT)0.};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += nv[a] * (gd[a * 3 + d] / sv[a]);
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

// cubic: the tables are the uniform-stride cubic re-interpolation
// (info = [lower, max, max, stride, stride, K] with K intervals and a
// guard row K holding the value and slope at max)
static int make_tables(TypeTables& tt, const float* const* tables, const float* info,
                       const int* sec, int nsec, int M, bool cubic = false) {
  if (nsec < 2 || nsec - 1 > PMAXT || tables == nullptr || info == nullptr || sec == nullptr) {
    set_error("se_a pipeline: need 1..%d neighbor types with tables, info and sec", PMAXT);
    return DPB_ERR_INVALID;
  }
  if (M <= 0 || M > MAXM || M % 4 != 0) {
    set_error("se_a pipeline: last_layer_size must be a multiple of 4 in [4, %d], got %d",
              MAXM, M);
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
    if (cubic) {
      if (!(f[5] >= 1.f) || f[1] != f[2] || f[3] != f[4] || !(f[3] > 0.f)) {
        set_error("se_a pipeline: invalid cubic table info for neighbor type %d", t);
        return DPB_ERR_INVALID;
      }
      x.first = (int)f[5];
      x.high_idx = x.first;  // the guard row at max
    } else {
      x.first = (int)((x.upper - x.lower) / x.s0);
      x.high_idx = x.first + (int)((nextafterf(x.max, x.lower) - x.upper) / x.s1);
    }
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
