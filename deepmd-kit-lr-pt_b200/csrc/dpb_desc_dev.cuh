// Device side of the fused se_e2_a descriptor passes (dpb_se_a.cu): the
// per-type compressed tables, the slot staging, and desc_fwd_atom /
// desc_bwd_atom, one center atom's descriptor forward / backward by one
// warp. Used by the descriptor kernels and by the batched-frames step
// kernel (dpb_bt_step.cu).
#pragma once

#include <math.h>

#include "dpb_common.cuh"
#include "dpb_envmath.cuh"

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
// coherent read of data written earlier in the same launch (the fused
// batched step): from L2, never from a possibly stale L1 line
__device__ __forceinline__ float4 ld_cg4(const float4* p) {
  float4 v;
  asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p) : "memory");
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

template <bool COH = false>
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
      if (q < nnei) ev[j] = COH ? ld_cg4(erow + q) : ld_stream4(erow + q, pol);
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
  if ((naxis & 3) == 0 && 32 % (naxis >> 2) == 0 && (M & 3) == 0 &&
      (reinterpret_cast<uintptr_t>(Dr) & 15) == 0) {
    // four columns a..a+3 per lane, kept in registers; naxis / 4 lanes per
    // row, so each pass stores 32 / (naxis / 4) whole rows as one contiguous
    // run of 16-byte stores, and reads x[k, m] once per row and lane
    const int lpr = naxis >> 2, rpi = 32 / lpr;
    const int a = (lane % lpr) * 4, mr = lane / lpr;
    float4 xa[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) xa[k] = *reinterpret_cast<const float4*>(sx + k * M + a);
    for (int m = mr; m < M; m += rpi) {
      const float x0 = sx[m], x1 = sx[M + m], x2 = sx[2 * M + m], x3 = sx[3 * M + m];
      float4 o;
      o.x = x0 * xa[0].x + x1 * xa[1].x + x2 * xa[2].x + x3 * xa[3].x;
      o.y = x0 * xa[0].y + x1 * xa[1].y + x2 * xa[2].y + x3 * xa[3].y;
      o.z = x0 * xa[0].z + x1 * xa[1].z + x2 * xa[2].z + x3 * xa[3].z;
      o.w = x0 * xa[0].w + x1 * xa[1].w + x2 * xa[2].w + x3 * xa[3].w;
      *reinterpret_cast<float4*>(Dr + m * naxis + a) = o;
    }
  } else if (32 % naxis == 0) {  // fixed column a per lane, 32 / naxis rows per pass
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
// COH: the env row was written earlier in the same launch (read coherently)
template <int CH, int NC, bool COH = false>
__device__ __forceinline__ void desc_fwd_atom(int i, int lane, float* wsm, float* __restrict__ xyz_out, float* __restrict__ D,
           const int* __restrict__ drow, const float* __restrict__ em,
           TypeTables tt, int M, int naxis, float inv_nnei) {
  const int nnei = tt.nnei;
  float4* se = reinterpret_cast<float4*>(wsm);
  float4* sl = se + nnei;
  stage_slots<COH>(se, sl, reinterpret_cast<const float4*>(em + (size_t)i * nnei * 4), tt, lane);
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
    auto row = [&](const float4& L) { return tab + (size_t)__float_as_int(L.x) * rs; };
    // two coefficient buffers in turn: the next slot's row is in flight while
    // the current one is evaluated (reusing a row shared by consecutive slots
    // saves L1 traffic but costs the prefetch distance, a net loss measured
    // on 12k-atom water); each buffer keeps the staged table coordinates of
    // its slot, read from shared memory once
    float4 La = Ls[0], Lb;
    Coef4<NC> ca = load_coef4<CH, NC>(row(La), M), cb;
    int q = 0;
    for (; q + 1 <= last; q += 2) {
      Lb = Ls[q + 1];
      cb = load_coef4<CH, NC>(row(Lb), M);
      fwd_slot<NC>(acc01, acc23, ca, E[q], La, rep(q));
      if (q + 2 <= last) {
        La = Ls[q + 2];
        ca = load_coef4<CH, NC>(row(La), M);
      }
      fwd_slot<NC>(acc01, acc23, cb, E[q + 1], Lb, rep(q + 1));
    }
    if (q <= last) fwd_slot<NC>(acc01, acc23, ca, E[q], La, rep(q));
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

template <int CH, int NC>
__device__ __forceinline__ void desc_bwd_atom(int i, int lane, float* wsm, float* __restrict__ net_deriv, const float* __restrict__ dD,
           const int* __restrict__ drow, const float* __restrict__ xyz,
           const float* __restrict__ em, TypeTables tt, int M, int naxis,
           float inv_nnei) {
  const int nnei = tt.nnei;
  float* s_x = wsm;                // [4][M]
  float* s_t = s_x + 4 * M;        // [4][naxis]
  // the atom's dD tile transposed, [naxis][M]: a lane's four channels of one
  // column a are one 16-byte read (M % 4 == 0), conflict-free across lanes;
  // later the slot staging
  float* s_d = s_t + 4 * MAXAX;
  const float* xi = xyz + (size_t)i * 4 * M;
  const unsigned long long pol = l2_policy_first();
  const float* dr = dD + (size_t)drow[i] * M * naxis;
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
      float* dst = s_d + a * M + m;
      dst[0] = v.x;
      dst[M] = v.y;
      dst[2 * M] = v.z;
      dst[3 * M] = v.w;
    }
  } else if (32 % naxis == 0) {
    for (int q = lane; q < 4 * M; q += 32) s_x[q] = ld_stream(xi + q, pol);
    const int per = 32 / naxis, a = lane % naxis;
    for (int m = lane / naxis; m < M; m += per) s_d[a * M + m] = ld_stream(dr + m * naxis + a, pol);
  } else {
    for (int q = lane; q < 4 * M; q += 32) s_x[q] = ld_stream(xi + q, pol);
    for (int q = lane; q < M * naxis; q += 32) {
      const int m = q / naxis, a = q - m * naxis;
      s_d[a * M + m] = ld_stream(dr + q, pol);
    }
  }
  __syncwarp();
  // second term of dxyz for the first naxis channels, spread over the warp:
  // T[k, a] = sum_m' dD[m', a] x[k, m']
  if (naxis == 16 && (M & 3) == 0) {
    // lane = (k, a) and (k + 2, a): one dD column read serves both rows of x,
    // x and the column read four channels at a time
    const int a = lane & 15, k = lane >> 4;
    const float* xa = s_x + k * M;
    const float* xb = s_x + (k + 2) * M;
    const float* da = s_d + a * M;
    float acc0 = 0.f, acc1 = 0.f;
    for (int mp = 0; mp < M; mp += 4) {
      const float4 u = *reinterpret_cast<const float4*>(xa + mp);
      const float4 v = *reinterpret_cast<const float4*>(xb + mp);
      const float4 dv = *reinterpret_cast<const float4*>(da + mp);
      const float d0 = dv.x, d1 = dv.y, d2 = dv.z, d3 = dv.w;
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
      for (int mp = 0; mp < M; ++mp) acc += s_d[a * M + mp] * s_x[k * M + mp];
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
      const float4 g4 = *reinterpret_cast<const float4*>(s_d + a * M + m0);
      const float gch[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {
        const float g = gch[ch];
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
    auto row = [&](const float4& L) { return tab + (size_t)__float_as_int(L.x) * rs; };
    // two coefficient buffers in turn (GRP is even, so slot parity fixes the
    // buffer): the next slot's row is in flight while the current one is
    // used; each buffer keeps its slot's staged table coordinates
    Coef4<NC> ca, cb;
    float4 La = make_float4(0.f, 0.f, 0.f, 0.f), Lb = La;
    if (act) {
      La = Ls[0];
      ca = load_coef4<CH, NC>(row(La), M);
    }
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
            if (qq + 1 <= last) {
              Lb = Ls[qq + 1];
              cb = load_coef4<CH, NC>(row(Lb), M);
            }
            bwd_slot<NC>(P[q], ca, E[qq], La, rep(qq), dyr01, dyr23);
          } else {
            if (qq + 1 <= last) {
              La = Ls[qq + 1];
              ca = load_coef4<CH, NC>(row(La), M);
            }
            bwd_slot<NC>(P[q], cb, E[qq], Lb, rep(qq), dyr01, dyr23);
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
