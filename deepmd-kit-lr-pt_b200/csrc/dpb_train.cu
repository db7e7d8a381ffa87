// Training step of the uncompressed se_e2_a model with a force and virial
// loss: energy, its first derivative (force, virial) and the second
// derivative the loss gradient needs, hand-written on the device.
//
// Model (deepmd/pt/model/descriptor/se_a.py:742-859, type_one_side):
//   s = R[n][0], G_t(s): 1 -> n1 -> n2 -> n3 tanh embedding of neighbor type t
//   with the residual y + [x, x] when a layer doubles its width (y + x when
//   it keeps it; deepmd/dpmodel/utils/network.py:282-330),
//   xyz[a][m] = sum_n R[n][a] G[n][m] / nnei, D[m][k] = sum_a xyz[a][m] xyz[a][k].
//
// Derivatives. The force F = -dE/dr depends on the weights only through
// g = dE/dem (the env derivative does not), so for a loss L(E, F, V)
//   dL/dtheta = sum_f Ebar_f dE_f/dtheta + d/dtheta <u, g>,
// with u[i][n][a] = dL/dg[i][n][a] = sum_d ed[a][d] (Fbar_j - Fbar_i + Vbar r)_d
// (ed = d em / d r_i, the env derivative, recomputed from the coordinates).
// <u, g> is the directional derivative of E along u in env-matrix space, so
// the second term is a tangent (forward-mode) pass of the network along u
// followed by one reverse pass over the primal and tangent values together
// (reverse over forward). Kernels, one warp per center atom, the embedding
// recomputed per row group instead of stored:
//   k_tr_fwd : G, xyz, D                          (forward)
//   k_tr_bwd : g = dE/dem from Dbar = dE/dD       (force backward)
//   k_tr_tan : xyz', D' along u                   (tangent)
//   k_tr_rev : embedding weight gradients of J = sum Ebar E + <u, g>
// Padded slots of one neighbor type share one env row when avg/std agree
// across the section, and are then evaluated once with a multiplicity.
// The fitting net (per center type, dense GEMMs) runs through the GEMM
// library with the elementwise kernels k_fit_*; Adam is k_adam.
#include <algorithm>
#include <cmath>

#include "dpb_batch.cuh"
#include "dpb_envmath.cuh"

namespace dpb {

constexpr int TR_MAXT = BT_MAXT;
constexpr int TR_C1 = 1, TR_C2 = 2, TR_C3 = 4;  // channels per lane: n1 <= 32, n2 <= 64, n3 <= 128
constexpr int TR_MAXAX = 32;
enum { TR_RES_NONE = 0, TR_RES_IDENT = 1, TR_RES_DUP = 2 };

// rows per group and where the weights live, per precision
template <typename T>
struct TrTraits;
template <>
struct TrTraits<float> {
  static constexpr int R = 8;
  static constexpr bool WSMEM = true;
};
template <>
struct TrTraits<double> {
  static constexpr int R = 4;
  static constexpr bool WSMEM = false;
};

__host__ __device__ constexpr int tr_res_kind(int n_out, int n_in) {
  return n_out == n_in ? TR_RES_IDENT : (n_out == 2 * n_in ? TR_RES_DUP : TR_RES_NONE);
}

__device__ __forceinline__ float tr_tanh(float x) { return tanhf(x); }
__device__ __forceinline__ double tr_tanh(double x) { return tanh(x); }

template <typename T>
struct TrNet {
  const T* W[TR_MAXT][3];  // [n_in, n_out] row-major
  const T* b[TR_MAXT][3];
  int n1, n2, n3, res2, res3;
};

template <typename T>
struct TrGrad {
  T* W[TR_MAXT][3];
  T* b[TR_MAXT][3];
};

// shared-memory layout (host computed); offsets in T elements
struct TrLayout {
  int nw;            // warps per block
  int ints_warp;     // ints per warp (entry list)
  int pw;            // T elements per type block of weights (padded strides)
  int s2, s3, sax;   // padded strides of W2, W3 and of a staged descriptor row
  int w_off, acc_off, warp_off, warp_sz;
  int o_rr, o_rd, o_mu, o_s, o_sd, o_A1, o_At1, o_A2, o_At2, o_Zt2, o_big;
  int wsmem;         // weights staged in shared memory
  int sacc;          // reverse pass: one gradient copy per block (shared-memory
                     // atomics) instead of one per warp
};

struct TrGeom {
  BtFrames fr;
  const double* cw;  // wrapped coordinates [N, 3]
  const int* type;   // [N]
  const int* nlist;  // [N, nnei] packed (atom * 27 + image) or -1
  const int* drow;   // [N] row of the atom in the type-grouped descriptor
  int ntypes, nnei, nrows, ax;
  int sec[TR_MAXT + 1];
  unsigned long long fold;  // bit ti * 8 + t: padded slots of section t share one row
  float rcut, rcut_smth;
};

template <typename T>
struct WV {
  const T *W1, *b1, *W2, *b2, *W3, *b3;
  int s2, s3;
};

// layer pointers of net t: staged in shared memory (odd strides sw2 = n2 | 1,
// sw3 = n3 | 1, type blocks of pw elements) or read from global memory
template <typename T, bool WS>
__device__ __forceinline__ WV<T> tr_wview(const TrNet<T>& net, const T* sw, int t, int pw,
                                          int n1, int n2, int sw2, int sw3) {
  WV<T> v;
  if (WS) {
    const T* base = sw + (size_t)t * pw;
    v.W1 = base;
    v.b1 = v.W1 + n1;
    v.W2 = v.b1 + n1;
    v.b2 = v.W2 + n1 * sw2;
    v.W3 = v.b2 + n2;
    v.b3 = v.W3 + n2 * sw3;
  } else {
    v.W1 = net.W[t][0];
    v.b1 = net.b[t][0];
    v.W2 = net.W[t][1];
    v.b2 = net.b[t][1];
    v.W3 = net.W[t][2];
    v.b3 = net.b[t][2];
  }
  v.s2 = sw2;
  v.s3 = sw3;
  return v;
}

// weights of every type into shared memory with odd row strides, so that
// both a row (lanes over outputs) and a column (lanes over inputs) of W2 / W3
// are read without bank conflicts
template <typename T>
__device__ void tr_stage_weights(T* sw, const TrNet<T>& net, const TrLayout& lay, int ntypes) {
  for (int t = 0; t < ntypes; ++t) {
    T* base = sw + (size_t)t * lay.pw;
    T* W1 = base;
    T* b1 = W1 + net.n1;
    T* W2 = b1 + net.n1;
    T* b2 = W2 + net.n1 * lay.s2;
    T* W3 = b2 + net.n2;
    T* b3 = W3 + net.n2 * lay.s3;
    for (int k = threadIdx.x; k < net.n1; k += blockDim.x) {
      W1[k] = net.W[t][0][k];
      b1[k] = net.b[t][0][k];
    }
    for (int e = threadIdx.x; e < net.n1 * net.n2; e += blockDim.x)
      W2[(e / net.n2) * lay.s2 + e % net.n2] = net.W[t][1][e];
    for (int k = threadIdx.x; k < net.n2; k += blockDim.x) b2[k] = net.b[t][1][k];
    for (int e = threadIdx.x; e < net.n2 * net.n3; e += blockDim.x)
      W3[(e / net.n3) * lay.s3 + e % net.n3] = net.W[t][2][e];
    for (int k = threadIdx.x; k < net.n3; k += blockDim.x) b3[k] = net.b[t][2][k];
  }
}

// entry list of one center: (slot | multiplicity << 16) per row to evaluate,
// grouped by neighbor type over the sections [t0, t1); secn[t] = first entry
// of section t, secn[t1] = the end
__device__ __forceinline__ void tr_entries(int* ent, int* secn, const int* nl, const TrGeom& g,
                                           int ti, bool with_pad, int lane, int t0, int t1) {
  int total = 0;
  for (int t = t0; t < t1; ++t) {
    secn[t] = total;
    const int s0 = g.sec[t], s1 = g.sec[t + 1];
    const bool fold = with_pad && ((g.fold >> (ti * 8 + t)) & 1ull);
    int npad = 0, first_pad = -1;
    for (int base = s0; base < s1; base += 32) {
      const int n = base + lane;
      const bool in = n < s1;
      const bool real = in && nl[n] >= 0;
      const bool pad = in && !real;
      const bool take = real || (pad && with_pad && !fold);
      const unsigned bt = __ballot_sync(0xffffffffu, take);
      if (take) ent[total + __popc(bt & bt_lanemask_lt())] = n | (1 << 16);
      total += __popc(bt);
      const unsigned bp = __ballot_sync(0xffffffffu, pad);
      if (bp != 0u && first_pad < 0) first_pad = base + __ffs(bp) - 1;
      npad += __popc(bp);
    }
    if (fold && npad > 0) {
      if (lane == 0) ent[total] = first_pad | (npad << 16);
      total += 1;
    }
  }
  if (lane == 0) secn[t1] = total;
  __syncwarp();
}

// Staged per-row vectors: the R rows of channel c are contiguous, and with
// two 16-byte chunks per channel the chunks are swapped when bit 2 of c is
// set (with four, chunk h goes to h ^ ((c >> 1) & 3)). A lane-owned channel
// then moves as whole 16-byte chunks without bank conflicts (the 8 lanes of
// a quarter-warp hit 8 different bank groups) and the next layer reads one
// channel as one to four broadcast 16-byte loads.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <typename T, int R>
__device__ __forceinline__ int stg_chunk(int c, int h) {
  constexpr int Q = R / Vec16<T>::n;
  static_assert(Q == 1 || Q == 2 || Q == 4, "one, two or four 16-byte chunks per channel");
  return Q == 4 ? (h ^ ((c >> 1) & 3)) : Q == 2 ? (h ^ ((c >> 2) & 1)) : h;
}

template <typename T, int R>
__device__ __forceinline__ void stg_load(T (&a)[R], const T* base, int c) {
  using V = typename Vec16<T>::type;
  constexpr int E = Vec16<T>::n, Q = R / E;
#pragma unroll
  for (int h = 0; h < Q; ++h) {
    const V v = *reinterpret_cast<const V*>(base + c * R + stg_chunk<T, R>(c, h) * E);
    const T* p = reinterpret_cast<const T*>(&v);
#pragma unroll
    for (int k = 0; k < E; ++k) a[h * E + k] = p[k];
  }
}

template <typename T, int R>
__device__ __forceinline__ void stg_store(T* base, int c, const T (&a)[R]) {
  using V = typename Vec16<T>::type;
  constexpr int E = Vec16<T>::n, Q = R / E;
#pragma unroll
  for (int h = 0; h < Q; ++h) {
    V v;
    T* p = reinterpret_cast<T*>(&v);
#pragma unroll
    for (int k = 0; k < E; ++k) p[k] = a[h * E + k];
    *reinterpret_cast<V*>(base + c * R + stg_chunk<T, R>(c, h) * E) = v;
  }
}

template <typename T, int R>
__device__ __forceinline__ void tr_load_col(T (&a)[R], const T* base, int c) {
  stg_load<T, R>(a, base, c);
}

// acc[j][r] = sum_i in[i][r] W[i * sw + c_j], c_j = lane + 32 j (< n_out)
template <typename T, int R, int CP>
__device__ __forceinline__ void tr_gemv(T (&acc)[CP][R], const T* in, int n_in, const T* W,
                                        int sw, int n_out, int lane) {
#pragma unroll
  for (int j = 0; j < CP; ++j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[j][r] = (T)0;
#pragma unroll 5
  for (int i = 0; i < n_in; ++i) {
    T a[R];
    tr_load_col<T, R>(a, in, i);
#pragma unroll
    for (int j = 0; j < CP; ++j) {
      const int c = lane + 32 * j;
      const T w = c < n_out ? W[i * sw + c] : (T)0;
#pragma unroll
      for (int r = 0; r < R; ++r) acc[j][r] = fma(a[r], w, acc[j][r]);
    }
  }
}

// the same for two inputs sharing the weight loads (primal and tangent)
template <typename T, int R, int CP>
__device__ __forceinline__ void tr_gemv2(T (&acc)[CP][R], T (&acd)[CP][R], const T* in,
                                         const T* ind, int n_in, const T* W, int sw, int n_out,
                                         int lane) {
#pragma unroll
  for (int j = 0; j < CP; ++j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[j][r] = acd[j][r] = (T)0;
#pragma unroll 5
  for (int i = 0; i < n_in; ++i) {
    T a[R], ad[R];
    tr_load_col<T, R>(a, in, i);
    tr_load_col<T, R>(ad, ind, i);
#pragma unroll
    for (int j = 0; j < CP; ++j) {
      const int c = lane + 32 * j;
      const T w = c < n_out ? W[i * sw + c] : (T)0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        acc[j][r] = fma(a[r], w, acc[j][r]);
        acd[j][r] = fma(ad[r], w, acd[j][r]);
      }
    }
  }
}

// transposed product, lanes over the inputs i_j = lane + 32 j (< n_in):
// acc[j][r] = sum_c zb[c][r] W[i_j * sw + c]
template <typename T, int R, int CP>
__device__ __forceinline__ void tr_gemvT(T (&acc)[CP][R], const T* zb, int n_out, const T* W,
                                         int sw, int n_in, int lane) {
#pragma unroll
  for (int j = 0; j < CP; ++j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[j][r] = (T)0;
#pragma unroll 5
  for (int c = 0; c < n_out; ++c) {
    T z[R];
    tr_load_col<T, R>(z, zb, c);
#pragma unroll
    for (int j = 0; j < CP; ++j) {
      const int i = lane + 32 * j;
      const T w = i < n_in ? W[i * sw + c] : (T)0;
#pragma unroll
      for (int r = 0; r < R; ++r) acc[j][r] = fma(z[r], w, acc[j][r]);
    }
  }
}

template <typename T, int R, int CP>
__device__ __forceinline__ void tr_gemvT2(T (&acc)[CP][R], T (&acd)[CP][R], const T* zb,
                                          const T* zbd, int n_out, const T* W, int sw, int n_in,
                                          int lane) {
#pragma unroll
  for (int j = 0; j < CP; ++j)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[j][r] = acd[j][r] = (T)0;
#pragma unroll 5
  for (int c = 0; c < n_out; ++c) {
    T z[R], zd[R];
    tr_load_col<T, R>(z, zb, c);
    tr_load_col<T, R>(zd, zbd, c);
#pragma unroll
    for (int j = 0; j < CP; ++j) {
      const int i = lane + 32 * j;
      const T w = i < n_in ? W[i * sw + c] : (T)0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        acc[j][r] = fma(z[r], w, acc[j][r]);
        acd[j][r] = fma(zd[r], w, acd[j][r]);
      }
    }
  }
}

// residual term of output channel c (< n_out), all R rows, from the staged
// input
template <typename T, int R>
__device__ __forceinline__ void tr_res_v(T (&o)[R], const T* in, int res, int c, int n_in) {
  if (res == TR_RES_IDENT) {
    stg_load<T, R>(o, in, c);
  } else if (res == TR_RES_DUP) {
    stg_load<T, R>(o, in, c < n_in ? c : c - n_in);
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = (T)0;
  }
}

// adjoint of the residual for input channel i (< n_in), all R rows, from the
// staged output adjoint
template <typename T, int R>
__device__ __forceinline__ void tr_res_adj_v(T (&o)[R], const T* gb, int res, int i, int n_in) {
  if (res == TR_RES_IDENT) {
    stg_load<T, R>(o, gb, i);
  } else if (res == TR_RES_DUP) {
    T u[R];
    stg_load<T, R>(o, gb, i);
    stg_load<T, R>(u, gb, i + n_in);
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] += u[r];
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) o[r] = (T)0;
  }
}

// sum over lanes of v[lane & (NV - 1)] (NV a power of two <= 32), NV - 1
// shuffles for the scatter plus log2(32 / NV) for the rest
template <int NV, typename T>
__device__ __forceinline__ T tr_reduce_scatter(T (&v)[NV], int lane) {
#pragma unroll
  for (int h = NV / 2; h >= 1; h >>= 1) {
    const bool up = (lane & h) != 0;
#pragma unroll
    for (int k = 0; k < h; ++k) {
      const T send = up ? v[k] : v[k + h];
      const T keep = up ? v[k + h] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
  T x = v[0];
#pragma unroll
  for (int o = NV; o < 32; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

struct TrAtom {
  int row, f, a0, i, ti;
  double xi[3], L[3];
  const double* fc;
};

__device__ __forceinline__ TrAtom tr_atom(const TrGeom& g, int row) {
  TrAtom A;
  A.row = row;
  A.f = g.fr.row_frame[row];
  A.a0 = g.fr.atom_off[A.f];
  A.i = row - A.a0;
  A.ti = g.type[row];
  A.fc = g.cw + 3 * (size_t)A.a0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    A.xi[d] = A.fc[3 * A.i + d];
    A.L[d] = g.fr.box ? g.fr.box[3 * A.f + d] : 0.0;
  }
  return A;
}

// env row R and its tangent Rd = ed . w of one slot, recomputed from the
// coordinates (padded slot: R = (0 - avg) / std, Rd = 0)
template <typename T>
__device__ __forceinline__ void tr_env_tangent(T Rv[4], T Rd[4], const TrGeom& g,
                                               const TrAtom& A, int slot, const T* av,
                                               const T* sd, const double* fbar,
                                               const double* vbar) {
  const int packed = g.nlist[(size_t)A.row * g.nnei + slot];
  if (packed >= 0) {
    T r[3];
    bt_rij<T>(r, A.fc, packed, A.xi, A.L);
    T v[4], gd[12];
    env_row<T>(r, g.rcut_smth, g.rcut, v, gd);
    const int j = packed / 27;
    const double* vb = vbar + 9 * (size_t)A.f;
    T w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      w[d] = (T)(fbar[3 * (size_t)(A.a0 + j) + d] - fbar[3 * (size_t)A.row + d] +
                 vb[3 * d + 0] * (double)r[0] + vb[3 * d + 1] * (double)r[1] +
                 vb[3 * d + 2] * (double)r[2]);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const T sa = sd[slot * 4 + a];
      Rv[a] = (v[a] - av[slot * 4 + a]) / sa;
      T acc = (T)0;
#pragma unroll
      for (int d = 0; d < 3; ++d) acc += (gd[a * 3 + d] / sa) * w[d];
      Rd[a] = acc;
    }
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      Rv[a] = ((T)0 - av[slot * 4 + a]) / sd[slot * 4 + a];
      Rd[a] = (T)0;
    }
  }
}

// xb[a][j] (lane channels c_j) += sum_k Db[c][k] X[a][k] + [c < ax] sum_m Db[m][c] X[a][m]
// with Db staged as [n3][sax] and X as [4][n3]
template <typename T>
__device__ __forceinline__ void tr_dbar_to_xbar(T (&xb)[4][TR_C3], const T* Db, const T* X,
                                                int n3, int ax, int sax, int lane) {
#pragma unroll
  for (int j = 0; j < TR_C3; ++j) {
    const int c = lane + 32 * j;
    if (c >= n3) continue;
    for (int k = 0; k < ax; ++k) {
      const T dv = Db[c * sax + k];
#pragma unroll
      for (int a = 0; a < 4; ++a) xb[a][j] = fma(dv, X[a * n3 + k], xb[a][j]);
    }
    if (c < ax)
      for (int m = 0; m < n3; ++m) {
        const T dv = Db[m * sax + c];
#pragma unroll
        for (int a = 0; a < 4; ++a) xb[a][j] = fma(dv, X[a * n3 + m], xb[a][j]);
      }
  }
}

template <typename T>
__device__ __forceinline__ void tr_stage_row(T* dst, const T* src, int n3, int ax, int sax,
                                             int lane) {
  for (int e = lane; e < n3 * ax; e += 32) dst[(e / ax) * sax + e % ax] = src[e];
}

template <typename T>
__device__ __forceinline__ T* tr_tbase(unsigned char* smem_raw, const TrLayout& lay) {
  return reinterpret_cast<T*>(smem_raw + (((size_t)lay.nw * lay.ints_warp * 4 + 15) & ~15));
}

template <typename T>
__device__ __forceinline__ T* tr_warp_base(unsigned char* smem_raw, const TrLayout& lay, int w,
                                           int*& ints) {
  ints = reinterpret_cast<int*>(smem_raw) + (size_t)w * lay.ints_warp;
  return tr_tbase<T>(smem_raw, lay) + lay.warp_off + (size_t)w * lay.warp_sz;
}

// lane channels of a per-atom [4][n3] vector from global memory
template <typename T>
__device__ __forceinline__ void tr_read_x4(T (&x)[4][TR_C3], const T* src, int n3, int lane) {
#pragma unroll
  for (int j = 0; j < TR_C3; ++j) {
    const int c = lane + 32 * j;
#pragma unroll
    for (int a = 0; a < 4; ++a) x[a][j] = c < n3 ? src[a * n3 + c] : (T)0;
  }
}

// ------------------------------------------------- per-atom adjoints of xyz --
// xb = (dJ/dxyz) / nnei and xbd = (dJ/dxyz') / nnei from the descriptor
// adjoints (D = xyz^T xyz[:, :ax], D' = xyz'^T xyz[:, :ax] + xyz^T xyz'[:, :ax]):
//   without Dd: xb from Dj only (force backward);
//   with Dd:    xbd from Dd and xyz; xb from Dj and xyz plus Dd and xyz'.
// One warp per atom, rows staged with the odd stride sax.
template <typename T>
__global__ void __launch_bounds__(64)
k_tr_xbar(T* __restrict__ xb_out, T* __restrict__ xbd_out, const T* __restrict__ xyz,
          const T* __restrict__ xyzd, const T* __restrict__ Dj, const T* __restrict__ Dd,
          const int* __restrict__ drow, int nrows, int n3, int ax, int nnei, int sax) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* base = reinterpret_cast<T*>(smem_raw) + (size_t)w * (8 * n3 + 2 * n3 * sax);
  T* X = base;
  T* Xd = base + 4 * n3;
  T* Sj = base + 8 * n3;
  T* Sd = Sj + n3 * sax;
  const T nn = (T)nnei;
  for (int row = blockIdx.x * 2 + w; row < nrows; row += gridDim.x * 2) {
    const size_t dr = (size_t)drow[row] * n3 * ax;
    for (int e = lane; e < 4 * n3; e += 32) {
      X[e] = xyz[(size_t)row * 4 * n3 + e];
      if (Dd) Xd[e] = xyzd[(size_t)row * 4 * n3 + e];
    }
    tr_stage_row(Sj, Dj + dr, n3, ax, sax, lane);
    if (Dd) tr_stage_row(Sd, Dd + dr, n3, ax, sax, lane);
    __syncwarp();
    T xb[4][TR_C3], xbd[4][TR_C3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < TR_C3; ++j) xb[a][j] = xbd[a][j] = (T)0;
    tr_dbar_to_xbar(xb, Sj, X, n3, ax, sax, lane);
    if (Dd) {
      tr_dbar_to_xbar(xb, Sd, Xd, n3, ax, sax, lane);
      tr_dbar_to_xbar(xbd, Sd, X, n3, ax, sax, lane);
    }
#pragma unroll
    for (int j = 0; j < TR_C3; ++j) {
      const int c = lane + 32 * j;
      if (c < n3)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          xb_out[((size_t)row * 4 + a) * n3 + c] = xb[a][j] / nn;
          if (Dd) xbd_out[((size_t)row * 4 + a) * n3 + c] = xbd[a][j] / nn;
        }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- forward --

template <typename T, int R, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 1)
k_tr_fwd(T* __restrict__ xyz_out, T* __restrict__ D_out, const T* __restrict__ em,
         TrNet<T> net, TrGeom g, TrLayout lay) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* sw = tr_tbase<T>(smem_raw, lay) + lay.w_off;
  if (TrTraits<T>::WSMEM) tr_stage_weights(sw, net, lay, g.ntypes);
  __syncthreads();
  int* ints;
  T* ws = tr_warp_base<T>(smem_raw, lay, w, ints);
  int* ent = ints;
  int* secn = ints + g.nnei;
  T *rr = ws + lay.o_rr, *mus = ws + lay.o_mu, *ss = ws + lay.o_s;
  T *A1 = ws + lay.o_A1, *A2 = ws + lay.o_A2, *big = ws + lay.o_big;
  // compile-time widths when N1 > 0 (the standard [25, 50, 100] net), else runtime
  constexpr bool WS = TrTraits<T>::WSMEM;
  const int n1 = N1 > 0 ? N1 : net.n1, n2 = N1 > 0 ? N2 : net.n2, n3 = N1 > 0 ? N3 : net.n3;
  const int res2 = N1 > 0 ? tr_res_kind(N2, N1) : net.res2;
  const int res3 = N1 > 0 ? tr_res_kind(N3, N2) : net.res3;
  const int sw2 = WS ? (n2 | 1) : n2, sw3 = WS ? (n3 | 1) : n3;
  const int gw = gridDim.x * lay.nw;
  for (int row = blockIdx.x * lay.nw + w; row < g.nrows; row += gw) {
    const int ti = g.type[row];
    const int* nl = g.nlist + (size_t)row * g.nnei;
    tr_entries(ent, secn, nl, g, ti, true, lane, 0, g.ntypes);
    T xyz[4][TR_C3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < TR_C3; ++j) xyz[a][j] = (T)0;
    for (int t = 0; t < g.ntypes; ++t) {
      const WV<T> W = tr_wview<T, WS>(net, sw, t, lay.pw, n1, n2, sw2, sw3);
      for (int e0 = secn[t]; e0 < secn[t + 1]; e0 += R) {
        const int ne = min(R, secn[t + 1] - e0);
        if (lane < R) {
          if (lane < ne) {
            const int en = ent[e0 + lane];
            const int slot = en & 0xFFFF;
            const T* src = em + ((size_t)row * g.nnei + slot) * 4;
#pragma unroll
            for (int a = 0; a < 4; ++a) rr[lane * 4 + a] = src[a];
            mus[lane] = (T)(en >> 16);
            ss[lane] = src[0];
          } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) rr[lane * 4 + a] = (T)0;
            mus[lane] = (T)0;
            ss[lane] = (T)0;
          }
        }
        __syncwarp();
        if (lane < n1) {
          const T w1 = W.W1[lane], b1 = W.b1[lane];
          T v1[R];
#pragma unroll
          for (int r = 0; r < R; ++r) v1[r] = tr_tanh(fma(ss[r], w1, b1));
          stg_store<T, R>(A1, lane, v1);
        }
        __syncwarp();
        {
          T acc[TR_C2][R];
          tr_gemv<T, R, TR_C2>(acc, A1, n1, W.W2, sw2, n2, lane);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int c = lane + 32 * j;
            if (c < n2) {
              const T bb = W.b2[c];
              T rs[R], v[R];
              tr_res_v<T, R>(rs, A1, res2, c, n1);
#pragma unroll
              for (int r = 0; r < R; ++r) v[r] = tr_tanh(acc[j][r] + bb) + rs[r];
              stg_store<T, R>(A2, c, v);
            }
          }
        }
        __syncwarp();
        {
          T acc[TR_C3][R];
          tr_gemv<T, R, TR_C3>(acc, A2, n2, W.W3, sw3, n3, lane);
#pragma unroll
          for (int j = 0; j < TR_C3; ++j) {
            const int c = lane + 32 * j;
            if (c < n3) {
              const T bb = W.b3[c];
              T rs[R];
              tr_res_v<T, R>(rs, A2, res3, c, n2);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T G = tr_tanh(acc[j][r] + bb) + rs[r];
                const T mg = mus[r] * G;
#pragma unroll
                for (int a = 0; a < 4; ++a) xyz[a][j] = fma(rr[r * 4 + a], mg, xyz[a][j]);
              }
            }
          }
        }
        __syncwarp();
      }
    }
    // xyz / nnei (se_a.py:844), D = xyz^T xyz[:, :ax]
    const T nn = (T)g.nnei;
    T* X = big;
#pragma unroll
    for (int j = 0; j < TR_C3; ++j) {
      const int c = lane + 32 * j;
      if (c < n3)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          xyz[a][j] = xyz[a][j] / nn;
          X[a * n3 + c] = xyz[a][j];
          xyz_out[((size_t)row * 4 + a) * n3 + c] = xyz[a][j];
        }
    }
    __syncwarp();
    T* Drow = D_out + (size_t)g.drow[row] * n3 * g.ax;
#pragma unroll
    for (int j = 0; j < TR_C3; ++j) {
      const int c = lane + 32 * j;
      if (c < n3)
        for (int k = 0; k < g.ax; ++k) {
          T d = (T)0;
#pragma unroll
          for (int a = 0; a < 4; ++a) d = fma(xyz[a][j], X[a * n3 + k], d);
          Drow[c * g.ax + k] = d;
        }
    }
    __syncwarp();
  }
}

// ------------------------------------------------------- force backward --

template <typename T, int R, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 1)
k_tr_bwd(T* __restrict__ gem, const T* __restrict__ em, const T* __restrict__ xbar,
         TrNet<T> net, TrGeom g, TrLayout lay) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* sw = tr_tbase<T>(smem_raw, lay) + lay.w_off;
  if (TrTraits<T>::WSMEM) tr_stage_weights(sw, net, lay, g.ntypes);
  __syncthreads();
  int* ints;
  T* ws = tr_warp_base<T>(smem_raw, lay, w, ints);
  int* ent = ints;
  int* secn = ints + g.nnei;
  T *rr = ws + lay.o_rr, *ss = ws + lay.o_s;
  T *A1 = ws + lay.o_A1, *A2 = ws + lay.o_A2, *big = ws + lay.o_big;
  // compile-time widths when N1 > 0 (the standard [25, 50, 100] net), else runtime
  constexpr bool WS = TrTraits<T>::WSMEM;
  const int n1 = N1 > 0 ? N1 : net.n1, n2 = N1 > 0 ? N2 : net.n2, n3 = N1 > 0 ? N3 : net.n3;
  const int res2 = N1 > 0 ? tr_res_kind(N2, N1) : net.res2;
  const int res3 = N1 > 0 ? tr_res_kind(N3, N2) : net.res3;
  const int sw2 = WS ? (n2 | 1) : n2, sw3 = WS ? (n3 | 1) : n3;
  const int gw = gridDim.x * lay.nw;
  for (int row = blockIdx.x * lay.nw + w; row < g.nrows; row += gw) {
    const int ti = g.type[row];
    const int* nl = g.nlist + (size_t)row * g.nnei;
    T xb[4][TR_C3];  // (dE/dxyz) / nnei, lane channels
    tr_read_x4(xb, xbar + (size_t)row * 4 * n3, n3, lane);
    tr_entries(ent, secn, nl, g, ti, false, lane, 0, g.ntypes);
    T* Zb3 = big;
    T* Gb = big + n3 * R;
    for (int t = 0; t < g.ntypes; ++t) {
      const WV<T> W = tr_wview<T, WS>(net, sw, t, lay.pw, n1, n2, sw2, sw3);
      for (int e0 = secn[t]; e0 < secn[t + 1]; e0 += R) {
        const int ne = min(R, secn[t + 1] - e0);
        if (lane < R) {
          if (lane < ne) {
            const int slot = ent[e0 + lane] & 0xFFFF;
            const T* src = em + ((size_t)row * g.nnei + slot) * 4;
#pragma unroll
            for (int a = 0; a < 4; ++a) rr[lane * 4 + a] = src[a];
            ss[lane] = src[0];
          } else {
#pragma unroll
            for (int a = 0; a < 4; ++a) rr[lane * 4 + a] = (T)0;
            ss[lane] = (T)0;
          }
        }
        __syncwarp();
        if (lane < n1) {
          const T w1 = W.W1[lane], b1 = W.b1[lane];
          T v1[R];
#pragma unroll
          for (int r = 0; r < R; ++r) v1[r] = tr_tanh(fma(ss[r], w1, b1));
          stg_store<T, R>(A1, lane, v1);
        }
        __syncwarp();
        {
          T acc[TR_C2][R];
          tr_gemv<T, R, TR_C2>(acc, A1, n1, W.W2, sw2, n2, lane);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int c = lane + 32 * j;
            if (c < n2) {
              const T bb = W.b2[c];
              T rs[R], v[R];
              tr_res_v<T, R>(rs, A1, res2, c, n1);
#pragma unroll
              for (int r = 0; r < R; ++r) v[r] = tr_tanh(acc[j][r] + bb) + rs[r];
              stg_store<T, R>(A2, c, v);
            }
          }
        }
        __syncwarp();
        T part[4 * R];  // dE/dR[r][a] partial over this lane's channels
#pragma unroll
        for (int k = 0; k < 4 * R; ++k) part[k] = (T)0;
        {
          T acc[TR_C3][R];
          tr_gemv<T, R, TR_C3>(acc, A2, n2, W.W3, sw3, n3, lane);
#pragma unroll
          for (int j = 0; j < TR_C3; ++j) {
            const int c = lane + 32 * j;
            if (c < n3) {
              const T bb = W.b3[c];
              T rs[R], zv[R], gv[R];
              tr_res_v<T, R>(rs, A2, res3, c, n2);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T y = tr_tanh(acc[j][r] + bb);
                const T G = y + rs[r];
                T gbar = (T)0;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                  part[r * 4 + a] = fma(G, xb[a][j], part[r * 4 + a]);
                  gbar = fma(rr[r * 4 + a], xb[a][j], gbar);
                }
                zv[r] = gbar * ((T)1 - y * y);
                gv[r] = gbar;
              }
              stg_store<T, R>(Zb3, c, zv);
              stg_store<T, R>(Gb, c, gv);
            }
          }
        }
        __syncwarp();
        // layer 2 adjoint, lanes over layer-2 channels
        T zb2[TR_C2][R], hb2[TR_C2][R];
        {
          tr_gemvT<T, R, TR_C2>(hb2, Zb3, n3, W.W3, sw3, n2, lane);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int i = lane + 32 * j;
            if (i < n2) {
              T ga[R], a2[R], rs[R];
              tr_res_adj_v<T, R>(ga, Gb, res3, i, n2);
              stg_load<T, R>(a2, A2, i);
              tr_res_v<T, R>(rs, A1, res2, i, n1);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                hb2[j][r] += ga[r];
                const T y2 = a2[r] - rs[r];
                zb2[j][r] = hb2[j][r] * ((T)1 - y2 * y2);
              }
            } else {
#pragma unroll
              for (int r = 0; r < R; ++r) zb2[j][r] = hb2[j][r] = (T)0;
            }
          }
        }
        __syncwarp();
        T* Zb2 = big;
        T* Hb2 = big + n2 * R;
#pragma unroll
        for (int j = 0; j < TR_C2; ++j) {
          const int i = lane + 32 * j;
          if (i < n2) {
            stg_store<T, R>(Zb2, i, zb2[j]);
            stg_store<T, R>(Hb2, i, hb2[j]);
          }
        }
        __syncwarp();
        {
          T hb1[TR_C1][R];
          tr_gemvT<T, R, TR_C1>(hb1, Zb2, n2, W.W2, sw2, n1, lane);
          if (lane < n1) {
            const T w1 = W.W1[lane];
            T ha[R], a1[R];
            tr_res_adj_v<T, R>(ha, Hb2, res2, lane, n1);
            stg_load<T, R>(a1, A1, lane);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const T h = hb1[0][r] + ha[r];
              const T y1 = a1[r];
              part[r * 4] = fma(h * ((T)1 - y1 * y1), w1, part[r * 4]);
            }
          }
        }
        const T tot = tr_reduce_scatter<4 * R, T>(part, lane);
        const int r = (lane >> 2) & (R - 1), a = lane & 3;
        if (lane < 4 * R && r < ne) {
          const int slot = ent[e0 + r] & 0xFFFF;
          gem[((size_t)row * g.nnei + slot) * 4 + a] = tot;
        }
        __syncwarp();
      }
    }
  }
}

// --------------------------------------------------------------- tangent --

template <typename T, int R, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 1)
k_tr_tan(T* __restrict__ xyzd_out, T* __restrict__ Dd_out, const T* __restrict__ xyz,
         const T* __restrict__ avg, const T* __restrict__ std_, const double* __restrict__ fbar,
         const double* __restrict__ vbar, TrNet<T> net, TrGeom g, TrLayout lay) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* sw = tr_tbase<T>(smem_raw, lay) + lay.w_off;
  if (TrTraits<T>::WSMEM) tr_stage_weights(sw, net, lay, g.ntypes);
  __syncthreads();
  int* ints;
  T* ws = tr_warp_base<T>(smem_raw, lay, w, ints);
  int* ent = ints;
  int* secn = ints + g.nnei;
  T *rr = ws + lay.o_rr, *rd = ws + lay.o_rd, *ss = ws + lay.o_s, *sd = ws + lay.o_sd;
  T *A1 = ws + lay.o_A1, *At1 = ws + lay.o_At1, *A2 = ws + lay.o_A2, *At2 = ws + lay.o_At2;
  T* big = ws + lay.o_big;
  // compile-time widths when N1 > 0 (the standard [25, 50, 100] net), else runtime
  constexpr bool WS = TrTraits<T>::WSMEM;
  const int n1 = N1 > 0 ? N1 : net.n1, n2 = N1 > 0 ? N2 : net.n2, n3 = N1 > 0 ? N3 : net.n3;
  const int res2 = N1 > 0 ? tr_res_kind(N2, N1) : net.res2;
  const int res3 = N1 > 0 ? tr_res_kind(N3, N2) : net.res3;
  const int sw2 = WS ? (n2 | 1) : n2, sw3 = WS ? (n3 | 1) : n3;
  const int gw = gridDim.x * lay.nw;
  for (int row = blockIdx.x * lay.nw + w; row < g.nrows; row += gw) {
    const TrAtom A = tr_atom(g, row);
    const T* av = avg + (size_t)A.ti * g.nnei * 4;
    const T* sdv = std_ + (size_t)A.ti * g.nnei * 4;
    tr_entries(ent, secn, g.nlist + (size_t)row * g.nnei, g, A.ti, false, lane, 0, g.ntypes);
    T xd[4][TR_C3];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < TR_C3; ++j) xd[a][j] = (T)0;
    for (int t = 0; t < g.ntypes; ++t) {
      const WV<T> W = tr_wview<T, WS>(net, sw, t, lay.pw, n1, n2, sw2, sw3);
      for (int e0 = secn[t]; e0 < secn[t + 1]; e0 += R) {
        const int ne = min(R, secn[t + 1] - e0);
        if (lane < R) {
          T Rv[4] = {(T)0, (T)0, (T)0, (T)0}, Rd[4] = {(T)0, (T)0, (T)0, (T)0};
          if (lane < ne)
            tr_env_tangent<T>(Rv, Rd, g, A, ent[e0 + lane] & 0xFFFF, av, sdv, fbar, vbar);
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            rr[lane * 4 + a] = Rv[a];
            rd[lane * 4 + a] = Rd[a];
          }
          ss[lane] = Rv[0];
          sd[lane] = Rd[0];
        }
        __syncwarp();
        if (lane < n1) {
          const T w1 = W.W1[lane], b1 = W.b1[lane];
          T v1[R], vt1[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const T y = tr_tanh(fma(ss[r], w1, b1));
            v1[r] = y;
            vt1[r] = ((T)1 - y * y) * (sd[r] * w1);
          }
          stg_store<T, R>(A1, lane, v1);
          stg_store<T, R>(At1, lane, vt1);
        }
        __syncwarp();
        {
          T acc[TR_C2][R], acd[TR_C2][R];
          tr_gemv2<T, R, TR_C2>(acc, acd, A1, At1, n1, W.W2, sw2, n2, lane);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int c = lane + 32 * j;
            if (c < n2) {
              const T bb = W.b2[c];
              T rs[R], rt[R], v[R], vt[R];
              tr_res_v<T, R>(rs, A1, res2, c, n1);
              tr_res_v<T, R>(rt, At1, res2, c, n1);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T y = tr_tanh(acc[j][r] + bb);
                v[r] = y + rs[r];
                vt[r] = ((T)1 - y * y) * acd[j][r] + rt[r];
              }
              stg_store<T, R>(A2, c, v);
              stg_store<T, R>(At2, c, vt);
            }
          }
        }
        __syncwarp();
        {
          T acc[TR_C3][R], acd[TR_C3][R];
          tr_gemv2<T, R, TR_C3>(acc, acd, A2, At2, n2, W.W3, sw3, n3, lane);
#pragma unroll
          for (int j = 0; j < TR_C3; ++j) {
            const int c = lane + 32 * j;
            if (c < n3) {
              const T bb = W.b3[c];
              T rs[R], rt[R];
              tr_res_v<T, R>(rs, A2, res3, c, n2);
              tr_res_v<T, R>(rt, At2, res3, c, n2);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T y = tr_tanh(acc[j][r] + bb);
                const T G = y + rs[r];
                const T Gd = ((T)1 - y * y) * acd[j][r] + rt[r];
#pragma unroll
                for (int a = 0; a < 4; ++a)
                  xd[a][j] = fma(rd[r * 4 + a], G, fma(rr[r * 4 + a], Gd, xd[a][j]));
              }
            }
          }
        }
        __syncwarp();
      }
    }
    // xyz' / nnei, D' = xyz'^T xyz[:, :ax] + xyz^T xyz'[:, :ax]
    const T nn = (T)g.nnei;
    T* X = big;
    T* Xd = big + 4 * n3;
    for (int e = lane; e < 4 * n3; e += 32) X[e] = xyz[(size_t)row * 4 * n3 + e];
#pragma unroll
    for (int j = 0; j < TR_C3; ++j) {
      const int c = lane + 32 * j;
      if (c < n3)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          xd[a][j] = xd[a][j] / nn;
          Xd[a * n3 + c] = xd[a][j];
          xyzd_out[((size_t)row * 4 + a) * n3 + c] = xd[a][j];
        }
    }
    __syncwarp();
    T* Drow = Dd_out + (size_t)g.drow[row] * n3 * g.ax;
#pragma unroll
    for (int j = 0; j < TR_C3; ++j) {
      const int c = lane + 32 * j;
      if (c < n3) {
        T xc[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) xc[a] = X[a * n3 + c];
        for (int k = 0; k < g.ax; ++k) {
          T d = (T)0;
#pragma unroll
          for (int a = 0; a < 4; ++a)
            d = fma(xd[a][j], X[a * n3 + k], fma(xc[a], Xd[a * n3 + k], d));
          Drow[c * g.ax + k] = d;
        }
      }
    }
    __syncwarp();
  }
}

// ------------------------------------------------- reverse over tangent --
// Neighbor types one after another: the block stages the weights of type t
// and every warp accumulates that net's gradient in a private shared-memory
// copy (plain adds, no atomics); the block sums its warps' copies into the
// global gradient after each type.

template <typename T, int R, int N1, int N2, int N3>
__global__ void __launch_bounds__(256, 1)
k_tr_rev(TrGrad<T> grad, const T* __restrict__ xbar, const T* __restrict__ xbard,
         const T* __restrict__ avg, const T* __restrict__ std_, const double* __restrict__ fbar,
         const double* __restrict__ vbar, TrNet<T> net, TrGeom g, TrLayout lay) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* tb = tr_tbase<T>(smem_raw, lay);
  T* sw = tb + lay.w_off;  // weights of the current type (at type 0 of the view)
  int* ints;
  T* ws = tr_warp_base<T>(smem_raw, lay, w, ints);
  int* ent = ints;
  int* secn = ints + g.nnei;
  T *rr = ws + lay.o_rr, *rd = ws + lay.o_rd, *mus = ws + lay.o_mu, *ss = ws + lay.o_s,
    *sd = ws + lay.o_sd;
  T *A1 = ws + lay.o_A1, *At1 = ws + lay.o_At1, *A2 = ws + lay.o_A2, *At2 = ws + lay.o_At2,
    *Zt2 = ws + lay.o_Zt2, *big = ws + lay.o_big;
  // compile-time widths when N1 > 0 (the standard [25, 50, 100] net), else runtime
  constexpr bool WS = TrTraits<T>::WSMEM;
  const int n1 = N1 > 0 ? N1 : net.n1, n2 = N1 > 0 ? N2 : net.n2, n3 = N1 > 0 ? N3 : net.n3;
  const int res2 = N1 > 0 ? tr_res_kind(N2, N1) : net.res2;
  const int res3 = N1 > 0 ? tr_res_kind(N3, N2) : net.res3;
  const int sw2 = WS ? (n2 | 1) : n2, sw3 = WS ? (n3 | 1) : n3;
  const int s2 = n2 | 1, s3 = n3 | 1;  // gradient copies: the staged layout
  // this warp's gradient copy, or the block's (lay.sacc: updated atomically)
  T* gacc = tb + lay.acc_off + (lay.sacc ? (size_t)0 : (size_t)w * lay.pw);
  auto gadd = [&](T* p, T v) {
    if (lay.sacc) atomicAdd(p, v);
    else *p += v;
  };
  T* gW1 = gacc;
  T* gb1 = gW1 + n1;
  T* gW2 = gb1 + n1;
  T* gb2 = gW2 + n1 * s2;
  T* gW3 = gb2 + n2;
  T* gb3 = gW3 + n2 * s3;
  const int gw = gridDim.x * lay.nw;
  for (int t = 0; t < g.ntypes; ++t) {
    __syncthreads();
    if (WS) {
      TrNet<T> one = net;
      one.W[0][0] = net.W[t][0];
      one.W[0][1] = net.W[t][1];
      one.W[0][2] = net.W[t][2];
      one.b[0][0] = net.b[t][0];
      one.b[0][1] = net.b[t][1];
      one.b[0][2] = net.b[t][2];
      tr_stage_weights(sw, one, lay, 1);
    }
    if (lay.sacc)
      for (int e = threadIdx.x; e < lay.pw; e += blockDim.x) gacc[e] = (T)0;
    else
      for (int e = lane; e < lay.pw; e += 32) gacc[e] = (T)0;
    __syncthreads();
    const WV<T> W = tr_wview<T, WS>(net, sw, WS ? 0 : t, lay.pw, n1, n2, sw2, sw3);
    for (int row = blockIdx.x * lay.nw + w; row < g.nrows; row += gw) {
      const TrAtom A = tr_atom(g, row);
      const T* av = avg + (size_t)A.ti * g.nnei * 4;
      const T* sdv = std_ + (size_t)A.ti * g.nnei * 4;
      tr_entries(ent, secn, g.nlist + (size_t)row * g.nnei, g, A.ti, true, lane, t, t + 1);
      if (secn[t + 1] == 0) continue;
      T xb[4][TR_C3], xbd[4][TR_C3];
      tr_read_x4(xb, xbar + (size_t)row * 4 * n3, n3, lane);
      tr_read_x4(xbd, xbard + (size_t)row * 4 * n3, n3, lane);
      for (int e0 = 0; e0 < secn[t + 1]; e0 += R) {
        const int ne = min(R, secn[t + 1] - e0);
        if (lane < R) {
          T Rv[4] = {(T)0, (T)0, (T)0, (T)0}, Rd[4] = {(T)0, (T)0, (T)0, (T)0};
          T mu = (T)0;
          if (lane < ne) {
            const int en = ent[e0 + lane];
            tr_env_tangent<T>(Rv, Rd, g, A, en & 0xFFFF, av, sdv, fbar, vbar);
            mu = (T)(en >> 16);
          }
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            rr[lane * 4 + a] = Rv[a];
            rd[lane * 4 + a] = Rd[a];
          }
          mus[lane] = mu;
          ss[lane] = Rv[0];
          sd[lane] = Rd[0];
        }
        __syncwarp();
        // forward and tangent of layers 1, 2
        if (lane < n1) {
          const T w1 = W.W1[lane], b1 = W.b1[lane];
          T v1[R], vt1[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const T y = tr_tanh(fma(ss[r], w1, b1));
            v1[r] = y;
            vt1[r] = ((T)1 - y * y) * (sd[r] * w1);
          }
          stg_store<T, R>(A1, lane, v1);
          stg_store<T, R>(At1, lane, vt1);
        }
        __syncwarp();
        {
          T acc[TR_C2][R], acd[TR_C2][R];
          tr_gemv2<T, R, TR_C2>(acc, acd, A1, At1, n1, W.W2, sw2, n2, lane);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int c = lane + 32 * j;
            if (c < n2) {
              const T bb = W.b2[c];
              T rs[R], rt[R], v[R], vt[R];
              tr_res_v<T, R>(rs, A1, res2, c, n1);
              tr_res_v<T, R>(rt, At1, res2, c, n1);
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T y = tr_tanh(acc[j][r] + bb);
                v[r] = y + rs[r];
                vt[r] = ((T)1 - y * y) * acd[j][r] + rt[r];
              }
              stg_store<T, R>(A2, c, v);
              stg_store<T, R>(At2, c, vt);
              stg_store<T, R>(Zt2, c, acd[j]);
            }
          }
        }
        __syncwarp();
        // layer 3: forward, tangent and its adjoints
        T* Zb3 = big;
        T* Zbt3 = big + n3 * R;
        T* Gb = big + 2 * n3 * R;
        T* Gbt = big + 3 * n3 * R;
        {
          T acc[TR_C3][R], acd[TR_C3][R];
          tr_gemv2<T, R, TR_C3>(acc, acd, A2, At2, n2, W.W3, sw3, n3, lane);
#pragma unroll
          for (int j = 0; j < TR_C3; ++j) {
            const int c = lane + 32 * j;
            if (c < n3) {
              const T bb = W.b3[c];
              T zsum = (T)0;
              T gv[R], gvt[R];
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const T y = tr_tanh(acc[j][r] + bb);
                const T q = (T)1 - y * y;
                T gbar = (T)0, gbard = (T)0;
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                  gbar = fma(rr[r * 4 + a], xb[a][j], fma(rd[r * 4 + a], xbd[a][j], gbar));
                  gbard = fma(rr[r * 4 + a], xbd[a][j], gbard);
                }
                gbar *= mus[r];
                gbard *= mus[r];
                const T zbd = gbard * q;
                const T zb = (gbar - (T)2 * y * acd[j][r] * gbard) * q;
                gv[r] = gbar;
                gvt[r] = gbard;
                zsum += zb;
                acc[j][r] = zb;   // reuse as z-bar
                acd[j][r] = zbd;  // and z-bar of the tangent
              }
              stg_store<T, R>(Zb3, c, acc[j]);
              stg_store<T, R>(Zbt3, c, acd[j]);
              stg_store<T, R>(Gb, c, gv);
              stg_store<T, R>(Gbt, c, gvt);
              gadd(&gb3[c], zsum);
            }
          }
          // W3 gradient: sum_r A2[i][r] zb[c][r] + At2[i][r] zbd[c][r]
          for (int i = 0; i < n2; ++i) {
            T a[R], ad[R];
            tr_load_col<T, R>(a, A2, i);
            tr_load_col<T, R>(ad, At2, i);
#pragma unroll
            for (int j = 0; j < TR_C3; ++j) {
              const int c = lane + 32 * j;
              if (c < n3) {
                T s = (T)0;
#pragma unroll
                for (int r = 0; r < R; ++r) s = fma(a[r], acc[j][r], fma(ad[r], acd[j][r], s));
                gadd(&gW3[i * s3 + c], s);
              }
            }
          }
        }
        __syncwarp();
        // layer 2 adjoints, lanes over layer-2 channels
        T zb2[TR_C2][R], zbd2[TR_C2][R], hb2[TR_C2][R], hbd2[TR_C2][R];
        tr_gemvT2<T, R, TR_C2>(hb2, hbd2, Zb3, Zbt3, n3, W.W3, sw3, n2, lane);
#pragma unroll
        for (int j = 0; j < TR_C2; ++j) {
          const int i = lane + 32 * j;
          if (i < n2) {
            T ga[R], gad[R], a2[R], rs[R], zt[R];
            tr_res_adj_v<T, R>(ga, Gb, res3, i, n2);
            tr_res_adj_v<T, R>(gad, Gbt, res3, i, n2);
            stg_load<T, R>(a2, A2, i);
            tr_res_v<T, R>(rs, A1, res2, i, n1);
            stg_load<T, R>(zt, Zt2, i);
            T zsum = (T)0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              hb2[j][r] += ga[r];
              hbd2[j][r] += gad[r];
              const T y = a2[r] - rs[r];
              const T q = (T)1 - y * y;
              zbd2[j][r] = hbd2[j][r] * q;
              zb2[j][r] = (hb2[j][r] - (T)2 * y * zt[r] * hbd2[j][r]) * q;
              zsum += zb2[j][r];
            }
            gadd(&gb2[i], zsum);
          } else {
#pragma unroll
            for (int r = 0; r < R; ++r) zb2[j][r] = zbd2[j][r] = hb2[j][r] = hbd2[j][r] = (T)0;
          }
        }
        for (int k = 0; k < n1; ++k) {
          T a[R], ad[R];
          tr_load_col<T, R>(a, A1, k);
          tr_load_col<T, R>(ad, At1, k);
#pragma unroll
          for (int j = 0; j < TR_C2; ++j) {
            const int i = lane + 32 * j;
            if (i < n2) {
              T s = (T)0;
#pragma unroll
              for (int r = 0; r < R; ++r) s = fma(a[r], zb2[j][r], fma(ad[r], zbd2[j][r], s));
              gadd(&gW2[k * s2 + i], s);
            }
          }
        }
        __syncwarp();
        T* Zb2 = big;
        T* Zbd2 = big + n2 * R;
        T* Hb2 = big + 2 * n2 * R;
        T* Hbd2 = big + 3 * n2 * R;
#pragma unroll
        for (int j = 0; j < TR_C2; ++j) {
          const int i = lane + 32 * j;
          if (i < n2) {
            stg_store<T, R>(Zb2, i, zb2[j]);
            stg_store<T, R>(Zbd2, i, zbd2[j]);
            stg_store<T, R>(Hb2, i, hb2[j]);
            stg_store<T, R>(Hbd2, i, hbd2[j]);
          }
        }
        __syncwarp();
        // layer 1, lanes over its channels
        {
          T hb1[TR_C1][R], hbd1[TR_C1][R];
          tr_gemvT2<T, R, TR_C1>(hb1, hbd1, Zb2, Zbd2, n2, W.W2, sw2, n1, lane);
          if (lane < n1) {
            const T w1 = W.W1[lane];
            T gws = (T)0, gbs = (T)0;
            T ha[R], had[R], a1[R];
            tr_res_adj_v<T, R>(ha, Hb2, res2, lane, n1);
            tr_res_adj_v<T, R>(had, Hbd2, res2, lane, n1);
            stg_load<T, R>(a1, A1, lane);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const T h = hb1[0][r] + ha[r];
              const T hd = hbd1[0][r] + had[r];
              const T y = a1[r];
              const T q = (T)1 - y * y;
              const T zd = sd[r] * w1;
              const T zbd = hd * q;
              const T zb = (h - (T)2 * y * zd * hd) * q;
              gws = fma(ss[r], zb, fma(sd[r], zbd, gws));
              gbs += zb;
            }
            gadd(&gW1[lane], gws);
            gadd(&gb1[lane], gbs);
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // the block's warps' copies -> the global gradient of net t (unpadded)
    const T* accb = tb + lay.acc_off;
    auto sumw = [&](int e) {
      T s = (T)0;
      for (int k = 0; k < (lay.sacc ? 1 : lay.nw); ++k) s += accb[(size_t)k * lay.pw + e];
      return s;
    };
    for (int k = threadIdx.x; k < n1; k += blockDim.x) {
      atomicAdd(&grad.W[t][0][k], sumw(k));
      atomicAdd(&grad.b[t][0][k], sumw(n1 + k));
    }
    for (int e = threadIdx.x; e < n1 * n2; e += blockDim.x)
      atomicAdd(&grad.W[t][1][e], sumw(2 * n1 + (e / n2) * s2 + e % n2));
    for (int k = threadIdx.x; k < n2; k += blockDim.x)
      atomicAdd(&grad.b[t][1][k], sumw(2 * n1 + n1 * s2 + k));
    for (int e = threadIdx.x; e < n2 * n3; e += blockDim.x)
      atomicAdd(&grad.W[t][2][e], sumw(2 * n1 + n1 * s2 + n2 + (e / n3) * s3 + e % n3));
    for (int k = threadIdx.x; k < n3; k += blockDim.x)
      atomicAdd(&grad.b[t][2][k], sumw(2 * n1 + n1 * s2 + n2 + n2 * s3 + k));
  }
}

// ------------------------------------------------------- fitting layers --
// Z = H_in W + b comes from the GEMM library; per element:

// y = tanh(z) (in place in Y); H = res(H_in) + d * y
template <typename T>
__global__ void k_fit_act(T* __restrict__ Y, T* __restrict__ H, const T* __restrict__ Hin,
                          const T* __restrict__ d, int n, int w_out, int w_in, int res) {
  pdl_wait();
  pdl_trigger();
  const long long tot = (long long)n * w_out;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % w_out);
    const long long i = e / w_out;
    const T y = tr_tanh(Y[e]);
    Y[e] = y;
    T h = d ? d[c] * y : y;
    if (res == TR_RES_IDENT) h += Hin[i * w_in + c];
    else if (res == TR_RES_DUP) h += Hin[i * w_in + (c < w_in ? c : c - w_in)];
    H[e] = h;
  }
}

// tangent: Hd = res(Hd_in) + d (1 - y^2) Zd, Zd = Hd_in W from the GEMM library
template <typename T>
__global__ void k_fit_tan(T* __restrict__ Hd, const T* __restrict__ Zd, const T* __restrict__ Hdin,
                          const T* __restrict__ Y, const T* __restrict__ d, int n, int w_out,
                          int w_in, int res) {
  pdl_wait();
  pdl_trigger();
  const long long tot = (long long)n * w_out;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % w_out);
    const long long i = e / w_out;
    const T y = Y[e];
    T h = ((T)1 - y * y) * Zd[e];
    if (d) h *= d[c];
    if (res == TR_RES_IDENT) h += Hdin[i * w_in + c];
    else if (res == TR_RES_DUP) h += Hdin[i * w_in + (c < w_in ? c : c - w_in)];
    Hd[e] = h;
  }
}

// first-order adjoint: Zb = G d (1 - y^2)
template <typename T>
__global__ void k_fit_bwd(T* __restrict__ Zb, const T* __restrict__ G, const T* __restrict__ Y,
                          const T* __restrict__ d, int n, int w) {
  pdl_wait();
  pdl_trigger();
  const long long tot = (long long)n * w;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const T y = Y[e];
    T z = G[e] * ((T)1 - y * y);
    if (d) z *= d[(int)(e % w)];
    Zb[e] = z;
  }
}

// reverse over tangent of one layer: from the adjoints A (of H) and Ad (of
// H'), Y = tanh(Z) and Zd = Z':
//   Zbd = d Ad q, Zb = (d A - 2 y Zd d Ad) q (q = 1 - y^2),
//   gb += sum_rows Zb, gd += sum_rows (A y + Ad q Zd)
// block (32, 8): columns over x, rows strided over y and the grid's y
template <typename T>
__global__ void k_fit_rev(T* __restrict__ Zb, T* __restrict__ Zbd, T* __restrict__ gb,
                          T* __restrict__ gd, const T* __restrict__ A, const T* __restrict__ Ad,
                          const T* __restrict__ Y, const T* __restrict__ Zd,
                          const T* __restrict__ d, int n, int w) {
  pdl_wait();
  pdl_trigger();
  __shared__ T red[2][8][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  T sb = (T)0, sd = (T)0;
  if (c < w) {
    const T dc = d ? d[c] : (T)1;
    for (int i = blockIdx.y * 8 + threadIdx.y; i < n; i += gridDim.y * 8) {
      const size_t e = (size_t)i * w + c;
      const T y = Y[e], q = (T)1 - y * y, zd = Zd[e], a = A[e], ad = Ad[e];
      const T ydb = dc * ad;
      const T zbd = ydb * q;
      const T zb = (dc * a - (T)2 * y * zd * ydb) * q;
      Zb[e] = zb;
      Zbd[e] = zbd;
      sb += zb;
      sd += a * y + ad * q * zd;
    }
  }
  red[0][threadIdx.y][threadIdx.x] = sb;
  red[1][threadIdx.y][threadIdx.x] = sd;
  __syncthreads();
  if (threadIdx.y == 0 && c < w) {
    T tb = (T)0, td = (T)0;
    for (int k = 0; k < 8; ++k) {
      tb += red[0][k][threadIdx.x];
      td += red[1][k][threadIdx.x];
    }
    atomicAdd(&gb[c], tb);
    if (gd) atomicAdd(&gd[c], td);
  }
}

// out[i][k] += G[i][k] (+ G[i][k + w_in] for a doubling layer), k < w_in
template <typename T>
__global__ void k_fit_res_adj(T* __restrict__ out, const T* __restrict__ G, int n, int w_out,
                              int w_in, int res) {
  pdl_wait();
  pdl_trigger();
  const long long tot = (long long)n * w_in;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e % w_in);
    const long long i = e / w_in;
    T v = G[i * w_out + k];
    if (res == TR_RES_DUP) v += G[i * w_out + k + w_in];
    if (res != TR_RES_NONE) out[e] += v;
  }
}

// atomic energy e[i] = H[i] . Wo + bo + ebias, one warp per row
template <typename T>
__global__ void k_fit_out(T* __restrict__ e, const T* __restrict__ H, const T* __restrict__ Wo,
                          const T* __restrict__ bo, T ebias, int n, int w) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31;
  for (long long i = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((long long)gridDim.x * blockDim.x) >> 5) {
    T s = (T)0;
    for (int k = lane; k < w; k += 32) s = fma(H[i * w + k], Wo[k], s);
    s = warp_sum(s);
    if (lane == 0) e[i] = s + bo[0] + ebias;
  }
}

// adjoints entering the last hidden layer: A[i] = lam[i] Wo (lam = 1 when
// null), Ad[i] = Wo (when Ad is given); output-layer gradients
// gWo += sum_i lam[i] H[i] + Hd[i], gbo += sum_i lam[i] (when gWo is given)
template <typename T>
__global__ void k_fit_out_adj(T* __restrict__ A, T* __restrict__ Ad, T* __restrict__ gWo,
                              T* __restrict__ gbo, const T* __restrict__ H,
                              const T* __restrict__ Hd, const T* __restrict__ Wo,
                              const T* __restrict__ lam, int n, int w) {
  pdl_wait();
  pdl_trigger();
  __shared__ T red[8][33];
  __shared__ T redb[8];
  const int c = blockIdx.x * 32 + threadIdx.x;
  T s = (T)0, sb = (T)0;
  for (int i = blockIdx.y * 8 + threadIdx.y; i < n; i += gridDim.y * 8) {
    const T l = lam ? lam[i] : (T)1;
    if (c < w) {
      const size_t e = (size_t)i * w + c;
      A[e] = l * Wo[c];
      if (Ad) Ad[e] = Wo[c];
      if (gWo) s += l * H[e] + (Hd ? Hd[e] : (T)0);
    }
    if (threadIdx.x == 0) sb += l;
  }
  if (!gWo) return;
  red[threadIdx.y][threadIdx.x] = s;
  if (threadIdx.x == 0) redb[threadIdx.y] = sb;
  __syncthreads();
  if (threadIdx.y == 0) {
    T t = (T)0;
    for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x];
    if (c < w) atomicAdd(&gWo[c], t);
    if (threadIdx.x == 0 && blockIdx.x == 0) {
      T tb = (T)0;
      for (int k = 0; k < 8; ++k) tb += redb[k];
      atomicAdd(gbo, tb);
    }
  }
}

// lam[drow[r]] = gE[row_frame[r]] (per-frame energy adjoint onto fitting rows)
template <typename T>
__global__ void k_tr_lam(T* __restrict__ lam, const double* __restrict__ gE,
                         const int* __restrict__ drow, const int* __restrict__ row_frame, int n) {
  pdl_wait();
  pdl_trigger();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    lam[drow[r]] = (T)gE[row_frame[r]];
}

// Adam (torch.optim.Adam, no weight decay, no amsgrad):
// m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
// p -= lr / bc1 * m / (sqrt(v) / sqrt(bc2) + eps);
// hp = {lr, bc1, sqrt(bc2)} on the device, so a captured step reads the
// current values
template <typename T>
__global__ void k_adam(T* __restrict__ p, const T* __restrict__ g, T* __restrict__ m,
                       T* __restrict__ v, long long n, const double* __restrict__ hp, double b1,
                       double b2, double eps) {
  pdl_wait();
  pdl_trigger();
  const T step = (T)(hp[0] / hp[1]);
  const T bc2s = (T)hp[2];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const T gg = g[e];
    const T mm = (T)b1 * m[e] + (T)(1.0 - b1) * gg;
    const T vv = (T)b2 * v[e] + (T)(1.0 - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    p[e] -= step * mm / (sqrt(vv) / bc2s + (T)eps);
  }
}

// ------------------------------------------------------------------ host --

struct TrDims {
  int n1, n2, n3, ax, nnei, ntypes;
};

enum TrKind { TR_FWD, TR_BWD, TR_TAN, TR_REV };

template <typename T>
static TrLayout tr_layout(TrKind kind, int R, const TrDims& d, bool wsmem, int nw,
                          bool sacc = false) {
  TrLayout L{};
  L.nw = nw;
  L.sacc = kind == TR_REV && sacc ? 1 : 0;
  L.ints_warp = (d.nnei + TR_MAXT + 1 + 3) & ~3;
  L.s2 = d.n2 | 1;
  L.s3 = d.n3 | 1;
  L.sax = d.ax | 1;
  L.pw = (2 * d.n1 + d.n1 * L.s2 + d.n2 + d.n2 * L.s3 + d.n3 + 3) & ~3;
  L.wsmem = wsmem ? 1 : 0;
  L.w_off = 0;
  if (kind == TR_REV) {  // one type's weights, then a gradient copy per warp (or block)
    L.acc_off = wsmem ? L.pw : 0;
    L.warp_off = L.acc_off + (L.sacc ? 1 : nw) * L.pw;
  } else {
    L.acc_off = wsmem ? d.ntypes * L.pw : 0;
    L.warp_off = L.acc_off;
  }
  const bool tan = kind == TR_TAN || kind == TR_REV;
  int o = 0;
  L.o_rr = o;
  o += 4 * R;
  L.o_rd = o;
  o += 4 * R;
  L.o_mu = o;
  o += R;
  L.o_s = o;
  o += R;
  L.o_sd = o;
  o += R;
  o = (o + 3) & ~3;
  L.o_A1 = o;
  o += d.n1 * R;
  L.o_At1 = o;
  if (tan) o += d.n1 * R;
  L.o_A2 = o;
  o += d.n2 * R;
  L.o_At2 = o;
  if (tan) o += d.n2 * R;
  L.o_Zt2 = o;
  if (kind == TR_REV) o += d.n2 * R;
  o = (o + 3) & ~3;
  L.o_big = o;
  int big = 4 * d.n3;
  if (kind == TR_BWD) big = std::max(2 * d.n3 * R, 2 * d.n2 * R);
  else if (kind == TR_TAN) big = 8 * d.n3;
  else if (kind == TR_REV) big = std::max(4 * d.n3 * R, 4 * d.n2 * R);
  o += big;
  L.warp_sz = (o + 3) & ~3;
  return L;
}

static size_t tr_smem_bytes(const TrLayout& L, size_t tsize) {
  const size_t ib = ((size_t)L.nw * L.ints_warp * 4 + 15) & ~(size_t)15;
  return ib + ((size_t)L.warp_off + (size_t)L.nw * L.warp_sz) * tsize;
}

// the standard embedding (1 -> 25 -> 50 -> 100, deepmd/dpmodel/descriptor/se_e2_a.py
// defaults) runs a build with compile-time widths; other widths the generic one
template <typename T>
static bool tr_std_net(const TrNet<T>& net) {
  return net.n1 == 25 && net.n2 == 50 && net.n3 == 100;
}

template <typename T>
static int tr_net(TrNet<T>& net, const T* const* W, const T* const* b, const int* widths,
                  int ntypes) {
  if (widths == nullptr || W == nullptr || b == nullptr || ntypes < 1 || ntypes > TR_MAXT) {
    set_error("se_a_train: invalid network arguments (ntypes=%d)", ntypes);
    return DPB_ERR_INVALID;
  }
  net.n1 = widths[1];
  net.n2 = widths[2];
  net.n3 = widths[3];
  if (widths[0] != 1 || net.n1 < 3 || net.n1 > 32 || net.n2 < 1 || net.n2 > 64 || net.n3 < 1 ||
      net.n3 > 128) {
    set_error("se_a_train: embedding widths [%d, %d, %d, %d] outside 1 -> (3..32) -> (..64) -> "
              "(..128)", widths[0], widths[1], widths[2], widths[3]);
    return DPB_ERR_INVALID;
  }
  net.res2 = net.n2 == net.n1 ? TR_RES_IDENT : (net.n2 == 2 * net.n1 ? TR_RES_DUP : TR_RES_NONE);
  net.res3 = net.n3 == net.n2 ? TR_RES_IDENT : (net.n3 == 2 * net.n2 ? TR_RES_DUP : TR_RES_NONE);
  for (int t = 0; t < ntypes; ++t)
    for (int l = 0; l < 3; ++l) {
      net.W[t][l] = W[t * 3 + l];
      net.b[t][l] = b[t * 3 + l];
      if (!net.W[t][l] || !net.b[t][l]) {
        set_error("se_a_train: null weight of type %d layer %d", t, l);
        return DPB_ERR_INVALID;
      }
    }
  return DPB_OK;
}

static int tr_geom(TrGeom& g, const double* cw, const int* type, const int* nlist,
                   const int* drow, const int* atom_off, const double* box, const int* row_frame,
                   int nframes, int nrows, const int* sec, int nsec, int ax,
                   const unsigned char* fold, float rcut, float rcut_smth) {
  if (sec == nullptr || nsec < 2 || nsec - 1 > TR_MAXT || sec[0] != 0 ||
      sec[nsec - 1] > BT_NMAX || sec[nsec - 1] < 1 || type == nullptr || nlist == nullptr ||
      drow == nullptr || ax < 1 || ax > TR_MAXAX || nrows < 0) {
    set_error("se_a_train: need 1..%d types, 1 <= sum(sel) <= %d, 1 <= axis <= %d", TR_MAXT,
              BT_NMAX, TR_MAXAX);
    return DPB_ERR_INVALID;
  }
  g = TrGeom{};
  g.fr = BtFrames{atom_off, nullptr, box, nullptr, row_frame, nframes};
  g.cw = cw;
  g.type = type;
  g.nlist = nlist;
  g.drow = drow;
  g.ntypes = nsec - 1;
  g.nnei = sec[nsec - 1];
  g.nrows = nrows;
  g.ax = ax;
  for (int k = 0; k < nsec; ++k) g.sec[k] = sec[k];
  g.fold = 0ull;
  if (fold)
    for (int ti = 0; ti < g.ntypes; ++ti)
      for (int t = 0; t < g.ntypes; ++t)
        if (fold[ti * g.ntypes + t]) g.fold |= 1ull << (ti * 8 + t);
  g.rcut = rcut;
  g.rcut_smth = rcut_smth;
  return DPB_OK;
}

template <typename K>
static int tr_launch_cfg(K kernel, const TrLayout& L, size_t tsize, int nrows, int& grid,
                         size_t& smem) {
  smem = tr_smem_bytes(L, tsize);
  if (smem > 227 * 1024) {
    set_error("se_a_train: %zu bytes of shared memory per block exceed 227 KB", smem);
    return DPB_ERR_INVALID;
  }
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    set_error("se_a_train: cannot reserve %zu bytes of shared memory", smem);
    return DPB_ERR_CUDA;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, L.nw * 32, smem);
  if (per_sm < 1) per_sm = 1;
  const int want = ceil_div(nrows, L.nw);
  grid = std::max(1, std::min(want, sm_count() * per_sm));
  return DPB_OK;
}

template <typename T>
static int tr_pick_warps(TrKind kind, const TrDims& d, int maxw, int R, bool sacc) {
  for (int nw = maxw; nw >= 1; --nw) {
    const TrLayout L = tr_layout<T>(kind, R, d, TrTraits<T>::WSMEM, nw, sacc);
    if (tr_smem_bytes(L, sizeof(T)) <= 227 * 1024) return nw;
  }
  return 0;
}

// rows per group: the train_rows_per_group knob for the FP32 standard net;
// train_rows_per_group_f64 for the FP64 force-backward kernel of the
// standard net (measured on the 12,288-atom FP64 plain step: backward 7.30
// ms with 4 rows, 5.88 ms with 8; the forward is faster with 4, 3.18 against
// 3.46 ms, and the tangent and reverse kernels spill at 8); else the
// precision's default
template <typename T>
static int tr_rows(const TrNet<T>& net, TrKind kind) {
  if (!tr_std_net(net)) return TrTraits<T>::R;
  if (sizeof(T) == 4) return tune_value("train_rows_per_group", TrTraits<T>::R) == 4 ? 4 : 8;
  if (kind != TR_BWD) return TrTraits<T>::R;
  return tune_value("train_rows_per_group_f64", 8) == 4 ? 4 : 8;
}

template <typename T>
static int tr_prepare(TrKind kind, TrNet<T>& net, TrGeom& g, TrLayout& L, int& R,
                      const T* const* W,
                      const T* const* b, const int* widths, const double* cw, const int* type,
                      const int* nlist, const int* drow, const int* atom_off, const double* box,
                      const int* row_frame, int nframes, int nrows, const int* sec, int nsec,
                      int ax, const unsigned char* fold, float rcut, float rcut_smth) {
  int rc = tr_geom(g, cw, type, nlist, drow, atom_off, box, row_frame, nframes, nrows, sec, nsec,
                   ax, fold, rcut, rcut_smth);
  if (rc) return rc;
  rc = tr_net<T>(net, W, b, widths, g.ntypes);
  if (rc) return rc;
  if (ax > net.n3) {
    set_error("se_a_train: axis %d larger than the embedding width %d", ax, net.n3);
    return DPB_ERR_INVALID;
  }
  const TrDims d{net.n1, net.n2, net.n3, ax, g.nnei, g.ntypes};
  R = tr_rows(net, kind);
  // the reverse pass: a gradient copy per warp (at most 4 warps fit), or one
  // per block updated with shared-memory atomics (up to 8 warps)
  const bool sacc = kind == TR_REV && tune_value("train_rev_shared_acc", 1) != 0;
  const int maxw =
      std::min(tune_value("train_warps_per_cta", 8), kind == TR_REV && !sacc ? 4 : 8);
  const int nw = tr_pick_warps<T>(kind, d, maxw, R, sacc);
  if (nw < 1) {
    set_error("se_a_train: the network does not fit in shared memory");
    return DPB_ERR_INVALID;
  }
  L = tr_layout<T>(kind, R, d, TrTraits<T>::WSMEM, nw, sacc);
  return DPB_OK;
}

static int fit_grid(long long items) { return grid_stride_blocks(items, 256); }

template <typename T>
static int tr_xbar(T* xb, T* xbd, const T* xyz, const T* xyzd, const T* Dj, const T* Dd,
                   const int* drow, int nrows, int n3, int ax, int nnei, cudaStream_t st) {
  const int sax = ax | 1;
  const size_t smem = 2 * (size_t)(8 * n3 + 2 * n3 * sax) * sizeof(T);
  if (cudaFuncSetAttribute(k_tr_xbar<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess) {
    set_error("se_a_train: cannot reserve %zu bytes of shared memory", smem);
    return DPB_ERR_CUDA;
  }
  const int grid = std::max(1, std::min(ceil_div(nrows, 2), sm_count() * 8));
  DPB_CUDA(launch_pdl(k_tr_xbar<T>, dim3(grid), dim3(64), smem, st, xb, xbd, xyz, xyzd, Dj,
        Dd, drow, nrows, n3, ax, nnei, sax), "se_a_train/xbar");
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;

#define DPB_TRAIN_ENTRIES(SUF, T)                                                               \
  int dpb_se_a_train_fwd_##SUF(T* xyz, T* descrpt, const T* em, const int* nlist,              \
                               const int* type, const int* drow, const T* const* W,             \
                               const T* const* b, const int* widths, const int* sec, int nsec,  \
                               int nrows, int axis, const unsigned char* fold,                  \
                               dpb_stream_t stream) {                                           \
    TrNet<T> net;                                                                               \
    TrGeom g;                                                                                   \
    TrLayout L;                                                                                 \
    int R;                                                                                      \
    int rc = tr_prepare<T>(TR_FWD, net, g, L, R, W, b, widths, nullptr, type, nlist, drow,         \
                           nullptr, nullptr, nullptr, 0, nrows, sec, nsec, axis, fold, 0.f, 0.f); \
    if (rc) return rc;                                                                          \
    if (nrows == 0) return DPB_OK;                                                              \
    if (!xyz || !descrpt || !em) {                                                              \
      set_error("se_a_train_fwd: null buffer");                                                 \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    auto kern = !tr_std_net(net) ? k_tr_fwd<T, TrTraits<T>::R, 0, 0, 0>                         \
                : (R == 4 ? k_tr_fwd<T, 4, 25, 50, 100> : k_tr_fwd<T, 8, 25, 50, 100>);\
    int grid;                                                                                   \
    size_t smem;                                                                                \
    rc = tr_launch_cfg(kern, L, sizeof(T), nrows, grid, smem);                                  \
    if (rc) return rc;                                                                          \
    DPB_CUDA(launch_pdl(kern, dim3(grid), dim3(L.nw * 32), smem, as_stream(stream), xyz,         \
          descrpt, em, net, g, L), "se_a_train_fwd");                                            \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_se_a_train_bwd_##SUF(T* net_deriv, T* scratch, const T* em, const T* xyz,          \
                               const T* d_descrpt, const int* nlist, const int* type,           \
                               const int* drow, const T* const* W, const T* const* b,           \
                               const int* widths, const int* sec, int nsec, int nrows, int axis,\
                               dpb_stream_t stream) {                                           \
    TrNet<T> net;                                                                               \
    TrGeom g;                                                                                   \
    TrLayout L;                                                                                 \
    int R;                                                                                      \
    int rc = tr_prepare<T>(TR_BWD, net, g, L, R, W, b, widths, nullptr, type, nlist, drow,         \
                           nullptr, nullptr, nullptr, 0, nrows, sec, nsec, axis, nullptr, 0.f,  \
                           0.f);                                                                \
    if (rc) return rc;                                                                          \
    if (nrows == 0) return DPB_OK;                                                              \
    if (!net_deriv || !scratch || !em || !xyz || !d_descrpt) {                                  \
      set_error("se_a_train_bwd: null buffer");                                                 \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    cudaStream_t st = as_stream(stream);                                                        \
    DPB_CUDA(cudaMemsetAsync(net_deriv, 0, sizeof(T) * (size_t)nrows * g.nnei * 4, st),         \
             "se_a_train_bwd");                                                                 \
    rc = tr_xbar<T>(scratch, nullptr, xyz, nullptr, d_descrpt, nullptr, drow, nrows, net.n3,    \
                    axis, g.nnei, st);                                                          \
    if (rc) return rc;                                                                          \
    auto kern = !tr_std_net(net) ? k_tr_bwd<T, TrTraits<T>::R, 0, 0, 0>                         \
                : (R == 4 ? k_tr_bwd<T, 4, 25, 50, 100> : k_tr_bwd<T, 8, 25, 50, 100>);\
    int grid;                                                                                   \
    size_t smem;                                                                                \
    rc = tr_launch_cfg(kern, L, sizeof(T), nrows, grid, smem);                                  \
    if (rc) return rc;                                                                          \
    DPB_CUDA(launch_pdl(kern, dim3(grid), dim3(L.nw * 32), smem, st, net_deriv, em, scratch,     \
          net, g, L), "se_a_train_bwd");                                                         \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_se_a_train_tan_##SUF(T* xyz_t, T* descrpt_t, const T* xyz, const T* avg,             \
                               const T* std_, const double* force_bar,                          \
                               const double* virial_bar, const double* cw, const int* nlist,    \
                               const int* type, const int* drow, const int* atom_off,           \
                               const double* box, const int* row_frame, int nframes,            \
                               const T* const* W, const T* const* b, const int* widths,         \
                               const int* sec, int nsec, int nrows, int axis, float rcut,       \
                               float rcut_smth, dpb_stream_t stream) {                          \
    TrNet<T> net;                                                                               \
    TrGeom g;                                                                                   \
    TrLayout L;                                                                                 \
    int R;                                                                                      \
    int rc = tr_prepare<T>(TR_TAN, net, g, L, R, W, b, widths, cw, type, nlist, drow, atom_off,    \
                           box, row_frame, nframes, nrows, sec, nsec, axis, nullptr, rcut,      \
                           rcut_smth);                                                          \
    if (rc) return rc;                                                                          \
    if (nrows == 0) return DPB_OK;                                                              \
    if (!xyz_t || !descrpt_t || !xyz || !avg || !std_ || !force_bar || !virial_bar || !cw ||    \
        !atom_off || !box || !row_frame) {                                                      \
      set_error("se_a_train_tan: null buffer");                                                 \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    auto kern = !tr_std_net(net) ? k_tr_tan<T, TrTraits<T>::R, 0, 0, 0>                         \
                : (R == 4 ? k_tr_tan<T, 4, 25, 50, 100> : k_tr_tan<T, 8, 25, 50, 100>);\
    int grid;                                                                                   \
    size_t smem;                                                                                \
    rc = tr_launch_cfg(kern, L, sizeof(T), nrows, grid, smem);                                  \
    if (rc) return rc;                                                                          \
    DPB_CUDA(launch_pdl(kern, dim3(grid), dim3(L.nw * 32), smem, as_stream(stream), xyz_t,       \
          descrpt_t, xyz, avg, std_, force_bar, virial_bar, net, g, L), "se_a_train_tan");       \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_se_a_train_rev_##SUF(T* const* gW, T* const* gb, T* scratch, const T* xyz,         \
                               const T* xyz_t, const T* d_descrpt, const T* d_descrpt_t,        \
                               const T* avg, const T* std_, const double* force_bar,            \
                               const double* virial_bar, const double* cw, const int* nlist,    \
                               const int* type, const int* drow, const int* atom_off,           \
                               const double* box, const int* row_frame, int nframes,            \
                               const T* const* W, const T* const* b, const int* widths,         \
                               const int* sec, int nsec, int nrows, int axis,                   \
                               const unsigned char* fold, float rcut, float rcut_smth,          \
                               dpb_stream_t stream) {                                           \
    TrNet<T> net;                                                                               \
    TrGeom g;                                                                                   \
    TrLayout L;                                                                                 \
    int R;                                                                                      \
    int rc = tr_prepare<T>(TR_REV, net, g, L, R, W, b, widths, cw, type, nlist, drow, atom_off,    \
                           box, row_frame, nframes, nrows, sec, nsec, axis, fold, rcut,         \
                           rcut_smth);                                                          \
    if (rc) return rc;                                                                          \
    if (nrows == 0) return DPB_OK;                                                              \
    if (!gW || !gb || !scratch || !xyz || !xyz_t || !d_descrpt || !d_descrpt_t || !avg ||       \
        !std_ || !force_bar || !virial_bar || !cw || !atom_off || !box || !row_frame) {         \
      set_error("se_a_train_rev: null buffer");                                                 \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    TrGrad<T> gr;                                                                               \
    for (int t = 0; t < g.ntypes; ++t)                                                          \
      for (int l = 0; l < 3; ++l) {                                                             \
        gr.W[t][l] = gW[t * 3 + l];                                                             \
        gr.b[t][l] = gb[t * 3 + l];                                                             \
        if (!gr.W[t][l] || !gr.b[t][l]) {                                                       \
          set_error("se_a_train_rev: null gradient of type %d layer %d", t, l);                 \
          return DPB_ERR_INVALID;                                                               \
        }                                                                                       \
      }                                                                                         \
    cudaStream_t st = as_stream(stream);                                                        \
    T* xb = scratch;                                                                            \
    T* xbd = scratch + (size_t)nrows * 4 * net.n3;                                              \
    rc = tr_xbar<T>(xb, xbd, xyz, xyz_t, d_descrpt, d_descrpt_t, drow, nrows, net.n3, axis,     \
                    g.nnei, st);                                                                \
    if (rc) return rc;                                                                          \
    auto kern = !tr_std_net(net) ? k_tr_rev<T, TrTraits<T>::R, 0, 0, 0>                         \
                : (R == 4 ? k_tr_rev<T, 4, 25, 50, 100> : k_tr_rev<T, 8, 25, 50, 100>);\
    int grid;                                                                                   \
    size_t smem;                                                                                \
    rc = tr_launch_cfg(kern, L, sizeof(T), nrows, grid, smem);                                  \
    if (rc) return rc;                                                                          \
    DPB_CUDA(launch_pdl(kern, dim3(grid), dim3(L.nw * 32), smem, st, gr, xb, xbd, avg, std_,     \
          force_bar, virial_bar, net, g, L), "se_a_train_rev");                                  \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_act_##SUF(T* Y, T* H, const T* Hin, const T* d, int n, int w_out, int w_in,      \
                        dpb_stream_t stream) {                                                  \
    if (n <= 0) return DPB_OK;                                                                  \
    const int res = w_out == w_in ? TR_RES_IDENT : (w_out == 2 * w_in ? TR_RES_DUP : TR_RES_NONE); \
    DPB_CUDA(launch_pdl(k_fit_act<T>, dim3(fit_grid((long long)n * w_out)), dim3(256), 0,        \
          as_stream(stream), Y, H, Hin, d, n, w_out, w_in, res), "fit_act");                     \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_tan_##SUF(T* Hd, const T* Zd, const T* Hdin, const T* Y, const T* d, int n,      \
                        int w_out, int w_in, dpb_stream_t stream) {                             \
    if (n <= 0) return DPB_OK;                                                                  \
    const int res = w_out == w_in ? TR_RES_IDENT : (w_out == 2 * w_in ? TR_RES_DUP : TR_RES_NONE); \
    DPB_CUDA(launch_pdl(k_fit_tan<T>, dim3(fit_grid((long long)n * w_out)), dim3(256), 0,        \
          as_stream(stream), Hd, Zd, Hdin, Y, d, n, w_out, w_in, res), "fit_tan");               \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_bwd_##SUF(T* Zb, const T* G, const T* Y, const T* d, int n, int w,               \
                        dpb_stream_t stream) {                                                  \
    if (n <= 0) return DPB_OK;                                                                  \
    DPB_CUDA(launch_pdl(k_fit_bwd<T>, dim3(fit_grid((long long)n * w)), dim3(256), 0,            \
          as_stream(stream), Zb, G, Y, d, n, w), "fit_bwd");                                     \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_rev_##SUF(T* Zb, T* Zbd, T* gb, T* gd, const T* A, const T* Ad, const T* Y,      \
                        const T* Zd, const T* d, int n, int w, dpb_stream_t stream) {           \
    if (n <= 0) return DPB_OK;                                                                  \
    dim3 grid(ceil_div(w, 32), std::max(1, std::min(ceil_div(n, 8), 64)));                      \
    DPB_CUDA(launch_pdl(k_fit_rev<T>, dim3(grid), dim3(dim3(32, 8)), 0, as_stream(stream), Zb,   \
          Zbd, gb, gd, A, Ad, Y, Zd, d, n, w), "fit_rev");                                       \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_res_adj_##SUF(T* out, const T* G, int n, int w_out, int w_in,                    \
                            dpb_stream_t stream) {                                              \
    if (n <= 0) return DPB_OK;                                                                  \
    const int res = w_out == w_in ? TR_RES_IDENT : (w_out == 2 * w_in ? TR_RES_DUP : TR_RES_NONE); \
    if (res == TR_RES_NONE) return DPB_OK;                                                      \
    DPB_CUDA(launch_pdl(k_fit_res_adj<T>, dim3(fit_grid((long long)n * w_in)), dim3(256), 0,     \
          as_stream(stream), out, G, n, w_out, w_in, res), "fit_res_adj");                       \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_out_##SUF(T* e, const T* H, const T* Wo, const T* bo, double ebias, int n, int w, \
                        dpb_stream_t stream) {                                                  \
    if (n <= 0) return DPB_OK;                                                                  \
    DPB_CUDA(launch_pdl(k_fit_out<T>, dim3(fit_grid((long long)n * 32)), dim3(256), 0,           \
          as_stream(stream), e, H, Wo, bo, (T)ebias, n, w), "fit_out");                          \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_fit_out_adj_##SUF(T* A, T* Ad, T* gWo, T* gbo, const T* H, const T* Hd, const T* Wo, \
                            const T* lam, int n, int w, dpb_stream_t stream) {                  \
    if (n <= 0) return DPB_OK;                                                                  \
    if ((gWo == nullptr) != (gbo == nullptr)) {                                                 \
      set_error("fit_out_adj: give both output-layer gradients or neither");                    \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    dim3 grid(ceil_div(w, 32), std::max(1, std::min(ceil_div(n, 8), 64)));                      \
    DPB_CUDA(launch_pdl(k_fit_out_adj<T>, dim3(grid), dim3(dim3(32, 8)), 0, as_stream(stream),   \
          A, Ad, gWo, gbo, H, Hd, Wo, lam, n, w), "fit_out_adj");                                \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_train_lam_##SUF(T* lam, const double* gE, const int* drow, const int* row_frame,     \
                          int n, dpb_stream_t stream) {                                         \
    if (n <= 0) return DPB_OK;                                                                  \
    DPB_CUDA(launch_pdl(k_tr_lam<T>, dim3(fit_grid(n)), dim3(256), 0, as_stream(stream), lam,    \
          gE, drow, row_frame, n), "train_lam");                                                 \
    return DPB_OK;                                                                              \
  }                                                                                             \
  int dpb_adam_##SUF(T* p, const T* g, T* m, T* v, long long n, const double* hp, double beta1, \
                     double beta2, double eps, dpb_stream_t stream) {                           \
    if (n <= 0) return DPB_OK;                                                                  \
    if (!p || !g || !m || !v || !hp) {                                                          \
      set_error("adam: null buffer");                                                           \
      return DPB_ERR_INVALID;                                                                   \
    }                                                                                           \
    DPB_CUDA(launch_pdl(k_adam<T>, dim3(fit_grid(n)), dim3(256), 0, as_stream(stream), p, g,     \
          m, v, n, hp, beta1, beta2, eps), "adam");                                              \
    return DPB_OK;                                                                              \
  }

extern "C" {
DPB_TRAIN_ENTRIES(f32, float)
DPB_TRAIN_ENTRIES(f64, double)
}  // extern "C"
