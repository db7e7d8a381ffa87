// Neighbor lists and the smooth environment matrix (se_e2_a).
//
// One warp owns one center atom. Candidates (from the cell grid, or from an
// input list) are filtered with the reference's exact tests, packed into
// 64-bit keys (type, float r^2 bits, index) in shared memory and ranked in
// place; the rank gives the sel slot. This reproduces format_nlist_i_cpu
// (source/lib/src/fmt_nlist.cc:98-143) bit for bit: the reference GPU path
// (source/lib/src/gpu/prod_env_mat.cu:86-219) instead sorts on a distance
// truncated to 2^-26 A with a per-atom CUB radix sort over a global key
// buffer and traps on key overflow; here there is no global scratch and an
// overflow sets a status bit.
#include "dpb_common.cuh"
#include "dpb_envmath.cuh"
#include "dpb_internal.cuh"

namespace dpb {

constexpr int MAXT = 32;    // neighbor types supported (sec has <= 33 entries)
constexpr int NMAX = 512;   // max sum(sel) per atom

struct SecInfo {
  int ntypes;
  int nnei;
  int sec[MAXT + 1];
};

static int make_sec(SecInfo& s, const int* sec, int nsec) {
  if (sec == nullptr || nsec < 2 || nsec - 1 > MAXT) {
    set_error("sec must have between 2 and %d entries (got %d)", MAXT + 1, nsec);
    return DPB_ERR_INVALID;
  }
  s.ntypes = nsec - 1;
  for (int k = 0; k < nsec; ++k) {
    s.sec[k] = sec[k];
    if (k > 0 && sec[k] < sec[k - 1]) {
      set_error("sec must be non-decreasing");
      return DPB_ERR_INVALID;
    }
  }
  if (sec[0] != 0) {
    set_error("sec[0] must be 0");
    return DPB_ERR_INVALID;
  }
  s.nnei = sec[nsec - 1];
  if (s.nnei > NMAX) {
    set_error("sum(sel)=%d exceeds the supported maximum %d", s.nnei, NMAX);
    return DPB_ERR_INVALID;
  }
  return DPB_OK;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Candidate test + key. FUSED: build_nlist's strict FP test on c_i - c_j
// (neighbor_list.cc:896-912) and format's float test on (float)c_j -
// (float)c_i (fmt_nlist.cc:114-127). Otherwise only the format test.
template <typename CT, bool FUSED>
__device__ __forceinline__ bool accept(unsigned long long& key, int j, int i,
                                       int ti, const CT* fc, const int* ft,
                                       const CT xi[3], const float fxi[3],
                                       CT rc2, float rc2f, int ntypes,
                                       int* status) {
  int tj = ft[j];
  if (tj < 0) return false;
  if (FUSED) {
    if (j == i || ti < 0) return false;
    CT d0 = sub_rn(xi[0], fc[3 * j + 0]);
    CT d1 = sub_rn(xi[1], fc[3 * j + 1]);
    CT d2 = sub_rn(xi[2], fc[3 * j + 2]);
    if (!(dot3_rn(d0, d1, d2) < rc2)) return false;
  }
  float e0 = sub_rn((float)fc[3 * j + 0], fxi[0]);
  float e1 = sub_rn((float)fc[3 * j + 1], fxi[1]);
  float e2 = sub_rn((float)fc[3 * j + 2], fxi[2]);
  float r2 = dot3_rn(e0, e1, e2);
  if (!(r2 <= rc2f)) return false;
  if (tj >= 128 || j >= (1 << 24)) {
    atomicOr(status, ST_KEY_OVERFLOW);
    return false;
  }
  if (tj >= ntypes) return false;  // no sel slot exists for this type
  key = ((unsigned long long)tj << 56) |
        ((unsigned long long)__float_as_uint(r2) << 24) | (unsigned long long)j;
  return true;
}

// accept<double, true> on one cell-ordered record of the grid (x, y, z and
// type << 32 | index as the fourth double's bits): the same tests on the
// same values, the record read as two 16-byte loads instead of the index,
// the type and three coordinates gathered
__device__ __forceinline__ bool accept_packed(unsigned long long& key, const double4* rec, int i,
                                              int ti, const double xi[3], const float fxi[3],
                                              double rc2, float rc2f, int ntypes, int* status) {
  const double2 xy = __ldg(reinterpret_cast<const double2*>(rec));
  const double2 zw = __ldg(reinterpret_cast<const double2*>(rec) + 1);
  const long long w = __double_as_longlong(zw.y);
  const int j = (int)(unsigned)(w & 0xffffffffll);
  const int tj = (int)(w >> 32);
  if (tj < 0) return false;
  if (j == i || ti < 0) return false;
  double d0 = sub_rn(xi[0], xy.x);
  double d1 = sub_rn(xi[1], xy.y);
  double d2 = sub_rn(xi[2], zw.x);
  if (!(dot3_rn(d0, d1, d2) < rc2)) return false;
  float e0 = sub_rn((float)xy.x, fxi[0]);
  float e1 = sub_rn((float)xy.y, fxi[1]);
  float e2 = sub_rn((float)zw.x, fxi[2]);
  float r2 = dot3_rn(e0, e1, e2);
  if (!(r2 <= rc2f)) return false;
  if (tj >= 128 || j >= (1 << 24)) {
    atomicOr(status, ST_KEY_OVERFLOW);
    return false;
  }
  if (tj >= ntypes) return false;  // no sel slot exists for this type
  key = ((unsigned long long)tj << 56) |
        ((unsigned long long)__float_as_uint(r2) << 24) | (unsigned long long)j;
  return true;
}

// em row = (v - avg) / std, or zeros for a center without a type row.
template <typename OT>
__device__ __forceinline__ void store_env_row(OT* e, const OT* a, const OT* s, const OT (&v)[4],
                                              bool valid) {
#pragma unroll
  for (int k = 0; k < 4; ++k) e[k] = valid ? (v[k] - a[k]) / s[k] : (OT)0.;
}
// FP32 rows: one 16-byte load of avg and of std and one 16-byte store when
// the three rows are 16-byte aligned (the same arithmetic either way)
template <>
__device__ __forceinline__ void store_env_row<float>(float* e, const float* a, const float* s,
                                                     const float (&v)[4], bool valid) {
  if (((reinterpret_cast<uintptr_t>(e) | reinterpret_cast<uintptr_t>(a) |
        reinterpret_cast<uintptr_t>(s)) & 15) != 0) {
#pragma unroll
    for (int k = 0; k < 4; ++k) e[k] = valid ? (v[k] - a[k]) / s[k] : 0.f;
    return;
  }
  float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
  if (valid) {
    const float4 a4 = *reinterpret_cast<const float4*>(a);
    const float4 s4 = *reinterpret_cast<const float4*>(s);
    o = make_float4((v[0] - a4.x) / s4.x, (v[1] - a4.y) / s4.y, (v[2] - a4.z) / s4.z,
                    (v[3] - a4.w) / s4.w);
  }
  *reinterpret_cast<float4*>(e) = o;
}

// Shared-memory workspace of one warp (one center atom).
template <int CAP>
struct EnvSmem {
  __align__(16) unsigned long long keys[CAP];  // read two at a time by the ranking
  int row[NMAX];
  int tcnt[MAXT];
};

template <typename CT, typename OT>
struct EnvIO {
  OT* em;
  OT* em_deriv;  // may be null
  OT* rij;       // may be null
  int* nlist;
  const CT* coord;
  const int* type;
  GridView g;
  const int* ilist;
  const int* numneigh;
  int* const* firstneigh;
  const OT* avg;
  const OT* std_;
  int nloc, nall;
  float rcut, rcut_smth;
  int* status;
};

// One center atom. With `defer`, an atom with more in-range candidates than
// CAP writes nothing and returns false (the caller queues it for the
// large-buffer pass); otherwise the overflow is reported in the status word.
template <typename CT, typename OT, int CAP, bool FROM_CELLS>
__device__ bool env_one(const EnvIO<CT, OT>& io, const SecInfo& sec, int row,
                        EnvSmem<CAP>& sm, bool defer) {
  const int lane = threadIdx.x & 31;
  int f, i;
  if (FROM_CELLS) {
    f = 0;
    i = row;
  } else {
    f = row / io.nloc;
    i = io.ilist[row];
  }
  const CT* fc = io.coord + (size_t)f * io.nall * 3;
  const int* ft = io.type + (size_t)f * io.nall;
  const int nnei = sec.nnei, ntypes = sec.ntypes;
  int ti = ft[i];
  if (ti >= ntypes) {  // no avg/std row exists for this center type
    atomicOr(io.status, ST_TYPE_RANGE);
    ti = -1;
  }
  const CT xi[3] = {fc[3 * i], fc[3 * i + 1], fc[3 * i + 2]};
  const float fxi[3] = {(float)xi[0], (float)xi[1], (float)xi[2]};
  const float rc2f = io.rcut * io.rcut;
  const CT rc2 = (CT)rc2f;
  unsigned long long* keys = sm.keys;
  int* srow = sm.row;
  int* tcnt = sm.tcnt;
  for (int t = lane; t < MAXT; t += 32) tcnt[t] = 0;
  for (int jj = lane; jj < nnei; jj += 32) srow[jj] = -1;
  __syncwarp();

  // ---- gather in-range candidates into shared keys
  int count = 0;
  auto push = [&](bool ok, unsigned long long key) {
    unsigned b = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      int pos = count + __popc(b & lanemask_lt());
      if (pos < CAP) {
        keys[pos] = key;
        atomicAdd(&tcnt[key >> 56], 1);
      }
    }
    count += __popc(b);
  };
  if (FROM_CELLS) {
    // the 27 neighbor cells' atom ranges loaded at once (lane L < 27: cell
    // (dx, dy, dz) = (L / 9, L / 3 % 3, L % 3) - 1), then one flat candidate
    // list walked in full batches of 32: with the grid's cell-ordered
    // records when the fused geometry pass wrote them, else through the
    // atom indices (the next batch's requested before the current batch is
    // tested)
    const GridHeader& h = *io.g.h;
    const int ci = io.g.cell_of[i];
    const int cz = ci % h.dims[2], cy = (ci / h.dims[2]) % h.dims[1],
              cx = ci / (h.dims[2] * h.dims[1]);
    int cb = 0, cn = 0;
    if (lane < 27) {
      const int x = cx + lane / 9 - 1, y = cy + (lane / 3) % 3 - 1, z = cz + lane % 3 - 1;
      if (x >= 0 && x < h.dims[0] && y >= 0 && y < h.dims[1] && z >= 0 && z < h.dims[2]) {
        const int c = (x * h.dims[1] + y) * h.dims[2] + z;
        cb = io.g.cell_start[c];
        cn = io.g.cell_start[c + 1] - cb;
      }
    }
    int incl = cn;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - cn;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    // position in the cell-ordered arrays of flat candidate fl (-1 past
    // the end): the cell is the last lane whose range starts at or before fl
    // (binary search over the lanes)
    auto slot_of = [&](int fl) -> int {
      int lo = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const int ev = __shfl_sync(0xffffffffu, excl, lo + st);
        if (ev <= fl) lo += st;
      }
      const int base_c = __shfl_sync(0xffffffffu, cb, lo);
      const int start_c = __shfl_sync(0xffffffffu, excl, lo);
      return fl < total ? base_c + (fl - start_c) : -1;
    };
    bool walked = false;
    if constexpr (sizeof(CT) == 8) {
      if (h.packed != 0) {
        // the grid's cell-ordered records (fused geometry pass): contiguous
        // 32-byte reads per batch
        for (int base = 0; base < total; base += 32) {
          const int k = slot_of(base + lane);
          unsigned long long key = 0;
          bool ok = false;
          if (k >= 0)
            ok = accept_packed(key, io.g.cell_pos + k, i, ti, xi, fxi, rc2, rc2f, ntypes,
                               io.status);
          push(ok, key);
        }
        walked = true;
      }
    }
    if (!walked) {
      auto cand_of = [&](int fl) -> int {
        const int k = slot_of(fl);
        return k >= 0 ? io.g.cell_atoms[k] : -1;
      };
      int jn = cand_of(lane);
      for (int base = 0; base < total; base += 32) {
        const int j = jn;
        jn = cand_of(base + 32 + lane);
        unsigned long long key = 0;
        bool ok = false;
        if (j >= 0)
          ok = accept<CT, true>(key, j, i, ti, fc, ft, xi, fxi, rc2, rc2f, ntypes, io.status);
        push(ok, key);
      }
    }
  } else {
    const int nn = io.numneigh[row];
    const int* cand = io.firstneigh[row];
    int jn = lane < nn ? cand[lane] : -1;  // the next batch's candidate, requested early
    for (int base = 0; base < nn; base += 32) {
      const int k = base + lane;
      const int j = jn;
      jn = k + 32 < nn ? cand[k + 32] : -1;
      unsigned long long key = 0;
      bool ok = false;
      if (k < nn)
        ok = accept<CT, false>(key, j, i, ti, fc, ft, xi, fxi, rc2, rc2f, ntypes, io.status);
      push(ok, key);
    }
  }
  __syncwarp();
  if (count > CAP) {
    if (defer) return false;
    if (lane == 0) atomicOr(io.status, ST_NLIST_CAPACITY);
  }
  const int n = count < CAP ? count : CAP;

  // ---- per-type start offsets (exclusive prefix over types, lane t holds t)
  int tstart = lane < ntypes ? tcnt[lane] : 0;
  {
    int x = tstart;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    tstart = x - tstart;
  }
  // ---- rank every key (keys are unique: they contain the index)
  for (int q = 0; q * 32 < n; ++q) {
    int kk = q * 32 + lane;
    unsigned long long own = kk < n ? keys[kk] : ~0ull;
    int r = 0;
    // two keys per 16-byte shared-memory load (broadcast to the warp)
    const ulonglong2* k2 = reinterpret_cast<const ulonglong2*>(keys);
    int p = 0;
    for (; 2 * p + 1 < n; ++p) {
      const ulonglong2 v = k2[p];
      r += (v.x < own ? 1 : 0) + (v.y < own ? 1 : 0);
    }
    if (2 * p < n) r += keys[2 * p] < own ? 1 : 0;
    int t = (int)(own >> 56) & 31;
    int ts = __shfl_sync(0xffffffffu, tstart, t);
    if (kk < n) {
      int rr = r - ts;
      int selt = sec.sec[t + 1] - sec.sec[t];
      if (rr < selt) srow[sec.sec[t] + rr] = (int)(own & 0xFFFFFFull);
      else atomicOr(io.status, ST_SEL_OVERFLOW);
    }
  }
  __syncwarp();

  // ---- environment matrix, one slot per lane
  const size_t orow = (size_t)f * io.nloc + i;
  const float rmin = io.rcut_smth, rmax = io.rcut;
  const OT* av = io.avg + (size_t)(ti < 0 ? 0 : ti) * nnei * 4;
  const OT* sd = io.std_ + (size_t)(ti < 0 ? 0 : ti) * nnei * 4;
  const bool want_d = io.em_deriv != nullptr;
  for (int jj = lane; jj < nnei; jj += 32) {
    const int j = srow[jj];
    io.nlist[orow * nnei + jj] = j;
    OT r[3] = {(OT)0., (OT)0., (OT)0.};
    OT v[4] = {(OT)0., (OT)0., (OT)0., (OT)0.};
    OT gd[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) gd[k] = (OT)0.;
    if (j >= 0) {
      for (int d = 0; d < 3; ++d) r[d] = (OT)(fc[3 * j + d] - xi[d]);
      env_row<OT>(r, rmin, rmax, v, want_d ? gd : nullptr);
    }
    OT* e = io.em + (orow * nnei + jj) * 4;
    store_env_row(e, av + jj * 4, sd + jj * 4, v, ti >= 0);
    if (want_d) {
      OT* ed = io.em_deriv + (orow * nnei + jj) * 12;
#pragma unroll
      for (int k = 0; k < 12; ++k) ed[k] = ti >= 0 ? gd[k] / sd[jj * 4 + k / 3] : (OT)0.;
    }
    if (io.rij) {
      OT* rr = io.rij + (orow * nnei + jj) * 3;
      rr[0] = r[0];
      rr[1] = r[1];
      rr[2] = r[2];
    }
  }
  return true;
}

template <typename CT, typename OT, int CAP, int WARPS, bool FROM_CELLS>
__global__ void __launch_bounds__(WARPS * 32, (CAP <= 256 && sizeof(OT) == 4) ? 32 / WARPS : 1)
k_env(EnvIO<CT, OT> io, SecInfo sec, int nrows, int* redo) {
  __shared__ EnvSmem<CAP> sm[WARPS];
  pdl_wait();
  pdl_trigger();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WARPS + w;
  if (row >= nrows) return;
  const bool ok = env_one<CT, OT, CAP, FROM_CELLS>(io, sec, row, sm[w], redo != nullptr);
  if (!ok && lane == 0) {
    int p = atomicAdd(&redo[0], 1);
    redo[1 + p] = row;
  }
}

// Atoms deferred by k_env: one warp each with the large key buffer. Launched
// unconditionally with a fixed grid; it reads the queue length on the device.
template <typename CT, typename OT, int CAP>
__global__ void __launch_bounds__(32) k_env_redo(EnvIO<CT, OT> io, SecInfo sec,
                                                 const int* redo) {
  __shared__ EnvSmem<CAP> sm;
  pdl_wait();
  pdl_trigger();
  const int n = redo[0];
  for (int r = blockIdx.x; r < n; r += gridDim.x) {
    env_one<CT, OT, CAP, true>(io, sec, redo[1 + r], sm, false);
    __syncwarp();
  }
}

constexpr int ENV_SMALL_CAP = 256;
constexpr int ENV_LARGE_CAP = 4096;

template <typename CT, typename OT>
static int env_cells(OT* em, OT* em_deriv, OT* rij, int* nlist, const CT* coord,
                     const int* type, const void* grid, const OT* avg,
                     const OT* std_, int nloc, int nall, float rcut,
                     float rcut_smth, const int* sec, int nsec, int* status,
                     dpb_stream_t stream) {
  SecInfo s;
  int rc = make_sec(s, sec, nsec);
  if (rc) return rc;
  if (nloc <= 0) return DPB_OK;
  if (grid == nullptr || status == nullptr) {
    set_error("env_mat_a_cells: grid and status are required");
    return DPB_ERR_INVALID;
  }
  if ((em_deriv == nullptr) != (rij == nullptr)) {
    set_error("env_mat_a_cells: em_deriv and rij are either both given or both null");
    return DPB_ERR_INVALID;
  }
  GridView g = carve_grid(const_cast<void*>(grid), nall);
  EnvIO<CT, OT> io{em, em_deriv, rij, nlist, coord, type, g, nullptr, nullptr, nullptr,
                   avg, std_, nloc, nall, rcut, rcut_smth, status};
  cudaStream_t st = as_stream(stream);
  DPB_CUDA(cudaMemsetAsync(g.redo, 0, sizeof(int), st), "env_mat_a_cells");
  constexpr int W = 4;
  DPB_CUDA(launch_pdl(k_env<CT, OT, ENV_SMALL_CAP, W, true>, dim3(ceil_div(nloc, W)),
                      dim3(W * 32), 0, st, io, s, nloc, g.redo),
           "env_mat_a_cells");
  DPB_CUDA(launch_pdl(k_env_redo<CT, OT, ENV_LARGE_CAP>, dim3(64), dim3(32), 0, st, io, s,
                      (const int*)g.redo),
           "env_mat_a_cells/large");
  return DPB_OK;
}

template <typename CT, typename OT = CT>
static int env_inlist(OT* em, OT* em_deriv, OT* rij, int* nlist, const CT* coord,
                      const int* type, int inum, const int* ilist,
                      const int* numneigh, int* const* firstneigh,
                      int max_nbor_size, const OT* avg, const OT* std_, int nloc,
                      int nall, int nframes, float rcut, float rcut_smth,
                      const int* sec, int nsec, int* status,
                      dpb_stream_t stream) {
  SecInfo s;
  int rc = make_sec(s, sec, nsec);
  if (rc) return rc;
  if (inum != nframes * nloc) {
    set_error("prod_env_mat_a: inum (%d) != nframes * nloc (%d)", inum, nframes * nloc);
    return DPB_ERR_INVALID;
  }
  if (status == nullptr) {
    set_error("prod_env_mat_a: a device status word is required");
    return DPB_ERR_INVALID;
  }
  if (inum <= 0) return DPB_OK;
  if (max_nbor_size > ENV_LARGE_CAP) {
    set_error("prod_env_mat_a: max_nbor_size %d exceeds 4096 (GPU_MAX_NBOR_SIZE)",
              max_nbor_size);
    return DPB_ERR_NLIST_CAPACITY;
  }
  cudaStream_t st = as_stream(stream);
  GridView g{};
  EnvIO<CT, OT> io{em, em_deriv, rij, nlist, coord, type, g, ilist, numneigh, firstneigh,
                   avg, std_, nloc, nall, rcut, rcut_smth, status};
  if (max_nbor_size <= 1024) {
    constexpr int W = 4;
    k_env<CT, OT, 1024, W, false><<<ceil_div(inum, W), W * 32, 0, st>>>(io, s, inum, nullptr);
  } else {
    k_env<CT, OT, ENV_LARGE_CAP, 1, false><<<inum, 32, 0, st>>>(io, s, inum, nullptr);
  }
  DPB_CHECK_LAUNCH("prod_env_mat_a");
  return DPB_OK;
}

// ------------------------------------------------------------ build_nlist --

constexpr int NL_CAP = 2048;

template <typename T>
__global__ void __launch_bounds__(128)
k_build_nlist(int* ilist, int* numneigh, int** firstneigh, int* max_size,
              const T* c, const int* type, GridView g, int nloc, int mem_size,
              int row0, float rcut, int* status) {
  // build_nlist_cpu semantics (neighbor_list.cc:875-928): j != i, both types
  // >= 0 when type is given, strict |c_i - c_j|^2 < (T)(rcut*rcut), rows in
  // ascending j.
  __shared__ int s_c[4][NL_CAP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 4 + w;
  if (i >= nloc) return;
  int* cand = s_c[w];
  const T rc2 = (T)(rcut * rcut);
  const T xi[3] = {c[3 * i], c[3 * i + 1], c[3 * i + 2]};
  const bool ti_ok = type == nullptr || type[i] >= 0;
  const GridHeader& h = *g.h;
  const int ci = g.cell_of[i];
  const int cz = ci % h.dims[2], cy = (ci / h.dims[2]) % h.dims[1],
            cx = ci / (h.dims[2] * h.dims[1]);
  int count = 0;
  for (int dx = -1; dx <= 1; ++dx) {
    int x = cx + dx;
    if (x < 0 || x >= h.dims[0]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      int y = cy + dy;
      if (y < 0 || y >= h.dims[1]) continue;
      for (int dz = -1; dz <= 1; ++dz) {
        int z = cz + dz;
        if (z < 0 || z >= h.dims[2]) continue;
        int cc = (x * h.dims[1] + y) * h.dims[2] + z;
        int b = g.cell_start[cc], e = g.cell_start[cc + 1];
        for (int base = b; base < e; base += 32) {
          int k = base + lane;
          bool ok = false;
          int j = -1;
          if (k < e && ti_ok) {
            j = g.cell_atoms[k];
            if (j != i && (type == nullptr || type[j] >= 0)) {
              T d0 = sub_rn(xi[0], c[3 * j + 0]);
              T d1 = sub_rn(xi[1], c[3 * j + 1]);
              T d2 = sub_rn(xi[2], c[3 * j + 2]);
              ok = dot3_rn(d0, d1, d2) < rc2;
            }
          }
          unsigned bm = __ballot_sync(0xffffffffu, ok);
          if (ok) {
            int pos = count + __popc(bm & lanemask_lt());
            if (pos < NL_CAP) cand[pos] = j;
          }
          count += __popc(bm);
        }
      }
    }
  }
  __syncwarp();
  const int row = row0 + i;
  if (lane == 0) {
    ilist[row] = i;
    numneigh[row] = count < mem_size ? count : mem_size;
    atomicMax(max_size, count);
  }
  if (count > mem_size) atomicOr(status, ST_ROW_CAPACITY);
  if (count > NL_CAP) atomicOr(status, ST_NLIST_CAPACITY);
  const int n = count < NL_CAP ? count : NL_CAP;
  int* out = firstneigh[row];
  for (int q = 0; q * 32 < n; ++q) {
    int kk = q * 32 + lane;
    int own = kk < n ? cand[kk] : 0x7fffffff;
    int r = 0;
    for (int p = 0; p < n; ++p) r += cand[p] < own ? 1 : 0;
    if (kk < n && r < mem_size) out[r] = own;
  }
}

template <typename T>
int build_nlist(int* ilist, int* numneigh, int** firstneigh,
                       int* max_list_size, void* scratch,
                       long long scratch_bytes, const T* c_cpy, int nloc,
                       int nall, int mem_size, float rcut, int nframes,
                       const int* type, cudaStream_t st) {
  if (nloc < 0 || nall < nloc || mem_size < 0 || nframes < 1 || !(rcut > 0.f)) {
    set_error("build_nlist: invalid sizes (nloc=%d nall=%d mem_size=%d nframes=%d)",
              nloc, nall, mem_size, nframes);
    return DPB_ERR_INVALID;
  }
  long long need = grid_bytes(nall) + 256;
  if (scratch == nullptr || scratch_bytes < need) {
    set_error("build_nlist: scratch too small (%lld < %lld bytes)", scratch_bytes, need);
    return DPB_ERR_INVALID;
  }
  int* dev_words = (int*)scratch;  // [0] status, [1] max size
  void* grid = (char*)scratch + 256;
  DPB_CUDA(cudaMemsetAsync(dev_words, 0, 2 * sizeof(int), st), "build_nlist");
  for (int f = 0; f < nframes; ++f) {
    const T* cf = c_cpy + (size_t)f * nall * 3;
    const int* tf = type ? type + (size_t)f * nall : nullptr;
    int rc = grid_build<T>(grid, scratch_bytes - 256, cf, nall, nullptr, rcut, st);
    if (rc) return rc;
    if (nloc > 0) {
      GridView g = carve_grid(grid, nall);
      k_build_nlist<T><<<ceil_div(nloc, 4), 128, 0, st>>>(
          ilist, numneigh, firstneigh, dev_words + 1, cf, tf, g, nloc, mem_size,
          f * nloc, rcut, dev_words);
      DPB_CHECK_LAUNCH("build_nlist");
    }
  }
  int h[2] = {0, 0};
  DPB_CUDA(cudaMemcpyAsync(h, dev_words, 2 * sizeof(int), cudaMemcpyDeviceToHost, st),
           "build_nlist");
  DPB_CUDA(cudaStreamSynchronize(st), "build_nlist");
  *max_list_size = h[1];
  if (h[0] & (ST_ROW_CAPACITY | ST_NLIST_CAPACITY)) {
    set_error("build_nlist: a row holds %d neighbors, more than mem_size=%d", h[1], mem_size);
    return DPB_ERR_CAPACITY;
  }
  return DPB_OK;
}

template int build_nlist<double>(int*, int*, int**, int*, void*, long long, const double*, int,
                                 int, int, float, int, const int*, cudaStream_t);
template int build_nlist<float>(int*, int*, int**, int*, void*, long long, const float*, int,
                                int, int, float, int, const int*, cudaStream_t);

}  // namespace dpb

using namespace dpb;
extern "C" {

long long dpb_build_nlist_scratch_bytes(int nloc, int nall) {
  (void)nloc;
  return grid_bytes(nall) + 256;
}

int dpb_build_nlist_f64(int* ilist, int* numneigh, int** firstneigh,
                        int* max_list_size, void* scratch,
                        long long scratch_bytes, const double* c_cpy, int nloc,
                        int nall, int mem_size, float rcut, int nframes,
                        const int* type, dpb_stream_t stream) {
  return build_nlist<double>(ilist, numneigh, firstneigh, max_list_size, scratch,
                             scratch_bytes, c_cpy, nloc, nall, mem_size, rcut,
                             nframes, type, as_stream(stream));
}

int dpb_build_nlist_f32(int* ilist, int* numneigh, int** firstneigh,
                        int* max_list_size, void* scratch,
                        long long scratch_bytes, const float* c_cpy, int nloc,
                        int nall, int mem_size, float rcut, int nframes,
                        const int* type, dpb_stream_t stream) {
  return build_nlist<float>(ilist, numneigh, firstneigh, max_list_size, scratch,
                            scratch_bytes, c_cpy, nloc, nall, mem_size, rcut,
                            nframes, type, as_stream(stream));
}

int dpb_prod_env_mat_a_f64(double* em, double* em_deriv, double* rij,
                           int* nlist, const double* coord, const int* type,
                           int inum, const int* ilist, const int* numneigh,
                           int* const* firstneigh, int max_nbor_size,
                           const double* avg, const double* std_, int nloc,
                           int nall, int nframes, float rcut, float rcut_smth,
                           const int* sec, int nsec, int* status,
                           dpb_stream_t stream) {
  return env_inlist<double>(em, em_deriv, rij, nlist, coord, type, inum, ilist,
                            numneigh, firstneigh, max_nbor_size, avg, std_,
                            nloc, nall, nframes, rcut, rcut_smth, sec, nsec,
                            status, stream);
}

int dpb_prod_env_mat_a_f32(float* em, float* em_deriv, float* rij, int* nlist,
                           const float* coord, const int* type, int inum,
                           const int* ilist, const int* numneigh,
                           int* const* firstneigh, int max_nbor_size,
                           const float* avg, const float* std_, int nloc,
                           int nall, int nframes, float rcut, float rcut_smth,
                           const int* sec, int nsec, int* status,
                           dpb_stream_t stream) {
  return env_inlist<float>(em, em_deriv, rij, nlist, coord, type, inum, ilist,
                           numneigh, firstneigh, max_nbor_size, avg, std_,
                           nloc, nall, nframes, rcut, rcut_smth, sec, nsec,
                           status, stream);
}

int dpb_prod_env_mat_a_mixed(float* em, float* em_deriv, float* rij, int* nlist,
                             const double* coord, const int* type, int inum,
                             const int* ilist, const int* numneigh,
                             int* const* firstneigh, int max_nbor_size,
                             const float* avg, const float* std_, int nloc, int nall,
                             int nframes, float rcut, float rcut_smth, const int* sec,
                             int nsec, int* status, dpb_stream_t stream) {
  return env_inlist<double, float>(em, em_deriv, rij, nlist, coord, type, inum, ilist,
                                   numneigh, firstneigh, max_nbor_size, avg, std_, nloc,
                                   nall, nframes, rcut, rcut_smth, sec, nsec, status,
                                   stream);
}

int dpb_env_mat_a_cells_f64(double* em, double* em_deriv, double* rij,
                            int* nlist, const double* coord, const int* type,
                            const void* grid, const double* avg,
                            const double* std_, int nloc, int nall, float rcut,
                            float rcut_smth, const int* sec, int nsec,
                            int* status, dpb_stream_t stream) {
  return env_cells<double, double>(em, em_deriv, rij, nlist, coord, type, grid,
                                   avg, std_, nloc, nall, rcut, rcut_smth, sec,
                                   nsec, status, stream);
}

int dpb_env_mat_a_cells_f32(float* em, float* em_deriv, float* rij, int* nlist,
                            const float* coord, const int* type,
                            const void* grid, const float* avg,
                            const float* std_, int nloc, int nall, float rcut,
                            float rcut_smth, const int* sec, int nsec,
                            int* status, dpb_stream_t stream) {
  return env_cells<float, float>(em, em_deriv, rij, nlist, coord, type, grid,
                                 avg, std_, nloc, nall, rcut, rcut_smth, sec,
                                 nsec, status, stream);
}

int dpb_env_mat_a_cells_mixed(float* em, float* em_deriv, float* rij,
                              int* nlist, const double* coord, const int* type,
                              const void* grid, const float* avg,
                              const float* std_, int nloc, int nall,
                              float rcut, float rcut_smth, const int* sec,
                              int nsec, int* status, dpb_stream_t stream) {
  return env_cells<double, float>(em, em_deriv, rij, nlist, coord, type, grid,
                                  avg, std_, nloc, nall, rcut, rcut_smth, sec,
                                  nsec, status, stream);
}

}  // extern "C"
