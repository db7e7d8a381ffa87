// Coordinates: wrap into the box, periodic ghost images, and the cell grid
// used by the neighbor search.
//
// copy_coord reproduces copy_coord_cpu (source/lib/src/coord.cc:29-64 ->
// source/lib/src/neighbor_list.cc:43-148,730-849) element for element: local
// atoms first, then for every ghost cell of the extended grid (x outer, z
// inner, local cells skipped) the atoms of its periodic source cell in
// ascending index, shifted by the box. The reference's own GPU version
// (source/lib/src/gpu/coord.cu:352-414) emits a different ghost order; this
// one matches the CPU path so that neighbor indices compare bit for bit.
#include <math.h>
#include <atomic>

#include "dpb_common.cuh"
#include "dpb_internal.cuh"

namespace dpb {

// --------------------------------------------------------------- region ----

void host_region(HostRegion& r, const double* b, float rcut) {
  // |det| and cofactor inverse (source/lib/include/SimulationRegion_Impl.h:
  // 429-480); distances between opposite faces (:364-372); cell counts
  // (source/lib/src/neighbor_list.cc:747-772).
  double vol = b[0] * (b[4] * b[8] - b[7] * b[5]) -
               b[1] * (b[3] * b[8] - b[6] * b[5]) +
               b[2] * (b[3] * b[7] - b[6] * b[4]);
  vol = fabs(vol);
  double vi = 1. / vol;
  double* rc = r.rec;
  rc[0] = (b[4] * b[8] - b[7] * b[5]) * vi;
  rc[4] = (b[0] * b[8] - b[6] * b[2]) * vi;
  rc[8] = (b[0] * b[4] - b[3] * b[1]) * vi;
  rc[1] = (-b[3] * b[8] + b[6] * b[5]) * vi;
  rc[2] = (b[3] * b[7] - b[6] * b[4]) * vi;
  rc[3] = (-b[1] * b[8] + b[7] * b[2]) * vi;
  rc[5] = (-b[0] * b[7] + b[6] * b[1]) * vi;
  rc[6] = (b[1] * b[5] - b[4] * b[2]) * vi;
  rc[7] = (-b[0] * b[5] + b[3] * b[2]) * vi;
  for (int k = 0; k < 9; ++k) r.box[k] = b[k];
  auto face = [&](const double* u, const double* v) {
    double t0 = u[1] * v[2] - u[2] * v[1];
    double t1 = u[2] * v[0] - u[0] * v[2];
    double t2 = u[0] * v[1] - u[1] * v[0];
    return vol * (1. / sqrt(t0 * t0 + t1 * t1 + t2 * t2));
  };
  double tf[3] = {face(b + 3, b + 6), face(b + 6, b + 0), face(b + 0, b + 3)};
  double rcd = (double)rcut;
  r.nloc_cells = 1;
  r.next_cells = 1;
  for (int d = 0; d < 3; ++d) {
    int n = (int)(tf[d] / rcd);
    if (n == 0) n = 1;
    double cs = tf[d] / n;
    r.nc[d] = n;
    r.ng[d] = (int)(rcd / cs) + 1;
    r.inv_nc[d] = 1. / n;
    r.nloc_cells *= n;
    r.next_cells *= n + 2 * r.ng[d];
  }
  r.volume = vol;
}

__device__ __forceinline__ void dev_t_dot_v(double* o, const double* t,
                                            const double* v) {
  // o = t . v, left-to-right, no fusion (SimulationRegion_Impl.h:388-396)
  o[0] = add_rn(add_rn(mul_rn(v[0], t[0]), mul_rn(v[1], t[1])), mul_rn(v[2], t[2]));
  o[1] = add_rn(add_rn(mul_rn(v[0], t[3]), mul_rn(v[1], t[4])), mul_rn(v[2], t[5]));
  o[2] = add_rn(add_rn(mul_rn(v[0], t[6]), mul_rn(v[1], t[7])), mul_rn(v[2], t[8]));
}
__device__ __forceinline__ void dev_tt_dot_v(double* o, const double* t,
                                             const double* v) {
  // o = t^T . v (SimulationRegion_Impl.h:399-407)
  o[0] = add_rn(add_rn(mul_rn(v[0], t[0]), mul_rn(v[1], t[3])), mul_rn(v[2], t[6]));
  o[1] = add_rn(add_rn(mul_rn(v[0], t[1]), mul_rn(v[1], t[4])), mul_rn(v[2], t[7]));
  o[2] = add_rn(add_rn(mul_rn(v[0], t[2]), mul_rn(v[1], t[5])), mul_rn(v[2], t[8]));
}

// ------------------------------------------------------------ normalize ----

// source/lib/src/coord.cc:14-27: inter = rec.p, fmod(.,1), +1 if < 0, back
// to physical. Region arithmetic runs in T like the reference.
template <typename T>
__device__ __forceinline__ void normalize_point(T* q, const T* p, const HostRegion& r) {
  T ri[3];
  for (int d = 0; d < 3; ++d) {
    ri[d] = add_rn(add_rn(mul_rn(p[0], (T)r.rec[3 * d]), mul_rn(p[1], (T)r.rec[3 * d + 1])),
                   mul_rn(p[2], (T)r.rec[3 * d + 2]));
    ri[d] = fmod(ri[d], (T)1.);
    if (ri[d] < (T)0.) ri[d] = add_rn(ri[d], (T)1.);
  }
  for (int d = 0; d < 3; ++d) {
    q[d] = add_rn(add_rn(mul_rn(ri[0], (T)r.box[d]), mul_rn(ri[1], (T)r.box[3 + d])),
                  mul_rn(ri[2], (T)r.box[6 + d]));
  }
}

template <typename T>
__global__ void k_normalize(T* coord, int natom, HostRegion r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= natom) return;
  T p[3] = {coord[3 * i], coord[3 * i + 1], coord[3 * i + 2]};
  T q[3];
  normalize_point(q, p, r);
  for (int d = 0; d < 3; ++d) coord[3 * i + d] = q[d];
}

// ------------------------------------------------------------ copy_coord ---

struct CopyScratch {
  int* cell_of;   // [nloc]
  int* cnt;       // [nloc_cells + 1] counts, then starts
  int* fill;      // [nloc_cells]
  int* order;     // [nloc]
  int* ext_off;   // [next_cells + 1]
  int* nall;      // [1]
};

static long long copy_scratch_ints(int nloc, const HostRegion& r) {
  return (long long)nloc * 2 + (r.nloc_cells + 1) + r.nloc_cells +
         (r.next_cells + 1) + 1 + 64;
}

static CopyScratch carve_copy(void* p, int nloc, const HostRegion& r) {
  int* q = (int*)p;
  CopyScratch s;
  s.cell_of = q; q += nloc;
  s.cnt = q; q += r.nloc_cells + 1;
  s.fill = q; q += r.nloc_cells;
  s.order = q; q += nloc;
  s.ext_off = q; q += r.next_cells + 1;
  s.nall = q;
  return s;
}

// Cell of a local atom as build_clist computes it
// (source/lib/src/neighbor_list.cc:84-111, nat_stt = 0, nat_end = ncell).
__device__ __forceinline__ int copy_cell_of(const double* p, const HostRegion& r) {
  double inter[3];
  dev_t_dot_v(inter, r.rec, p);
  int idx[3];
  for (int d = 0; d < 3; ++d) {
    double csz = r.inv_nc[d];
    idx[d] = (int)(__ddiv_rn(inter[d] - 0., csz));
    if (inter[d] - 0. < 0.) idx[d]--;
    if (idx[d] < 0) idx[d] = 0;
    else if (idx[d] >= r.nc[d]) idx[d] = r.nc[d] - 1;
  }
  return (idx[0] * r.nc[1] + idx[1]) * r.nc[2] + idx[2];
}

template <typename T>
__global__ void k_cc_cell(CopyScratch s, T* out_c, int* out_t, int* mapping,
                          const T* in_c, const int* in_t, int nloc,
                          int mem_nall, HostRegion r) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  double p[3] = {(double)in_c[3 * i], (double)in_c[3 * i + 1], (double)in_c[3 * i + 2]};
  int c = copy_cell_of(p, r);
  s.cell_of[i] = c;
  atomicAdd(&s.cnt[c], 1);
  if (i < mem_nall) {
    out_c[3 * i] = in_c[3 * i];
    out_c[3 * i + 1] = in_c[3 * i + 1];
    out_c[3 * i + 2] = in_c[3 * i + 2];
    out_t[i] = in_t[i];
    mapping[i] = i;
  }
}

// Exclusive scan of n ints in place by one block (n may be large: chunked).
__device__ void block_exclusive_scan(int* a, int n, int* total) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (int base = 0; base < n; base += blockDim.x) {
    int k = base + threadIdx.x;
    int v = k < n ? a[k] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;  // inclusive
    }
    __syncthreads();
    int prefix = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + x - v;
    if (k < n) a[k] = prefix;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = prefix + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__device__ __forceinline__ int pbc_shift(int idx, int n) {
  // source/lib/src/neighbor_list.cc:730-745
  int s = 0;
  if (idx < 0) {
    s = 1;
    while (idx + s * n < 0) s++;
  } else if (idx >= n) {
    s = -1;
    while (idx + s * n >= n) s--;
  }
  return s;
}

__device__ __forceinline__ void ext_cell_coords(int e, const HostRegion& r,
                                                int* ii) {
  int E1 = r.nc[1] + 2 * r.ng[1], E2 = r.nc[2] + 2 * r.ng[2];
  ii[2] = e % E2 - r.ng[2];
  int t = e / E2;
  ii[1] = t % E1 - r.ng[1];
  ii[0] = t / E1 - r.ng[0];
}

__global__ void k_cc_scan(CopyScratch s, int nloc, HostRegion r) {
  // starts of the local cells, then ghost offsets in the reference's ghost
  // loop order (source/lib/src/neighbor_list.cc:799-826)
  __shared__ int tot;
  block_exclusive_scan(s.cnt, r.nloc_cells + 1, &tot);
  __syncthreads();
  for (int e = threadIdx.x; e <= r.next_cells; e += blockDim.x) {
    if (e == r.next_cells) {
      s.ext_off[e] = 0;
      continue;
    }
    int ii[3];
    ext_cell_coords(e, r, ii);
    bool local = ii[0] >= 0 && ii[0] < r.nc[0] && ii[1] >= 0 &&
                 ii[1] < r.nc[1] && ii[2] >= 0 && ii[2] < r.nc[2];
    int v = 0;
    if (!local) {
      int jj[3];
      for (int d = 0; d < 3; ++d) jj[d] = ii[d] + pbc_shift(ii[d], r.nc[d]) * r.nc[d];
      int c = (jj[0] * r.nc[1] + jj[1]) * r.nc[2] + jj[2];
      v = s.cnt[c + 1] - s.cnt[c];
    }
    s.ext_off[e] = v;
  }
  __syncthreads();
  block_exclusive_scan(s.ext_off, r.next_cells + 1, &tot);
  __syncthreads();
  if (threadIdx.x == 0) *s.nall = nloc + s.ext_off[r.next_cells];
}

__global__ void k_cc_fill(CopyScratch s, int nloc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nloc) return;
  int c = s.cell_of[i];
  int pos = s.cnt[c] + atomicAdd(&s.fill[c], 1);
  s.order[pos] = i;
}

constexpr int SORT_CAP = 256;

__global__ void k_cc_sort(CopyScratch s, int ncells) {
  // ascending atom index within each cell (build_clist pushes in index
  // order): one warp per cell ranks the cell's entries in shared memory;
  // cells larger than SORT_CAP (none at cell edges near rcut) fall back to a
  // serial insertion sort by lane 0.
  __shared__ int buf[4][SORT_CAP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 4 + w;
  if (c >= ncells) return;
  const int b = s.cnt[c], e = s.cnt[c + 1], n = e - b;
  if (n <= 1) return;
  if (n <= SORT_CAP) {
    int* v = buf[w];
    for (int k = lane; k < n; k += 32) v[k] = s.order[b + k];
    __syncwarp();
    for (int k = lane; k < n; k += 32) {
      const int x = v[k];
      int r = 0;
      for (int q = 0; q < n; ++q) r += v[q] < x ? 1 : 0;
      s.order[b + r] = x;  // indices are distinct: ranks are a permutation
    }
    return;
  }
  if (lane == 0) {
    for (int a = b + 1; a < e; ++a) {
      int v = s.order[a], q = a - 1;
      while (q >= b && s.order[q] > v) {
        s.order[q + 1] = s.order[q];
        q--;
      }
      s.order[q + 1] = v;
    }
  }
}

template <typename T>
__global__ void k_cc_copy(CopyScratch s, T* out_c, int* out_t, int* mapping,
                          const T* in_c, const int* in_t, int nloc,
                          int mem_nall, HostRegion r) {
  // one warp per extended cell: ghost = source atom - box shift
  // (source/lib/src/neighbor_list.cc:815-831)
  int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (e >= r.next_cells) return;
  int ii[3];
  ext_cell_coords(e, r, ii);
  if (ii[0] >= 0 && ii[0] < r.nc[0] && ii[1] >= 0 && ii[1] < r.nc[1] &&
      ii[2] >= 0 && ii[2] < r.nc[2])
    return;
  int jj[3];
  double ps[3];
  for (int d = 0; d < 3; ++d) {
    int sh = pbc_shift(ii[d], r.nc[d]);
    ps[d] = (double)sh;
    jj[d] = ii[d] + sh * r.nc[d];
  }
  double sv[3];
  dev_tt_dot_v(sv, r.box, ps);
  int c = (jj[0] * r.nc[1] + jj[1]) * r.nc[2] + jj[2];
  int b = s.cnt[c], n = s.cnt[c + 1] - b;
  int w0 = nloc + s.ext_off[e];
  for (int k = lane; k < n; k += 32) {
    int p = s.order[b + k];
    int w = w0 + k;
    if (w < mem_nall) {
      out_c[3 * w + 0] = (T)sub_rn((double)in_c[3 * p + 0], sv[0]);
      out_c[3 * w + 1] = (T)sub_rn((double)in_c[3 * p + 1], sv[1]);
      out_c[3 * w + 2] = (T)sub_rn((double)in_c[3 * p + 2], sv[2]);
      out_t[w] = in_t[p];
      mapping[w] = p;
    }
  }
}

// The copy on a given cell decomposition (nc local cells and ng ghost layers
// per dimension): the steps of copy_coord_cpu (coord.cc:29-64) as kernels.
template <typename T>
static int copy_coord_region_async(T* out_c, int* out_t, int* mapping, int* nall_dev,
                                   void* scratch, long long scratch_bytes, const T* in_c,
                                   const int* in_t, int nloc, int mem_nall,
                                   const HostRegion& r, cudaStream_t st) {
  if (!(r.volume > 0.)) {
    set_error("copy_coord: the box has zero volume");
    return DPB_ERR_INVALID;
  }
  long long need = copy_scratch_ints(nloc, r) * (long long)sizeof(int);
  if (scratch == nullptr || scratch_bytes < need) {
    set_error("copy_coord: scratch too small (%lld < %lld bytes)",
              scratch_bytes, need);
    return DPB_ERR_INVALID;
  }
  CopyScratch s = carve_copy(scratch, nloc, r);
  DPB_CUDA(cudaMemsetAsync(s.cnt, 0, sizeof(int) * (2 * r.nloc_cells + 1), st),
           "copy_coord");
  if (nloc > 0) {
    k_cc_cell<T><<<ceil_div(nloc, 256), 256, 0, st>>>(s, out_c, out_t, mapping, in_c,
                                                     in_t, nloc, mem_nall, r);
    DPB_CHECK_LAUNCH("copy_coord/cell");
  }
  k_cc_scan<<<1, 1024, 0, st>>>(s, nloc, r);
  DPB_CHECK_LAUNCH("copy_coord/scan");
  if (nloc > 0) {
    k_cc_fill<<<ceil_div(nloc, 256), 256, 0, st>>>(s, nloc);
    DPB_CHECK_LAUNCH("copy_coord/fill");
  }
  k_cc_sort<<<ceil_div(r.nloc_cells, 4), 128, 0, st>>>(s, r.nloc_cells);
  DPB_CHECK_LAUNCH("copy_coord/sort");
  k_cc_copy<T><<<ceil_div((long long)r.next_cells * 32, 256), 256, 0, st>>>(
      s, out_c, out_t, mapping, in_c, in_t, nloc, mem_nall, r);
  DPB_CHECK_LAUNCH("copy_coord/copy");
  if (nall_dev) {
    DPB_CUDA(cudaMemcpyAsync(nall_dev, s.nall, sizeof(int),
                             cudaMemcpyDeviceToDevice, st),
             "copy_coord");
  }
  return DPB_OK;
}

template <typename T>
int copy_coord_async(T* out_c, int* out_t, int* mapping, int* nall_dev,
                     void* scratch, long long scratch_bytes, const T* in_c,
                     const int* in_t, int nloc, int mem_nall, float rcut,
                     const double* boxt, cudaStream_t st) {
  if (nloc < 0 || mem_nall < 0 || !(rcut > 0.f)) {
    set_error("copy_coord: invalid sizes (nloc=%d mem_nall=%d rcut=%g)", nloc,
              mem_nall, (double)rcut);
    return DPB_ERR_INVALID;
  }
  HostRegion r;
  host_region(r, boxt, rcut);
  return copy_coord_region_async<T>(out_c, out_t, mapping, nall_dev, scratch, scratch_bytes,
                                    in_c, in_t, nloc, mem_nall, r, st);
}

// the copy, then nall read back (DPB_ERR_CAPACITY when it exceeds mem_nall)
template <typename T>
static int copy_coord_region_sync(T* out_c, int* out_t, int* mapping, int* nall,
                                  void* scratch, long long scratch_bytes, const T* in_c,
                                  const int* in_t, int nloc, int mem_nall,
                                  const HostRegion& r, cudaStream_t st) {
  int rc = copy_coord_region_async<T>(out_c, out_t, mapping, nullptr, scratch, scratch_bytes,
                                      in_c, in_t, nloc, mem_nall, r, st);
  if (rc != DPB_OK) return rc;
  CopyScratch s = carve_copy(scratch, nloc, r);
  int h = 0;
  DPB_CUDA(cudaMemcpyAsync(&h, s.nall, sizeof(int), cudaMemcpyDeviceToHost, st),
           "copy_coord");
  DPB_CUDA(cudaStreamSynchronize(st), "copy_coord");
  *nall = h;
  if (h > mem_nall) {
    set_error("copy_coord: nall=%d exceeds mem_nall=%d", h, mem_nall);
    return DPB_ERR_CAPACITY;
  }
  return DPB_OK;
}

template <typename T>
int copy_coord_sync(T* out_c, int* out_t, int* mapping, int* nall,
                    void* scratch, long long scratch_bytes, const T* in_c,
                    const int* in_t, int nloc, int mem_nall, float rcut,
                    const T* boxt, cudaStream_t st) {
  if (nloc < 0 || mem_nall < 0 || !(rcut > 0.f)) {
    set_error("copy_coord: invalid sizes (nloc=%d mem_nall=%d rcut=%g)", nloc,
              mem_nall, (double)rcut);
    return DPB_ERR_INVALID;
  }
  double b[9];
  for (int k = 0; k < 9; ++k) b[k] = (double)boxt[k];
  HostRegion r;
  host_region(r, b, rcut);
  return copy_coord_region_sync<T>(out_c, out_t, mapping, nall, scratch, scratch_bytes, in_c,
                                   in_t, nloc, mem_nall, r, st);
}

// A region whose cell decomposition is given in the layout of
// compute_cell_info (coord.cc:69-108: ncell at [3..5], ngcell at [12..14],
// loc_cellnum at [21], total_cellnum at [22]) instead of derived from rcut.
static int host_region_cells(HostRegion& r, const double* boxt, const int* cell_info) {
  host_region(r, boxt, 1.f);
  long long nl = 1, ne = 1;
  for (int d = 0; d < 3; ++d) {
    const int n = cell_info[3 + d], g = cell_info[12 + d];
    if (n < 1 || g < 1 || n > (1 << 20) || g > (1 << 20)) {
      set_error("copy_coord: invalid cell_info (ncell %d, ngcell %d in dimension %d)", n, g, d);
      return DPB_ERR_INVALID;
    }
    r.nc[d] = n;
    r.ng[d] = g;
    r.inv_nc[d] = 1. / n;
    nl *= n;
    ne *= n + 2LL * g;
  }
  if (nl != cell_info[21] || ne != cell_info[22] || ne > (1LL << 30)) {
    set_error("copy_coord: cell_info counts (%d local, %d total cells) disagree with its "
              "ncell / ngcell", cell_info[21], cell_info[22]);
    return DPB_ERR_INVALID;
  }
  r.nloc_cells = (int)nl;
  r.next_cells = (int)ne;
  return DPB_OK;
}

template <typename T>
static int copy_coord_cells(T* out_c, int* out_t, int* mapping, int* nall, void* scratch,
                            long long scratch_bytes, const T* in_c, const int* in_t, int nloc,
                            int mem_nall, const int* cell_info, const T* boxt,
                            cudaStream_t st) {
  if (nloc < 0 || mem_nall < 0 || cell_info == nullptr || boxt == nullptr || nall == nullptr) {
    set_error("copy_coord: invalid arguments (nloc=%d mem_nall=%d)", nloc, mem_nall);
    return DPB_ERR_INVALID;
  }
  double b[9];
  for (int k = 0; k < 9; ++k) b[k] = (double)boxt[k];
  HostRegion r;
  int rc = host_region_cells(r, b, cell_info);
  if (rc != DPB_OK) return rc;
  return copy_coord_region_sync<T>(out_c, out_t, mapping, nall, scratch, scratch_bytes, in_c,
                                   in_t, nloc, mem_nall, r, st);
}

long long copy_coord_cells_scratch_bytes(int nloc, const int* cell_info) {
  double b[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  HostRegion r;
  if (cell_info == nullptr || nloc < 0 || host_region_cells(r, b, cell_info) != DPB_OK) return -1;
  return copy_scratch_ints(nloc, r) * (long long)sizeof(int);
}

// ------------------------------------------------------------ cell grid ----

__device__ __forceinline__ unsigned long long ord_key(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
  unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)u);
}

__global__ void k_grid_init(GridHeader* h) {
  for (int d = 0; d < 3; ++d) {
    h->kmin[d] = ~0ull;
    h->kmax[d] = 0ull;
  }
  h->packed = 0;  // these builders do not write cell_pos
}

template <typename T>
__global__ void k_grid_bbox(GridHeader* h, const T* coord, int nall,
                            const int* nall_dev) {
  int n = nall_dev ? min(*nall_dev, nall) : nall;
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    for (int d = 0; d < 3; ++d) {
      unsigned long long k = ord_key((double)coord[3 * i + d]);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
    }
  }
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[d], o);
      unsigned long long b = __shfl_xor_sync(0xffffffffu, mx[d], o);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = b > mx[d] ? b : mx[d];
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&h->kmin[d], mn[d]);
      atomicMax(&h->kmax[d], mx[d]);
    }
  }
}

// Cells of edge >= rcut * (1 + 1e-4) over the bounding box [kmin, kmax] of n
// points, so that every pair closer than rcut lies in adjacent cells whatever
// the rounding; the dimensions are halved until at most max_cells remain.
__device__ __forceinline__ void grid_setup_from_keys(GridHeader& h,
                                                     const unsigned long long* kmin,
                                                     const unsigned long long* kmax, int n,
                                                     float rcut, int max_cells) {
  double edge = (double)rcut * 1.0001;
  int dims[3];
  double lo[3], ext[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = n > 0 ? ord_val(kmin[d]) : 0.;
    double hi = n > 0 ? ord_val(kmax[d]) : 0.;
    ext[d] = hi - lo[d];
    dims[d] = (int)(ext[d] / edge);
    if (dims[d] < 1) dims[d] = 1;
  }
  while ((long long)dims[0] * dims[1] * dims[2] > max_cells) {
    for (int d = 0; d < 3; ++d) dims[d] = dims[d] > 1 ? (dims[d] + 1) / 2 : 1;
  }
  for (int d = 0; d < 3; ++d) {
    h.dims[d] = dims[d];
    h.origin[d] = lo[d];
    double cs = ext[d] / dims[d];
    h.inv_cs[d] = cs > 0. ? 1. / cs : 0.;
  }
  h.ncells = dims[0] * dims[1] * dims[2];
  h.natoms = n;
}

__global__ void k_grid_setup(GridHeader* h, float rcut, int max_cells,
                             int nall, const int* nall_dev) {
  int n = nall_dev ? min(*nall_dev, nall) : nall;
  GridHeader v;
  grid_setup_from_keys(v, h->kmin, h->kmax, n, rcut, max_cells);
  for (int d = 0; d < 3; ++d) {
    h->dims[d] = v.dims[d];
    h->origin[d] = v.origin[d];
    h->inv_cs[d] = v.inv_cs[d];
  }
  h->ncells = v.ncells;
  h->natoms = v.natoms;
}

template <typename T>
__device__ __forceinline__ int grid_cell_of(const GridHeader& h, const T* p) {
  int c[3];
  for (int d = 0; d < 3; ++d) {
    int k = (int)(((double)p[d] - h.origin[d]) * h.inv_cs[d]);
    c[d] = k < 0 ? 0 : (k >= h.dims[d] ? h.dims[d] - 1 : k);
  }
  return (c[0] * h.dims[1] + c[1]) * h.dims[2] + c[2];
}

template <typename T>
__global__ void k_grid_count(GridView g, const T* coord) {
  const GridHeader& h = *g.h;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h.natoms) return;
  int c = grid_cell_of(h, coord + 3 * i);
  g.cell_of[i] = c;
  atomicAdd(&g.cell_start[c], 1);
}

__global__ void k_grid_scan(GridView g) {
  __shared__ int tot;
  block_exclusive_scan(g.cell_start, g.h->ncells + 1, &tot);
}

__global__ void k_grid_fill(GridView g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.h->natoms) return;
  int c = g.cell_of[i];
  int pos = g.cell_start[c] + atomicAdd(&g.fill[c], 1);
  g.cell_atoms[pos] = i;
}

long long grid_bytes(int nall) {
  int max_cells = nall > 64 ? nall : 64;
  long long ints = (long long)(max_cells + 1) + max_cells + 3LL * nall + 1 + 64;
  return (long long)sizeof(GridHeader) + 256 + ints * (long long)sizeof(int);
}

static long long packed_offset(int nall) { return (grid_bytes(nall) + 255) / 256 * 256; }

long long grid_bytes_packed(int nall) { return packed_offset(nall) + 32LL * nall; }

GridView carve_grid(void* p, int nall) {
  int max_cells = nall > 64 ? nall : 64;
  GridView g;
  // address only: dereferenced while h->packed == 1, which the fused
  // geometry pass sets only when the buffer has grid_bytes_packed(nall) bytes
  g.cell_pos = (double4*)((char*)p + packed_offset(nall));
  g.h = (GridHeader*)p;
  int* q = (int*)((char*)p + ((sizeof(GridHeader) + 255) / 256) * 256);
  g.cell_start = q; q += max_cells + 1;
  g.fill = q; q += max_cells;
  g.cell_of = q; q += nall;
  g.cell_atoms = q; q += nall;
  g.redo = q;
  g.max_cells = max_cells;
  g.cap_atoms = nall;
  return g;
}

template <typename T>
int grid_build(void* grid, long long bytes, const T* coord, int nall,
               const int* nall_dev, float rcut, cudaStream_t st) {
  if (nall < 0 || !(rcut > 0.f)) {
    set_error("cell grid: invalid arguments (nall=%d rcut=%g)", nall, (double)rcut);
    return DPB_ERR_INVALID;
  }
  if (grid == nullptr || bytes < grid_bytes(nall)) {
    set_error("cell grid: buffer too small (%lld < %lld bytes)", bytes, grid_bytes(nall));
    return DPB_ERR_INVALID;
  }
  GridView g = carve_grid(grid, nall);
  k_grid_init<<<1, 1, 0, st>>>(g.h);
  DPB_CHECK_LAUNCH("cell grid/init");
  int nb = nall > 0 ? ceil_div(nall, 256) : 1;
  if (nb > 148 * 8) nb = 148 * 8;
  k_grid_bbox<T><<<nb, 256, 0, st>>>(g.h, coord, nall, nall_dev);
  DPB_CHECK_LAUNCH("cell grid/bbox");
  k_grid_setup<<<1, 1, 0, st>>>(g.h, rcut, g.max_cells, nall, nall_dev);
  DPB_CHECK_LAUNCH("cell grid/setup");
  DPB_CUDA(cudaMemsetAsync(g.cell_start, 0, sizeof(int) * (2 * g.max_cells + 1), st),
           "cell grid");
  int na = nall > 0 ? ceil_div(nall, 256) : 1;
  k_grid_count<T><<<na, 256, 0, st>>>(g, coord);
  DPB_CHECK_LAUNCH("cell grid/count");
  k_grid_scan<<<1, 1024, 0, st>>>(g);
  DPB_CHECK_LAUNCH("cell grid/scan");
  k_grid_fill<<<na, 256, 0, st>>>(g);
  DPB_CHECK_LAUNCH("cell grid/fill");
  return DPB_OK;
}

// ------------------------------------------------- fused geometry pass ----
// normalize_coord + copy_coord + cell grid of one frame as ONE cooperative
// launch (64 blocks of 512 threads, at most one per SM). The separate path
// above takes twelve small launches and three memsets, each a few
// microseconds of latency for a few hundred kilobytes of work; here the
// phases are separated by four grid-wide barriers instead:
//   P0 local atoms: wrap into the box, copy-grid cell and a slot in it
//      (atomic count), local part of the extended arrays, bounding box keys
//   P1 every block scans the copy-cell counts in its own shared memory (no
//      single-block scan to wait for); atoms placed by cell; ghost offsets in
//      the reference's ghost loop order scanned the same way
//   P2 one warp per ghost cell: the source cell's atoms ranked by index in
//      registers or shared memory (copy_coord_cpu's ascending order), ghost
//      coordinates / types / mapping, bounding box keys
//   P3 every block derives the cell grid from the bounding box; atoms counted
//      per grid cell (atomic slot)
//   P4 every block scans the grid-cell counts; block 0 publishes the cell
//      starts and the grid header; atoms written in cell order.
// The results equal the separate path's bit for bit (extended coordinates,
// types, mapping, nall, grid header, cell starts, cell of every atom); only
// the order of atoms inside a grid cell may differ, which the neighbor
// search does not depend on (its keys are sorted).
//
// Barriers wait at most GEO_WAIT_NS; a block that gives up sets
// ST_SYNC_TIMEOUT in the status word and returns. Block 0 writes an empty
// grid header in P0 and the real one only in P4, so a pass that gave up
// leaves a grid in which the neighbor search finds nothing, never one that
// points outside its arrays.

constexpr int GEO_THREADS = 512;
constexpr int GEO_SCAN_CAP = 32768;  // ints of the block-local scans
constexpr int GEO_SORT_CAP = 256;    // per-warp buffer of one cell's atoms
constexpr int GEO_BLOCKS = 64;       // CTAs of the cooperative launch (at most the SMs)
constexpr unsigned long long GEO_WAIT_NS = 200000000ull;  // per barrier

struct GeoHeader {
  unsigned int arrive;  // barrier arrivals, zeroed before the launch
  unsigned int pad;
  unsigned long long kmin_inv[3];  // max of ~key, i.e. ~(min key)
  unsigned long long kmax[3];
};

struct GeoArgs {
  double* cext;
  int* text;
  int* mapping;
  int* nall_dev;
  GeoHeader* hdr;
  int* cnt;      // [nloc_cells] copy-cell counts, zeroed before the launch
  int* cell_of;  // [nloc] copy cell of each local atom
  int* slot;     // [nloc] slot inside it
  int* order;    // [nloc] local atoms by copy cell
  GridView g;
  int gcap;       // grid cells at most (<= g.max_cells, <= GEO_SCAN_CAP)
  int scan_ints;  // shared ints of the scans
  const double* coord;
  const int* atype;
  int nloc, mem_nall;
  float rcut;
  int* status;
  HostRegion r;
};

static long long geo_scratch_bytes(int nloc, const HostRegion& r) {
  const long long fused = 256 + 4LL * ((r.nloc_cells + 1) + 3LL * nloc) + 256;
  const long long sep = copy_scratch_ints(nloc, r) * (long long)sizeof(int);
  return fused > sep ? fused : sep;
}

__device__ __forceinline__ unsigned long long geo_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier number k (targets k * gridDim.x arrivals). Returns false
// in every thread of a block that gave up waiting.
__device__ bool geo_sync(const GeoArgs& a, unsigned k, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned target = k * gridDim.x;
    __threadfence();
    atomicAdd(&a.hdr->arrive, 1u);
    int ok = 1;
    if (ld_acquire_u32(&a.hdr->arrive) < target) {
      const unsigned long long t0 = geo_clock();
      unsigned it = 0;
      while (ld_acquire_u32(&a.hdr->arrive) < target) {
        if (++it > (1u << 24) || geo_clock() - t0 > GEO_WAIT_NS) {
          atomicOr(a.status, ST_SYNC_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Exclusive prefix sum of s[0, n) in shared memory, in place, by the whole
// block (each thread a contiguous run); returns the total.
__device__ int geo_scan(int* s, int n, int* s_warp) {
  __syncthreads();
  const int T = blockDim.x, t = threadIdx.x, lane = t & 31, wid = t >> 5, nw = T >> 5;
  const int k = (n + T - 1) / T;
  const int lo = min(n, t * k), hi = min(n, lo + k);
  int sum = 0;
  for (int j = lo; j < hi; ++j) sum += s[j];
  int x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  int run = (wid > 0 ? s_warp[wid - 1] : 0) + x - sum;
  for (int j = lo; j < hi; ++j) {
    const int v = s[j];
    s[j] = run;
    run += v;
  }
  const int total = s_warp[nw - 1];
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(GEO_THREADS, 1) k_geometry(GeoArgs a) {
  extern __shared__ int geo_smem[];
  __shared__ int s_warp[32];
  __shared__ int s_ok;
  __shared__ unsigned long long s_red[GEO_THREADS / 32][6];
  int* s_scan = geo_smem;
  int* s_sort = geo_smem + a.scan_ints;
  const HostRegion& r = a.r;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  unsigned long long kmn[3] = {0ull, 0ull, 0ull}, kmx[3] = {0ull, 0ull, 0ull};
  auto bbox = [&](const double* q) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const unsigned long long k = ord_key(q[d]);
      kmn[d] = max(kmn[d], ~k);
      kmx[d] = max(kmx[d], k);
    }
  };

  // ---- P0: local atoms
  for (int i = tid; i < a.nloc; i += nthr) {
    const double p[3] = {a.coord[3 * i], a.coord[3 * i + 1], a.coord[3 * i + 2]};
    double q[3];
    normalize_point(q, p, r);
    const int c = copy_cell_of(q, r);
    a.cell_of[i] = c;
    a.slot[i] = atomicAdd(&a.cnt[c], 1);
#pragma unroll
    for (int d = 0; d < 3; ++d) a.cext[3 * i + d] = q[d];
    a.text[i] = a.atype[i];
    a.mapping[i] = i;
    bbox(q);
  }
  for (int c = tid; c < a.gcap; c += nthr) a.g.fill[c] = 0;
  if (tid == 0) {
    GridHeader* h = a.g.h;
    for (int d = 0; d < 3; ++d) {
      h->dims[d] = 1;
      h->origin[d] = 0.;
      h->inv_cs[d] = 0.;
    }
    h->ncells = 1;
    h->natoms = 0;
    a.g.cell_start[0] = 0;
    a.g.cell_start[1] = 0;
  }
  if (!geo_sync(a, 1, &s_ok)) return;

  // ---- P1: copy-cell starts, local atoms by cell, ghost offsets
  const int ncl = r.nloc_cells, nce = r.next_cells;
  int* s_cs = s_scan;             // [ncl + 1]
  int* s_ext = s_scan + ncl + 1;  // [nce + 1]
  for (int j = threadIdx.x; j < ncl; j += blockDim.x) s_cs[j] = __ldcg(a.cnt + j);
  if (threadIdx.x == 0) s_cs[ncl] = 0;
  geo_scan(s_cs, ncl + 1, s_warp);
  for (int i = tid; i < a.nloc; i += nthr) a.order[s_cs[a.cell_of[i]] + a.slot[i]] = i;
  for (int e = threadIdx.x; e < nce; e += blockDim.x) {
    int ii[3];
    ext_cell_coords(e, r, ii);
    int v = 0;
    if (!(ii[0] >= 0 && ii[0] < r.nc[0] && ii[1] >= 0 && ii[1] < r.nc[1] && ii[2] >= 0 &&
          ii[2] < r.nc[2])) {
      int jj[3];
      for (int d = 0; d < 3; ++d) jj[d] = ii[d] + pbc_shift(ii[d], r.nc[d]) * r.nc[d];
      const int c = (jj[0] * r.nc[1] + jj[1]) * r.nc[2] + jj[2];
      v = s_cs[c + 1] - s_cs[c];
    }
    s_ext[e] = v;
  }
  if (threadIdx.x == 0) s_ext[nce] = 0;
  const int nall = a.nloc + geo_scan(s_ext, nce + 1, s_warp);
  if (tid == 0) *a.nall_dev = nall;
  if (!geo_sync(a, 2, &s_ok)) return;

  // ---- P2: ghosts, one warp per extended cell
  for (int e = blockIdx.x * nwb + wid; e < nce; e += gridDim.x * nwb) {
    int ii[3];
    ext_cell_coords(e, r, ii);
    if (ii[0] >= 0 && ii[0] < r.nc[0] && ii[1] >= 0 && ii[1] < r.nc[1] && ii[2] >= 0 &&
        ii[2] < r.nc[2])
      continue;
    int jj[3];
    double ps[3];
    for (int d = 0; d < 3; ++d) {
      const int sh = pbc_shift(ii[d], r.nc[d]);
      ps[d] = (double)sh;
      jj[d] = ii[d] + sh * r.nc[d];
    }
    double sv[3];
    dev_tt_dot_v(sv, r.box, ps);
    const int c = (jj[0] * r.nc[1] + jj[1]) * r.nc[2] + jj[2];
    const int b = s_cs[c], n = s_cs[c + 1] - b, w0 = a.nloc + s_ext[e];
    auto emit = [&](int w, int p) {
      if (w < a.mem_nall) {
        double q[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          q[d] = sub_rn(__ldcg(a.cext + 3 * p + d), sv[d]);
          a.cext[3 * w + d] = q[d];
        }
        a.text[w] = a.atype[p];
        a.mapping[w] = p;
        bbox(q);
      }
    };
    if (n <= 32) {
      const int v = lane < n ? __ldcg(a.order + b + lane) : 0x7fffffff;
      int rank = 0;
      for (int q = 0; q < n; ++q) rank += __shfl_sync(0xffffffffu, v, q) < v ? 1 : 0;
      if (lane < n) emit(w0 + rank, v);
    } else if (n <= GEO_SORT_CAP) {
      int* buf = s_sort + wid * GEO_SORT_CAP;
      for (int k = lane; k < n; k += 32) buf[k] = __ldcg(a.order + b + k);
      __syncwarp();
      for (int k = lane; k < n; k += 32) {
        const int x = buf[k];
        int rank = 0;
        for (int q = 0; q < n; ++q) rank += buf[q] < x ? 1 : 0;
        emit(w0 + rank, x);
      }
      __syncwarp();
    } else {
      for (int k = lane; k < n; k += 32) {
        const int x = __ldcg(a.order + b + k);
        int rank = 0;
        for (int q = 0; q < n; ++q) rank += __ldcg(a.order + b + q) < x ? 1 : 0;
        emit(w0 + rank, x);
      }
    }
  }
  // bounding box of this block's atoms: warp, then block, one atomic per key
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      kmn[d] = max(kmn[d], __shfl_xor_sync(0xffffffffu, kmn[d], o));
      kmx[d] = max(kmx[d], __shfl_xor_sync(0xffffffffu, kmx[d], o));
    }
    if (lane == 0) {
      s_red[wid][d] = kmn[d];
      s_red[wid][3 + d] = kmx[d];
    }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    unsigned long long m = 0ull;
    for (int w = 0; w < nwb; ++w) m = max(m, s_red[w][threadIdx.x]);
    if (m) {
      unsigned long long* dst = threadIdx.x < 3 ? &a.hdr->kmin_inv[threadIdx.x]
                                                : &a.hdr->kmax[threadIdx.x - 3];
      atomicMax(dst, m);
    }
  }
  if (!geo_sync(a, 3, &s_ok)) return;

  // ---- P3: cell grid over the extended atoms; counts per grid cell
  const int n = min(nall, a.mem_nall);
  unsigned long long kmin[3], kmax[3];
  for (int d = 0; d < 3; ++d) {
    kmin[d] = ~__ldcg(&a.hdr->kmin_inv[d]);
    kmax[d] = __ldcg(&a.hdr->kmax[d]);
  }
  GridHeader gh;
  grid_setup_from_keys(gh, kmin, kmax, n, a.rcut, a.gcap);
  int* gslot = a.g.redo + 1;  // the neighbor search zeroes redo[0] before use
  for (int i = tid; i < n; i += nthr) {
    const double q[3] = {__ldcg(a.cext + 3 * i), __ldcg(a.cext + 3 * i + 1),
                         __ldcg(a.cext + 3 * i + 2)};
    const int c = grid_cell_of(gh, q);
    a.g.cell_of[i] = c;
    gslot[i] = atomicAdd(&a.g.fill[c], 1);
  }
  if (!geo_sync(a, 4, &s_ok)) return;

  // ---- P4: grid cell starts; atoms in cell order
  const int ncg = gh.ncells;
  for (int j = threadIdx.x; j < ncg; j += blockDim.x) s_scan[j] = __ldcg(a.g.fill + j);
  if (threadIdx.x == 0) s_scan[ncg] = 0;
  geo_scan(s_scan, ncg + 1, s_warp);
  if (blockIdx.x == 0) {
    for (int j = threadIdx.x; j <= ncg; j += blockDim.x) a.g.cell_start[j] = s_scan[j];
    if (threadIdx.x == 0) {
      GridHeader* h = a.g.h;
      for (int d = 0; d < 3; ++d) {
        h->kmin[d] = kmin[d];
        h->kmax[d] = kmax[d];
        h->dims[d] = gh.dims[d];
        h->origin[d] = gh.origin[d];
        h->inv_cs[d] = gh.inv_cs[d];
      }
      h->ncells = gh.ncells;
      h->natoms = gh.natoms;
      h->packed = a.g.cell_pos != nullptr ? 1 : 0;
    }
  }
  if (a.g.cell_pos != nullptr) {
    // the atoms' positions, types and indices in cell order as well, so
    // that the env kernel's candidate walk reads them contiguously (written
    // in this launch before the last barrier: L2-coherent loads)
    for (int i = tid; i < n; i += nthr) {
      const int pos = s_scan[a.g.cell_of[i]] + gslot[i];
      a.g.cell_atoms[pos] = i;
      const long long w = ((long long)__ldcg(a.text + i) << 32) | (long long)(unsigned)i;
      a.g.cell_pos[pos] = make_double4(__ldcg(a.cext + 3 * i), __ldcg(a.cext + 3 * i + 1),
                                       __ldcg(a.cext + 3 * i + 2), __longlong_as_double(w));
    }
  } else {
    for (int i = tid; i < n; i += nthr) a.g.cell_atoms[s_scan[a.g.cell_of[i]] + gslot[i]] = i;
  }
}

// normalize_coord + copy_coord + cell grid of one frame. The fused pass runs
// when the copy grid's cells fit its block-local scans and the device can
// hold one block per SM; otherwise the separate kernels run (normalized
// coordinates written straight into the extended array).
int geometry_cells(double* cext, int* text, int* mapping, int* nall_dev, void* grid,
                   long long gbytes, void* scratch, long long sbytes, const double* coord,
                   const int* atype, int nloc, int mem_nall, float rcut, const double* boxt,
                   int* status, cudaStream_t st) {
  if (nloc < 0 || mem_nall < nloc || !(rcut > 0.f) || nall_dev == nullptr ||
      status == nullptr || (nloc > 0 && (!cext || !text || !mapping || !coord || !atype))) {
    set_error("geometry_cells: invalid arguments (nloc=%d mem_nall=%d rcut=%g; mem_nall "
              ">= nloc, nall_dev and status required)", nloc, mem_nall, (double)rcut);
    return DPB_ERR_INVALID;
  }
  HostRegion r;
  host_region(r, boxt, rcut);
  if (!(r.volume > 0.)) {
    set_error("geometry_cells: the box has zero volume");
    return DPB_ERR_INVALID;
  }
  const long long need = geo_scratch_bytes(nloc, r);
  if (scratch == nullptr || sbytes < need) {
    set_error("geometry_cells: scratch too small (%lld < %lld bytes)", sbytes, need);
    return DPB_ERR_INVALID;
  }
  if (grid == nullptr || gbytes < grid_bytes(mem_nall)) {
    set_error("geometry_cells: grid buffer too small (%lld < %lld bytes)", gbytes,
              grid_bytes(mem_nall));
    return DPB_ERR_INVALID;
  }
  GridView g = carve_grid(grid, mem_nall);
  if (gbytes < grid_bytes_packed(mem_nall)) g.cell_pos = nullptr;  // no room: not written
  const int gcap = g.max_cells < GEO_SCAN_CAP ? g.max_cells : GEO_SCAN_CAP;
  const long long copy_ints = (long long)r.nloc_cells + r.next_cells + 2;
  bool fused = nloc > 0 && copy_ints <= GEO_SCAN_CAP && tune_value("geometry_fused", 1) != 0;
  if (fused) {
    const int scan_ints = (int)(copy_ints > gcap + 1 ? copy_ints : gcap + 1);
    const size_t smem = (size_t)scan_ints * 4 + (size_t)(GEO_THREADS / 32) * GEO_SORT_CAP * 4;
    // devices whose shared-memory limit is raised; atomic so that host
    // threads calling this concurrently do not race on the mask (setting the
    // attribute twice is harmless)
    static std::atomic<unsigned long long> attr_devs{0};
    int dev = 0;
    DPB_CUDA(cudaGetDevice(&dev), "geometry_cells");
    if (dev < 64 && !(attr_devs.load(std::memory_order_acquire) >> dev & 1ull)) {
      // scan_ints is at most GEO_SCAN_CAP + 1 (gcap + 1 cell starts)
      const int most = (GEO_SCAN_CAP + 1) * 4 + (GEO_THREADS / 32) * GEO_SORT_CAP * 4;
      DPB_CUDA(cudaFuncSetAttribute(k_geometry, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    most),
               "geometry_cells");
      attr_devs.fetch_or(1ull << dev, std::memory_order_acq_rel);
    }
    int occ = 0;
    DPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_geometry, GEO_THREADS,
                                                           smem),
             "geometry_cells");
    if (occ >= 1) {
      char* p = (char*)scratch;
      GeoArgs a;
      a.cext = cext;
      a.text = text;
      a.mapping = mapping;
      a.nall_dev = nall_dev;
      a.hdr = (GeoHeader*)p;
      a.cnt = (int*)(p + 256);
      a.cell_of = a.cnt + r.nloc_cells + 1;
      a.slot = a.cell_of + nloc;
      a.order = a.slot + nloc;
      a.g = g;
      a.gcap = gcap;
      a.scan_ints = scan_ints;
      a.coord = coord;
      a.atype = atype;
      a.nloc = nloc;
      a.mem_nall = mem_nall;
      a.rcut = rcut;
      a.status = status;
      a.r = r;
      DPB_CUDA(cudaMemsetAsync(scratch, 0, 256 + sizeof(int) * (size_t)r.nloc_cells, st),
               "geometry_cells");
      void* args[] = {&a};
      // 64 CTAs: every phase is grid-stride and small, and each barrier costs
      // one arrival per CTA
      const int blocks = sm_count() < GEO_BLOCKS ? sm_count() : GEO_BLOCKS;
      DPB_CUDA(cudaLaunchCooperativeKernel((const void*)k_geometry, dim3(blocks),
                                           dim3(GEO_THREADS), args, smem, st),
               "geometry_cells");
      return DPB_OK;
    }
  }
  if (nloc > 0) {
    DPB_CUDA(cudaMemcpyAsync(cext, coord, sizeof(double) * 3 * (size_t)nloc,
                             cudaMemcpyDeviceToDevice, st),
             "geometry_cells");
    k_normalize<double><<<ceil_div(nloc, 256), 256, 0, st>>>(cext, nloc, r);
    DPB_CHECK_LAUNCH("geometry_cells/normalize");
  }
  int rc = copy_coord_async<double>(cext, text, mapping, nall_dev, scratch, sbytes, cext,
                                    atype, nloc, mem_nall, rcut, boxt, st);
  if (rc != DPB_OK) return rc;
  return grid_build<double>(grid, gbytes, cext, mem_nall, nall_dev, rcut, st);
}

long long geometry_scratch_bytes(int nloc, float rcut, const double* boxt) {
  HostRegion r;
  host_region(r, boxt, rcut);
  return geo_scratch_bytes(nloc, r);
}

template int grid_build<double>(void*, long long, const double*, int, const int*, float, cudaStream_t);
template int grid_build<float>(void*, long long, const float*, int, const int*, float, cudaStream_t);
template int copy_coord_async<double>(double*, int*, int*, int*, void*, long long, const double*,
                                      const int*, int, int, float, const double*, cudaStream_t);
template int copy_coord_async<float>(float*, int*, int*, int*, void*, long long, const float*,
                                     const int*, int, int, float, const double*, cudaStream_t);

long long copy_coord_scratch_bytes(int nloc, float rcut, const double* boxt) {
  HostRegion r;
  host_region(r, boxt, rcut);
  return copy_scratch_ints(nloc, r) * (long long)sizeof(int);
}

}  // namespace dpb

// ------------------------------------------------------------- C-ABI -------
using namespace dpb;
// ghost j keeps its periodic image between list rebuilds: shift_j =
// c_ext_j - c_{mapping_j} at the rebuild, c_ext_j = c_{mapping_j} + shift_j
// at every later step (the positions are not re-wrapped between rebuilds)
__global__ void k_ghost_shift(double* shift, const double* cext, const double* coord,
                              const int* mapping, const int* nall_dev, int mem_nall) {
  const int n = nall_dev ? min(*nall_dev, mem_nall) : mem_nall;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int o = mapping[j];
#pragma unroll
    for (int d = 0; d < 3; ++d) shift[3 * j + d] = cext[3 * j + d] - coord[3 * o + d];
  }
}

__global__ void k_ghost_refresh(double* cext, const double* shift, const double* coord,
                                const int* mapping, const int* nall_dev, int mem_nall) {
  const int n = nall_dev ? min(*nall_dev, mem_nall) : mem_nall;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int o = mapping[j];
#pragma unroll
    for (int d = 0; d < 3; ++d) cext[3 * j + d] = coord[3 * o + d] + shift[3 * j + d];
  }
}

extern "C" {

int dpb_ghost_shift_f64(double* shift, const double* cext, const double* coord,
                        const int* mapping, const int* nall_dev, int mem_nall,
                        dpb_stream_t stream) {
  if (mem_nall < 0 || (mem_nall > 0 && (!shift || !cext || !coord || !mapping))) {
    set_error("ghost_shift: invalid arguments");
    return DPB_ERR_INVALID;
  }
  if (mem_nall == 0) return DPB_OK;
  k_ghost_shift<<<grid_stride_blocks(mem_nall, 256), 256, 0, as_stream(stream)>>>(
      shift, cext, coord, mapping, nall_dev, mem_nall);
  DPB_CHECK_LAUNCH("ghost_shift");
  return DPB_OK;
}

int dpb_ghost_refresh_f64(double* cext, const double* shift, const double* coord,
                          const int* mapping, const int* nall_dev, int mem_nall,
                          dpb_stream_t stream) {
  if (mem_nall < 0 || (mem_nall > 0 && (!shift || !cext || !coord || !mapping))) {
    set_error("ghost_refresh: invalid arguments");
    return DPB_ERR_INVALID;
  }
  if (mem_nall == 0) return DPB_OK;
  k_ghost_refresh<<<grid_stride_blocks(mem_nall, 256), 256, 0, as_stream(stream)>>>(
      cext, shift, coord, mapping, nall_dev, mem_nall);
  DPB_CHECK_LAUNCH("ghost_refresh");
  return DPB_OK;
}


int dpb_normalize_coord_f64(double* coord, int natom, const double* boxt,
                            dpb_stream_t stream) {
  if (natom <= 0) return DPB_OK;
  HostRegion r;
  host_region(r, boxt, 1.f);
  k_normalize<double><<<ceil_div(natom, 256), 256, 0, as_stream(stream)>>>(coord, natom, r);
  DPB_CHECK_LAUNCH("normalize_coord");
  return DPB_OK;
}

int dpb_normalize_coord_f32(float* coord, int natom, const float* boxt,
                            dpb_stream_t stream) {
  if (natom <= 0) return DPB_OK;
  // the reference keeps float boxes in float (region.cc:38-90)
  double b[9];
  for (int k = 0; k < 9; ++k) b[k] = boxt[k];
  HostRegion r;
  host_region(r, b, 1.f);
  float bf[9], rf[9];
  for (int k = 0; k < 9; ++k) bf[k] = boxt[k];
  float v = bf[0] * (bf[4] * bf[8] - bf[7] * bf[5]) - bf[1] * (bf[3] * bf[8] - bf[6] * bf[5]) +
            bf[2] * (bf[3] * bf[7] - bf[6] * bf[4]);
  v = fabsf(v);
  float vi = 1.f / v;
  rf[0] = (bf[4] * bf[8] - bf[7] * bf[5]) * vi;
  rf[4] = (bf[0] * bf[8] - bf[6] * bf[2]) * vi;
  rf[8] = (bf[0] * bf[4] - bf[3] * bf[1]) * vi;
  rf[1] = (-bf[3] * bf[8] + bf[6] * bf[5]) * vi;
  rf[2] = (bf[3] * bf[7] - bf[6] * bf[4]) * vi;
  rf[3] = (-bf[1] * bf[8] + bf[7] * bf[2]) * vi;
  rf[5] = (-bf[0] * bf[7] + bf[6] * bf[1]) * vi;
  rf[6] = (bf[1] * bf[5] - bf[4] * bf[2]) * vi;
  rf[7] = (-bf[0] * bf[5] + bf[3] * bf[2]) * vi;
  for (int k = 0; k < 9; ++k) {
    r.rec[k] = rf[k];
    r.box[k] = bf[k];
  }
  k_normalize<float><<<ceil_div(natom, 256), 256, 0, as_stream(stream)>>>(coord, natom, r);
  DPB_CHECK_LAUNCH("normalize_coord");
  return DPB_OK;
}

long long dpb_copy_coord_scratch_bytes(int nloc, float rcut, const double* boxt) {
  return copy_coord_scratch_bytes(nloc, rcut, boxt);
}

int dpb_copy_coord_f64(double* out_c, int* out_t, int* mapping, int* nall,
                       void* scratch, long long scratch_bytes,
                       const double* in_c, const int* in_t, int nloc,
                       int mem_nall, float rcut, const double* boxt,
                       dpb_stream_t stream) {
  return copy_coord_sync<double>(out_c, out_t, mapping, nall, scratch,
                                 scratch_bytes, in_c, in_t, nloc, mem_nall,
                                 rcut, boxt, as_stream(stream));
}

int dpb_copy_coord_f32(float* out_c, int* out_t, int* mapping, int* nall,
                       void* scratch, long long scratch_bytes,
                       const float* in_c, const int* in_t, int nloc,
                       int mem_nall, float rcut, const float* boxt,
                       dpb_stream_t stream) {
  return copy_coord_sync<float>(out_c, out_t, mapping, nall, scratch,
                                scratch_bytes, in_c, in_t, nloc, mem_nall,
                                rcut, boxt, as_stream(stream));
}

long long dpb_copy_coord_cells_scratch_bytes(int nloc, const int* cell_info) {
  return copy_coord_cells_scratch_bytes(nloc, cell_info);
}

int dpb_copy_coord_cells_f64(double* out_c, int* out_t, int* mapping, int* nall, void* scratch,
                             long long scratch_bytes, const double* in_c, const int* in_t,
                             int nloc, int mem_nall, const int* cell_info, const double* boxt,
                             dpb_stream_t stream) {
  return copy_coord_cells<double>(out_c, out_t, mapping, nall, scratch, scratch_bytes, in_c,
                                  in_t, nloc, mem_nall, cell_info, boxt, as_stream(stream));
}

int dpb_copy_coord_cells_f32(float* out_c, int* out_t, int* mapping, int* nall, void* scratch,
                             long long scratch_bytes, const float* in_c, const int* in_t,
                             int nloc, int mem_nall, const int* cell_info, const float* boxt,
                             dpb_stream_t stream) {
  return copy_coord_cells<float>(out_c, out_t, mapping, nall, scratch, scratch_bytes, in_c,
                                 in_t, nloc, mem_nall, cell_info, boxt, as_stream(stream));
}

long long dpb_cell_grid_bytes(int nall) { return grid_bytes(nall); }

long long dpb_cell_grid_bytes_packed(int nall) { return grid_bytes_packed(nall); }

long long dpb_geometry_scratch_bytes(int nloc, float rcut, const double* boxt) {
  return geometry_scratch_bytes(nloc, rcut, boxt);
}

int dpb_geometry_cells_f64(double* cext, int* text, int* mapping, int* nall_dev, void* grid,
                           long long grid_bytes_, void* scratch, long long scratch_bytes,
                           const double* coord, const int* atype, int nloc, int mem_nall,
                           float rcut, const double* boxt, int* status,
                           dpb_stream_t stream) {
  return geometry_cells(cext, text, mapping, nall_dev, grid, grid_bytes_, scratch,
                        scratch_bytes, coord, atype, nloc, mem_nall, rcut, boxt, status,
                        as_stream(stream));
}

int dpb_cell_grid_build_f64(void* grid, long long grid_bytes_, const double* coord,
                            int nall, float rcut, dpb_stream_t stream) {
  return grid_build<double>(grid, grid_bytes_, coord, nall, nullptr, rcut,
                            as_stream(stream));
}

int dpb_cell_grid_build_f32(void* grid, long long grid_bytes_, const float* coord,
                            int nall, float rcut, dpb_stream_t stream) {
  return grid_build<float>(grid, grid_bytes_, coord, nall, nullptr, rcut,
                           as_stream(stream));
}

}  // extern "C"
