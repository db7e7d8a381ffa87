// Device bodies of the batched-frames passes (dpb_batch.cu): one frame's
// wrap and cell binning, one center row's env pass, one row's force / virial
// and one frame's energy. The per-stage kernels of dpb_batch.cu and the
// persistent fused kernels of dpb_se_a.cu call them.
#pragma once

#include "dpb_batch.cuh"
#include "dpb_envmath.cuh"

namespace dpb {

// one frame's wrap and cell binning (counting sort); every thread of the
// block takes part; cnt: shared memory of BT_MAXCELLS + 1 ints
__device__ __forceinline__ void bt_cells_frame(int f, double* __restrict__ cw,
                                               int* __restrict__ cell_of,
                                               int* __restrict__ cell_start,
                                               int* __restrict__ cell_atoms,
                                               const double* __restrict__ coord,
                                               const BtFrames& fr, int* cnt) {
  const int a0 = fr.atom_off[f], na = fr.atom_off[f + 1] - a0;
  const int nx = fr.ncell[3 * f], ny = fr.ncell[3 * f + 1], nz = fr.ncell[3 * f + 2];
  const int nc = nx * ny * nz;
  const double L[3] = {fr.box[3 * f], fr.box[3 * f + 1], fr.box[3 * f + 2]};
  for (int c = threadIdx.x; c <= nc; c += blockDim.x) cnt[c] = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < na; k += blockDim.x) {
    double w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double x = coord[3 * (size_t)(a0 + k) + d];
      w[d] = x - floor(x / L[d]) * L[d];
      if (w[d] >= L[d]) w[d] -= L[d];  // rounding at the upper edge
      if (w[d] < 0.0) w[d] += L[d];    // and at the lower one
      cw[3 * (size_t)(a0 + k) + d] = w[d];
    }
    const int c = (bt_wrap_cell(w[0], L[0], nx) * ny + bt_wrap_cell(w[1], L[1], ny)) * nz +
                  bt_wrap_cell(w[2], L[2], nz);
    cell_of[a0 + k] = c;
    atomicAdd(&cnt[c + 1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0)  // exclusive offsets over at most 4096 cells
    for (int c = 0; c < nc; ++c) cnt[c + 1] += cnt[c];
  __syncthreads();
  int* cs = cell_start + fr.cell_off[f];
  for (int c = threadIdx.x; c <= nc; c += blockDim.x) cs[c] = cnt[c];
  __syncthreads();
  for (int k = threadIdx.x; k < na; k += blockDim.x) {
    const int pos = atomicAdd(&cnt[cell_of[a0 + k]], 1);
    cell_atoms[a0 + pos] = k;
  }
}

struct BtEnvSmem {
  __align__(16) unsigned long long keys[BT_CAP];  // read two at a time by the ranking
  int row[BT_NMAX];
  int tcnt[32];
};

// one center row of the batched env pass (one warp): candidates over the 27
// lattice cells, keys, sel slots, env rows; sm: this warp's shared memory
template <typename ET>
__device__ __forceinline__ void bt_env_row(int row, int lane, BtEnvSmem& sm,
                                           ET* __restrict__ em, int* __restrict__ nlist,
                                           const double* __restrict__ cw,
                                           const int* __restrict__ type,
                                           const int* __restrict__ cell_of,
                                           const int* __restrict__ cell_start,
                                           const int* __restrict__ cell_atoms,
                                           const ET* __restrict__ avg,
                                           const ET* __restrict__ std_, const BtFrames& fr,
                                           const BtSec& sec, float rcut, float rcut_smth,
                                           int* status) {
  const int f = fr.row_frame[row];
  const int a0 = fr.atom_off[f];
  const int i = row - a0;
  const int nx = fr.ncell[3 * f], ny = fr.ncell[3 * f + 1], nz = fr.ncell[3 * f + 2];
  const double L[3] = {fr.box[3 * f], fr.box[3 * f + 1], fr.box[3 * f + 2]};
  const double* fc = cw + 3 * (size_t)a0;
  const int* ft = type + a0;
  const int* cs = cell_start + fr.cell_off[f];
  const int* ca = cell_atoms + a0;
  const int nnei = sec.nnei, ntypes = sec.ntypes;
  int ti = ft[i];
  if (ti < 0 || ti >= ntypes) {
    if (lane == 0) atomicOr(status, ST_TYPE_RANGE);
    ti = -1;
  }
  const double xi[3] = {fc[3 * i], fc[3 * i + 1], fc[3 * i + 2]};
  const float fxi[3] = {(float)xi[0], (float)xi[1], (float)xi[2]};
  const float rc2f = rcut * rcut;
  const double rc2 = (double)rc2f;
  for (int t = lane; t < 32; t += 32) sm.tcnt[t] = 0;
  for (int jj = lane; jj < nnei; jj += 32) sm.row[jj] = -1;
  __syncwarp();
  int count = 0;
  const int ci = cell_of[row];
  const int cz = ci % nz, cy = (ci / nz) % ny, cx = ci / (nz * ny);
  // lane L < 27 owns lattice cell (cx, cy, cz) + (L / 9, L / 3 % 3, L % 3) - 1:
  // its stored (wrapped) cell's atom range and its image code; the 27 ranges
  // are then walked as one flat list in full batches of 32, the next batch's
  // atom indices requested before the current batch is tested
  int cb = 0, cn = 0, ccode = 13;
  if (lane < 27) {
    int X = cx + lane / 9 - 1, Y = cy + (lane / 3) % 3 - 1, Z = cz + lane % 3 - 1;
    const int sx = X < 0 ? -1 : (X >= nx ? 1 : 0);
    const int sy = Y < 0 ? -1 : (Y >= ny ? 1 : 0);
    const int sz = Z < 0 ? -1 : (Z >= nz ? 1 : 0);
    X -= sx * nx;
    Y -= sy * ny;
    Z -= sz * nz;
    ccode = (sx + 1) * 9 + (sy + 1) * 3 + (sz + 1);
    const int c = (X * ny + Y) * nz + Z;
    cb = cs[c];
    cn = cs[c + 1] - cb;
  }
  int incl = cn;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int excl = incl - cn;
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  // atom (-1 past the end) and image code of flat candidate fl
  auto cand_of = [&](int fl, int& code) -> int {
    int lo = 0;
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
      const int ev = __shfl_sync(0xffffffffu, excl, lo + st);
      if (ev <= fl) lo += st;
    }
    const int base_c = __shfl_sync(0xffffffffu, cb, lo);
    const int start_c = __shfl_sync(0xffffffffu, excl, lo);
    code = __shfl_sync(0xffffffffu, ccode, lo);
    return fl < total ? ca[base_c + (fl - start_c)] : -1;
  };
  int coden = 13;
  int jn = cand_of(lane, coden);
  for (int base = 0; base < total; base += 32) {
    const int j = jn, code = coden;
    jn = cand_of(base + 32 + lane, coden);
    bool ok = false;
    unsigned long long key = 0;
    if (j >= 0) {
      const int tj = ft[j];
      if (tj >= 0 && tj < ntypes && ti >= 0 && !(j == i && code == 13)) {
        const int sx = code / 9 - 1, sy = (code / 3) % 3 - 1, sz = code % 3 - 1;
        const double sh[3] = {sx * L[0], sy * L[1], sz * L[2]};
        // the image's position, then the single-frame path's two tests
        const double g0 = fc[3 * j] + sh[0], g1 = fc[3 * j + 1] + sh[1],
                     g2 = fc[3 * j + 2] + sh[2];
        const double d0 = sub_rn(xi[0], g0), d1 = sub_rn(xi[1], g1), d2 = sub_rn(xi[2], g2);
        if (dot3_rn(d0, d1, d2) < rc2) {
          const float e0 = sub_rn((float)g0, fxi[0]), e1 = sub_rn((float)g1, fxi[1]),
                      e2 = sub_rn((float)g2, fxi[2]);
          const float r2 = dot3_rn(e0, e1, e2);
          if (r2 <= rc2f) {
            ok = true;
            key = ((unsigned long long)tj << 56) |
                  ((unsigned long long)__float_as_uint(r2) << 24) |
                  (unsigned long long)(j * 27 + code);
          }
        }
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) {
      const int pos = count + __popc(bal & bt_lanemask_lt());
      if (pos < BT_CAP) {
        sm.keys[pos] = key;
        atomicAdd(&sm.tcnt[key >> 56], 1);
      }
    }
    count += __popc(bal);
  }
  __syncwarp();
  if (count > BT_CAP && lane == 0) atomicOr(status, ST_NLIST_CAPACITY);
  const int n = count < BT_CAP ? count : BT_CAP;
  int tstart = lane < ntypes ? sm.tcnt[lane] : 0;
  {
    int x = tstart;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    tstart = x - tstart;
  }
  for (int q = 0; q * 32 < n; ++q) {
    const int kk = q * 32 + lane;
    const unsigned long long own = kk < n ? sm.keys[kk] : ~0ull;
    int r = 0;
    const ulonglong2* k2 = reinterpret_cast<const ulonglong2*>(sm.keys);
    int p = 0;
    for (; 2 * p + 1 < n; ++p) {  // two keys per 16-byte load (broadcast)
      const ulonglong2 v = k2[p];
      r += (v.x < own ? 1 : 0) + (v.y < own ? 1 : 0);
    }
    if (2 * p < n) r += sm.keys[2 * p] < own ? 1 : 0;
    const int t = (int)(own >> 56) & 31;
    const int ts = __shfl_sync(0xffffffffu, tstart, t);
    if (kk < n) {
      const int rr = r - ts;
      if (rr < sec.sec[t + 1] - sec.sec[t]) sm.row[sec.sec[t] + rr] = (int)(own & 0xFFFFFFull);
      else atomicOr(status, ST_SEL_OVERFLOW);
    }
  }
  __syncwarp();
  const ET* av = avg + (size_t)(ti < 0 ? 0 : ti) * nnei * 4;
  const ET* sd = std_ + (size_t)(ti < 0 ? 0 : ti) * nnei * 4;
  for (int jj = lane; jj < nnei; jj += 32) {
    const int packed = sm.row[jj];
    nlist[(size_t)row * nnei + jj] = packed;
    ET v[4] = {(ET)0, (ET)0, (ET)0, (ET)0};
    if (packed >= 0) {
      ET r[3];
      bt_rij<ET>(r, fc, packed, xi, L);
      env_row<ET>(r, rcut_smth, rcut, v, nullptr);
    }
    ET* e = em + ((size_t)row * nnei + jj) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      e[k] = ti >= 0 ? (v[k] - av[jj * 4 + k]) / sd[jj * 4 + k] : (ET)0;
  }
}

// forces and virial of one center row (one warp): the env derivative
// recomputed from the packed (atom, image) neighbors, pair forces added to
// the owners, the frame's virial by one atomic per component. COH: the row's
// net_deriv was written earlier in the same launch (read from L2)
template <typename ET, bool COH = false>
__device__ __forceinline__ void bt_force_row(int row, int lane, double* __restrict__ force,
                                             double* __restrict__ virial,
                                             const ET* __restrict__ nd,
                                             const double* __restrict__ cw,
                                             const int* __restrict__ type,
                                             const ET* __restrict__ std_,
                                             const int* __restrict__ nlist, const BtFrames& fr,
                                             int ntypes, int nnei, float rcut,
                                             float rcut_smth) {
  const int f = fr.row_frame[row];
  const int a0 = fr.atom_off[f];
  const int i = row - a0;
  const int ti = type[row];
  if (ti < 0 || ti >= ntypes) return;  // env derivative rows are zero
  const double L[3] = {fr.box[3 * f], fr.box[3 * f + 1], fr.box[3 * f + 2]};
  const double* fc = cw + 3 * (size_t)a0;
  const double xi[3] = {fc[3 * i], fc[3 * i + 1], fc[3 * i + 2]};
  const ET* sd = std_ + (size_t)ti * nnei * 4;
  const ET* ndr = nd + (size_t)row * nnei * 4;
  const ET inv_span = (ET)1. / (ET)(rcut - rcut_smth);
  double c0 = 0., c1 = 0., c2 = 0.;
  double vs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vs[k] = 0.;
  for (int jj = lane; jj < nnei; jj += 32) {
    const int packed = nlist[(size_t)row * nnei + jj];
    if (packed < 0) continue;
    const int j = packed / 27;
    ET r[3];
    bt_rij<ET>(r, fc, packed, xi, L);
    ET gd[12];
    env_deriv<ET>(r, rcut_smth, rcut, inv_span, gd);
    ET p[3] = {(ET)0, (ET)0, (ET)0};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const ET n = COH ? __ldcg(ndr + jj * 4 + a) : ndr[jj * 4 + a];
      const ET ns = n / sd[jj * 4 + a];  // dE/d(env): one division per env column
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += ns * gd[a * 3 + d];
    }
    const double q[3] = {(double)p[0], (double)p[1], (double)p[2]};
    c0 += q[0];
    c1 += q[1];
    c2 += q[2];
    atomicAdd(&force[3 * (size_t)(a0 + j) + 0], q[0]);
    atomicAdd(&force[3 * (size_t)(a0 + j) + 1], q[1]);
    atomicAdd(&force[3 * (size_t)(a0 + j) + 2], q[2]);
#pragma unroll
    for (int d0 = 0; d0 < 3; ++d0)
#pragma unroll
      for (int d1 = 0; d1 < 3; ++d1) vs[d0 * 3 + d1] += q[d0] * (double)r[d1];
  }
  c0 = warp_sum(c0);
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  if (lane == 0) {
    atomicAdd(&force[3 * (size_t)row + 0], -c0);
    atomicAdd(&force[3 * (size_t)row + 1], -c1);
    atomicAdd(&force[3 * (size_t)row + 2], -c2);
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const double t = warp_sum(vs[k]);
    if (lane == 0) atomicAdd(&virial[9 * (size_t)f + k], t);
  }
}

// energy of one frame (every thread of the block): e_const[f] plus its
// fitting rows' atomic energies in FP64; part: shared memory of blockDim/32
template <typename ET>
__device__ __forceinline__ void bt_energy_frame(int f, double* __restrict__ energy,
                                                const ET* __restrict__ e_rows,
                                                const int* __restrict__ drow,
                                                const double* __restrict__ e_const,
                                                const BtFrames& fr, double* part) {
  double s = 0.;
  for (int r = fr.atom_off[f] + threadIdx.x; r < fr.atom_off[f + 1]; r += blockDim.x)
    s += (double)e_rows[drow[r]];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = e_const[f];
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
    energy[f] = t;
  }
}

}  // namespace dpb
