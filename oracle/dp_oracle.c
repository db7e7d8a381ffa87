/* Test infrastructure only: plain-C restatement of the reference DeePMD-kit CPU
 * algorithms on the se_e2_a energy/force/virial path (the checker for the CUDA
 * implementation; never linked into the product). See dp_oracle.h for the
 * reference file:line each function restates. Built with -ffp-contract=off. */
#include "dp_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- region -- */

static double det3(const double* b) {
  /* source/lib/include/SimulationRegion_Impl.h:429-438 */
  double v = b[0] * (b[4] * b[8] - b[7] * b[5]) -
             b[1] * (b[3] * b[8] - b[6] * b[5]) +
             b[2] * (b[3] * b[7] - b[6] * b[4]);
  return fabs(v);
}

void orc_rec_boxt(double* r, double* volume, const double* b) {
  /* cofactor inverse, same term order as
   * source/lib/include/SimulationRegion_Impl.h:455-480 */
  double vol = det3(b);
  double vi = 1. / vol;
  r[0] = (b[4] * b[8] - b[7] * b[5]) * vi;
  r[4] = (b[0] * b[8] - b[6] * b[2]) * vi;
  r[8] = (b[0] * b[4] - b[3] * b[1]) * vi;
  r[1] = (-b[3] * b[8] + b[6] * b[5]) * vi;
  r[2] = (b[3] * b[7] - b[6] * b[4]) * vi;
  r[3] = (-b[1] * b[8] + b[7] * b[2]) * vi;
  r[5] = (-b[0] * b[7] + b[6] * b[1]) * vi;
  r[6] = (b[1] * b[5] - b[4] * b[2]) * vi;
  r[7] = (-b[0] * b[5] + b[3] * b[2]) * vi;
  if (volume) *volume = vol;
}

/* o = t . v (row-major), SimulationRegion_Impl.h:388-396 */
static void t_dot_v(double* o, const double* t, const double* v) {
  o[0] = v[0] * t[0] + v[1] * t[1] + v[2] * t[2];
  o[1] = v[0] * t[3] + v[1] * t[4] + v[2] * t[5];
  o[2] = v[0] * t[6] + v[1] * t[7] + v[2] * t[8];
}
/* o = t^T . v, SimulationRegion_Impl.h:399-407 */
static void tt_dot_v(double* o, const double* t, const double* v) {
  o[0] = v[0] * t[0] + v[1] * t[3] + v[2] * t[6];
  o[1] = v[0] * t[1] + v[1] * t[4] + v[2] * t[7];
  o[2] = v[0] * t[2] + v[1] * t[5] + v[2] * t[8];
}

void orc_normalize_coord(double* coord, int natom, const double* boxt) {
  double rec[9];
  orc_rec_boxt(rec, NULL, boxt);
  for (int ii = 0; ii < natom; ++ii) {
    double ri[3];
    t_dot_v(ri, rec, coord + 3 * ii);
    for (int dd = 0; dd < 3; ++dd) {
      ri[dd] = fmod(ri[dd], 1.);
      if (ri[dd] < 0.) ri[dd] += 1.;
    }
    tt_dot_v(coord + 3 * ii, boxt, ri);
  }
}

static void cprod(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

static void to_face(double* d, const double* b) {
  /* SimulationRegion_Impl.h:364-372 */
  double vol = det3(b), tmp[3];
  cprod(b + 3, b + 6, tmp);
  d[0] = vol * (1. / sqrt(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]));
  cprod(b + 6, b + 0, tmp);
  d[1] = vol * (1. / sqrt(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]));
  cprod(b + 0, b + 3, tmp);
  d[2] = vol * (1. / sqrt(tmp[0] * tmp[0] + tmp[1] * tmp[1] + tmp[2] * tmp[2]));
}

int orc_compute_cell_info(int* ci, float rcut, const double* boxt) {
  double tf[3], cs[3];
  to_face(tf, boxt);
  for (int dd = 0; dd < 3; ++dd) {
    ci[dd] = 0;
    ci[3 + dd] = (int)(tf[dd] / rcut);
    if (ci[3 + dd] == 0) ci[3 + dd] = 1;
    cs[dd] = tf[dd] / ci[3 + dd];
    ci[12 + dd] = (int)(rcut / cs[dd]) + 1;
    ci[6 + dd] = -ci[12 + dd];
    ci[9 + dd] = ci[3 + dd] + ci[12 + dd];
    ci[15 + dd] = ci[12 + dd];
    ci[18 + dd] = (int)(rcut / cs[dd]);
    if (ci[18 + dd] * cs[dd] < rcut) ci[18 + dd] += 1;
  }
  ci[21] = ci[3] * ci[4] * ci[5];
  ci[22] = (2 * ci[12] + ci[3]) * (2 * ci[13] + ci[4]) * (2 * ci[14] + ci[5]);
  return ci[21] > 0 ? 0 : 2;
}

static int pbc_shift(int idx, int n) {
  /* source/lib/src/neighbor_list.cc:730-745 */
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

int orc_copy_coord(double* out_c, int* out_t, int* mapping, int* nall,
                   const double* in_c, const int* in_t, int nloc, int mem_nall,
                   float rcut, const double* boxt) {
  double rec[9], tf[3], cs[3], rc = (double)rcut;
  int nc[3], ng[3];
  orc_rec_boxt(rec, NULL, boxt);
  to_face(tf, boxt);
  for (int dd = 0; dd < 3; ++dd) {
    nc[dd] = (int)(tf[dd] / rc);
    if (nc[dd] == 0) nc[dd] = 1;
    cs[dd] = tf[dd] / nc[dd];
    ng[dd] = (int)(rc / cs[dd]) + 1;
  }
  /* cell list of the local atoms (build_clist, neighbor_list.cc:43-112), with
   * nat_stt = ext_stt = 0, nat_end = ext_end = global_grid = ncell */
  int ncl = nc[0] * nc[1] * nc[2];
  if (ncl <= 0 || nloc < 0) return 2; /* cell count out of int range: not a box */
  int* cell_of = (int*)malloc(sizeof(int) * (nloc > 0 ? nloc : 1));
  int* cnt = (int*)calloc(ncl + 1, sizeof(int));
  for (int ii = 0; ii < nloc; ++ii) {
    double inter[3];
    int idx[3];
    t_dot_v(inter, rec, in_c + 3 * ii);
    for (int dd = 0; dd < 3; ++dd) {
      double csz = 1. / nc[dd];
      idx[dd] = (int)((inter[dd] - 0.) / csz);
      if (inter[dd] - 0. < 0.) idx[dd]--;
      if (idx[dd] < 0) idx[dd] = 0;
      else if (idx[dd] >= nc[dd]) idx[dd] = nc[dd] - 1;
    }
    cell_of[ii] = (idx[0] * nc[1] + idx[1]) * nc[2] + idx[2];
    cnt[cell_of[ii] + 1]++;
  }
  for (int c = 0; c < ncl; ++c) cnt[c + 1] += cnt[c];
  int* order = (int*)malloc(sizeof(int) * (nloc > 0 ? nloc : 1));
  int* fill = (int*)calloc(ncl, sizeof(int));
  for (int ii = 0; ii < nloc; ++ii) {
    int c = cell_of[ii];
    order[cnt[c] + fill[c]++] = ii; /* ascending atom index within a cell */
  }
  /* count first (so nall is known even when it does not fit) */
  int total = nloc;
  int ii_[3], jj_[3], ps[3];
  for (ii_[0] = -ng[0]; ii_[0] < nc[0] + ng[0]; ++ii_[0])
    for (ii_[1] = -ng[1]; ii_[1] < nc[1] + ng[1]; ++ii_[1])
      for (ii_[2] = -ng[2]; ii_[2] < nc[2] + ng[2]; ++ii_[2]) {
        if (ii_[0] >= 0 && ii_[0] < nc[0] && ii_[1] >= 0 && ii_[1] < nc[1] &&
            ii_[2] >= 0 && ii_[2] < nc[2])
          continue;
        for (int dd = 0; dd < 3; ++dd)
          jj_[dd] = ii_[dd] + pbc_shift(ii_[dd], nc[dd]) * nc[dd];
        int c = (jj_[0] * nc[1] + jj_[1]) * nc[2] + jj_[2];
        total += cnt[c + 1] - cnt[c];
      }
  *nall = total;
  if (total > mem_nall) {
    free(cell_of); free(cnt); free(order); free(fill);
    return 1;
  }
  memcpy(out_c, in_c, sizeof(double) * 3 * (size_t)nloc);
  memcpy(out_t, in_t, sizeof(int) * (size_t)nloc);
  for (int ii = 0; ii < nloc; ++ii) mapping[ii] = ii;
  int w = nloc;
  for (ii_[0] = -ng[0]; ii_[0] < nc[0] + ng[0]; ++ii_[0])
    for (ii_[1] = -ng[1]; ii_[1] < nc[1] + ng[1]; ++ii_[1])
      for (ii_[2] = -ng[2]; ii_[2] < nc[2] + ng[2]; ++ii_[2]) {
        if (ii_[0] >= 0 && ii_[0] < nc[0] && ii_[1] >= 0 && ii_[1] < nc[1] &&
            ii_[2] >= 0 && ii_[2] < nc[2])
          continue;
        double psd[3], sv[3];
        for (int dd = 0; dd < 3; ++dd) {
          ps[dd] = pbc_shift(ii_[dd], nc[dd]);
          psd[dd] = ps[dd];
          jj_[dd] = ii_[dd] + ps[dd] * nc[dd];
        }
        tt_dot_v(sv, boxt, psd);
        int c = (jj_[0] * nc[1] + jj_[1]) * nc[2] + jj_[2];
        for (int k = cnt[c]; k < cnt[c + 1]; ++k) {
          int p = order[k];
          out_c[w * 3 + 0] = in_c[p * 3 + 0] - sv[0];
          out_c[w * 3 + 1] = in_c[p * 3 + 1] - sv[1];
          out_c[w * 3 + 2] = in_c[p * 3 + 2] - sv[2];
          out_t[w] = in_t[p];
          mapping[w] = p;
          w++;
        }
      }
  free(cell_of); free(cnt); free(order); free(fill);
  return 0;
}

/* ----------------------------------------------------- type-generic part -- */

#define ORC_DEFINE(T, SUF)                                                     \
  int orc_build_nlist_##SUF(int* ilist, int* numneigh, int* rowbuf,            \
                            int* max_list_size, const T* c, int nloc,          \
                            int nall, int mem_size, float rcut, int nframes,   \
                            const int* type) {                                 \
    /* neighbor_list.cc:875-928: diff = c_i - c_j, strict < (T)(rc*rc) */     \
    const float rc2f = rcut * rcut;                                            \
    const T rc2 = (T)rc2f;                                                     \
    *max_list_size = 0;                                                        \
    for (int ii = 0; ii < nframes * nloc; ++ii) {                              \
      int a = ii % nloc, f = ii / nloc, off = f * nall, n = 0;                 \
      ilist[ii] = a;                                                           \
      for (int jj = 0; jj < nall; ++jj) {                                      \
        if (jj == a) continue;                                                 \
        if (type && (type[off + a] < 0 || type[off + jj] < 0)) continue;       \
        T d0 = c[(off + a) * 3 + 0] - c[(off + jj) * 3 + 0];                   \
        T d1 = c[(off + a) * 3 + 1] - c[(off + jj) * 3 + 1];                   \
        T d2 = c[(off + a) * 3 + 2] - c[(off + jj) * 3 + 2];                   \
        T r2 = d0 * d0 + d1 * d1 + d2 * d2;                                    \
        if (r2 < rc2) {                                                        \
          if (n < mem_size) rowbuf[(size_t)ii * mem_size + n] = jj;            \
          n++;                                                                 \
        }                                                                      \
      }                                                                        \
      if (n > mem_size) {                                                      \
        *max_list_size = n;                                                    \
        return 1;                                                              \
      }                                                                        \
      numneigh[ii] = n;                                                        \
      if (n > *max_list_size) *max_list_size = n;                              \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_format_nlist_i_##SUF(int* fmt, const T* posi, const int* type,       \
                               int i_idx, const int* cand, int ncand,          \
                               float rcut, const int* sec, int nsec) {         \
    /* fmt_nlist.cc:98-143: keys (type, float r^2, index), float arithmetic */ \
    int nnei = sec[nsec - 1];                                                  \
    for (int k = 0; k < nnei; ++k) fmt[k] = -1;                                \
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (ncand + 1));        \
    int nk = 0;                                                                \
    const float rc2 = rcut * rcut;                                             \
    for (int k = 0; k < ncand; ++k) {                                          \
      int j = cand[k];                                                         \
      if (type[j] < 0) continue;                                               \
      float d0 = (float)posi[j * 3 + 0] - (float)posi[i_idx * 3 + 0];          \
      float d1 = (float)posi[j * 3 + 1] - (float)posi[i_idx * 3 + 1];          \
      float d2 = (float)posi[j * 3 + 2] - (float)posi[i_idx * 3 + 2];          \
      float r2 = d0 * d0 + d1 * d1 + d2 * d2;                                  \
      if (r2 <= rc2) {                                                         \
        uint32_t rb;                                                           \
        memcpy(&rb, &r2, 4);                                                   \
        /* (type, r^2 bits, index) compares like NeighborInfo::operator< for  \
         * non-negative floats; keys are kept in a 128-bit-free packing       \
         * because j < 2^24 and type < 128 are checked by the caller */       \
        keys[nk++] = ((uint64_t)type[j] << 56) | ((uint64_t)rb << 24) |        \
                     (uint64_t)j;                                              \
      }                                                                        \
    }                                                                          \
    /* insertion sort: candidate lists are short */                            \
    for (int a = 1; a < nk; ++a) {                                             \
      uint64_t v = keys[a];                                                    \
      int b = a - 1;                                                           \
      while (b >= 0 && keys[b] > v) {                                          \
        keys[b + 1] = keys[b];                                                 \
        b--;                                                                   \
      }                                                                        \
      keys[b + 1] = v;                                                         \
    }                                                                          \
    int* iter = (int*)malloc(sizeof(int) * nsec);                              \
    for (int t = 0; t < nsec; ++t) iter[t] = sec[t];                           \
    int overflowed = -1;                                                       \
    for (int k = 0; k < nk; ++k) {                                             \
      int t = (int)(keys[k] >> 56);                                            \
      int j = (int)(keys[k] & 0xFFFFFF);                                       \
      if (iter[t] < sec[t + 1]) fmt[iter[t]++] = j;                            \
      else overflowed = t;                                                     \
    }                                                                          \
    free(iter);                                                                \
    free(keys);                                                                \
    return overflowed;                                                         \
  }                                                                            \
                                                                               \
  static void spline5_##SUF(T* vv, T* dd, T xx, float rmin, float rmax) {      \
    /* source/lib/include/switcher.h:60-83 */                                  \
    if (xx < rmin) {                                                           \
      *dd = (T)0.;                                                             \
      *vv = (T)1.;                                                             \
    } else if (xx < rmax) {                                                    \
      T uu = (xx - rmin) / (rmax - rmin);                                      \
      T du = (T)1. / (rmax - rmin);                                            \
      *vv = uu * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) + (T)1.;  \
      *dd = ((T)3. * uu * uu * ((T)-6. * uu * uu + (T)15. * uu - (T)10.) +     \
             uu * uu * uu * ((T)-12. * uu + (T)15.)) *                         \
            du;                                                                \
    } else {                                                                   \
      *dd = (T)0.;                                                             \
      *vv = (T)0.;                                                             \
    }                                                                          \
  }                                                                            \
                                                                               \
  static void env_mat_a_##SUF(T* da, T* dd_, T* rij, const T* posi,            \
                              int i_idx, const int* fmt, const int* sec,       \
                              int nsec, float rmin, float rmax) {              \
    /* source/lib/src/env_mat.cc:123-209 */                                    \
    int nnei = sec[nsec - 1];                                                  \
    memset(rij, 0, sizeof(T) * nnei * 3);                                      \
    memset(da, 0, sizeof(T) * nnei * 4);                                       \
    memset(dd_, 0, sizeof(T) * nnei * 12);                                     \
    for (int s = 0; s < nsec - 1; ++s)                                         \
      for (int jj = sec[s]; jj < sec[s + 1]; ++jj) {                           \
        if (fmt[jj] < 0) break;                                                \
        int j = fmt[jj];                                                       \
        for (int d = 0; d < 3; ++d)                                            \
          rij[jj * 3 + d] = posi[j * 3 + d] - posi[i_idx * 3 + d];             \
      }                                                                        \
    for (int s = 0; s < nsec - 1; ++s)                                         \
      for (int jj = sec[s]; jj < sec[s + 1]; ++jj) {                           \
        if (fmt[jj] < 0) break;                                                \
        const T* rr = rij + jj * 3;                                            \
        T nr2 = rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2];                 \
        T inr = (T)1. / sqrt(nr2);                                             \
        T nr = nr2 * inr;                                                      \
        T inr2 = inr * inr;                                                    \
        T inr4 = inr2 * inr2;                                                  \
        T inr3 = inr4 * nr;                                                    \
        T sw, dsw;                                                             \
        spline5_##SUF(&sw, &dsw, nr, rmin, rmax);                              \
        T* v = da + jj * 4;                                                    \
        T* g = dd_ + jj * 12;                                                  \
        v[0] = (T)1. / nr;                                                     \
        v[1] = rr[0] / nr2;                                                    \
        v[2] = rr[1] / nr2;                                                    \
        v[3] = rr[2] / nr2;                                                    \
        for (int d = 0; d < 3; ++d)                                            \
          g[d] = rr[d] * inr3 * sw - v[0] * dsw * rr[d] * inr;                 \
        for (int a = 0; a < 3; ++a)                                            \
          for (int d = 0; d < 3; ++d) {                                        \
            T base = (T)2. * rr[a] * rr[d] * inr4;                             \
            if (a == d) base = base - inr2;                                    \
            g[3 + a * 3 + d] = base * sw - v[1 + a] * dsw * rr[d] * inr;       \
          }                                                                    \
        v[0] *= sw;                                                            \
        v[1] *= sw;                                                            \
        v[2] *= sw;                                                            \
        v[3] *= sw;                                                            \
      }                                                                        \
  }                                                                            \
                                                                               \
  int orc_prod_env_mat_a_##SUF(                                                \
      T* em, T* em_deriv, T* rij, int* nlist, const T* coord,                  \
      const int* type, int inum, const int* ilist, const int* numneigh,        \
      const int* rowbuf, int stride, const T* avg, const T* std_, int nloc,    \
      int nall, int nframes, float rcut, float rcut_smth, const int* sec,      \
      int nsec) {                                                              \
    /* source/lib/src/prod_env_mat.cc:14-133 */                                \
    int nnei = sec[nsec - 1], nem = nnei * 4;                                  \
    if (inum != nframes * nloc) return 2;                                      \
    int* fmt = (int*)malloc(sizeof(int) * (nnei + 1));                         \
    T* da = (T*)malloc(sizeof(T) * (nem + 1));                                 \
    T* dg = (T*)malloc(sizeof(T) * (nem * 3 + 1));                             \
    T* dr = (T*)malloc(sizeof(T) * (nnei * 3 + 1));                            \
    int** rows = (int**)calloc((size_t)nframes * nloc + 1, sizeof(int*));      \
    int* rown = (int*)calloc((size_t)nframes * nloc + 1, sizeof(int));         \
    for (int r = 0; r < inum; ++r) {                                           \
      int f = r / nloc, i = ilist[r];                                          \
      rows[(size_t)f * nloc + i] = (int*)(rowbuf + (size_t)r * stride);        \
      rown[(size_t)f * nloc + i] = numneigh[r];                                \
    }                                                                          \
    for (int row = 0; row < nframes * nloc; ++row) {                           \
      int f = row / nloc, ii = row % nloc;                                     \
      const T* fc = coord + (size_t)f * nall * 3;                              \
      const int* ft = type + (size_t)f * nall;                                 \
      orc_format_nlist_i_##SUF(fmt, fc, ft, ii, rows[row], rown[row], rcut,    \
                               sec, nsec);                                     \
      env_mat_a_##SUF(da, dg, dr, fc, ii, fmt, sec, nsec, rcut_smth, rcut);    \
      T* e = em + (size_t)row * nem;                                           \
      T* ed = em_deriv + (size_t)row * nem * 3;                                \
      for (int jj = 0; jj < nem; ++jj)                                         \
        e[jj] = ft[ii] >= 0 ? (da[jj] - avg[ft[ii] * nem + jj]) /              \
                                  std_[ft[ii] * nem + jj]                      \
                            : (T)0;                                            \
      for (int jj = 0; jj < nem * 3; ++jj)                                     \
        ed[jj] = ft[ii] >= 0 ? dg[jj] / std_[ft[ii] * nem + jj / 3] : (T)0;    \
      memcpy(rij + (size_t)row * nnei * 3, dr, sizeof(T) * nnei * 3);          \
      memcpy(nlist + (size_t)row * nnei, fmt, sizeof(int) * nnei);             \
    }                                                                          \
    free(fmt); free(da); free(dg); free(dr); free(rows); free(rown);           \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  static void locate_##SUF(T lower, T upper, T mx, T s0, T s1, T* xx,          \
                           int* idx, T* delta) {                               \
    /* source/lib/src/tabulate.cc:21-73 */                                     \
    T x0 = *xx;                                                                \
    *delta = (T)0.;                                                            \
    if (*xx < lower) {                                                         \
      *idx = 0;                                                                \
      *xx = (T)0.;                                                             \
      *delta = x0 - lower;                                                     \
    } else if (*xx < upper) {                                                  \
      *idx = (int)((*xx - lower) / s0);                                        \
      *xx -= (*idx * s0 + lower);                                              \
    } else if (*xx < mx) {                                                     \
      int first = (int)((upper - lower) / s0);                                 \
      *idx = first + (int)((*xx - upper) / s1);                                \
      *xx -= ((*idx - first) * s1 + upper);                                    \
    } else {                                                                   \
      int first = (int)((upper - lower) / s0);                                 \
      T bxx = (sizeof(T) == 8) ? (T)nextafter((double)mx, (double)lower)       \
                               : (T)nextafterf((float)mx, (float)lower);       \
      *idx = first + (int)((bxx - upper) / s1);                                \
      *xx = mx - ((*idx - first) * s1 + upper);                                \
      *delta = x0 - mx;                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  static int fold_start_##SUF(const T* em_x, const T* em, int ii, int nnei) {  \
    /* sorted-padding fold: first jj with em_x == em_x[last] and em[1..3]==0 \
     * (source/lib/src/tabulate.cc:184-189) */                                 \
    T ago = em_x[(size_t)ii * nnei + nnei - 1];                                \
    for (int jj = 0; jj < nnei; ++jj) {                                        \
      const T* l = em + ((size_t)ii * nnei + jj) * 4;                          \
      if (ago == em_x[(size_t)ii * nnei + jj] && l[1] == 0. && l[2] == 0. &&   \
          l[3] == 0.)                                                          \
        return jj;                                                             \
    }                                                                          \
    return nnei;                                                               \
  }                                                                            \
                                                                               \
  int orc_tabulate_fusion_se_a_##SUF(T* out, const T* table, const T* info,    \
                                     const T* em_x, const T* em, int nloc,     \
                                     int nnei, int M) {                        \
    /* source/lib/src/tabulate.cc:162-232 */                                   \
    memset(out, 0, sizeof(T) * (size_t)nloc * 4 * M);                          \
    if (nnei <= 0) return 0;                                                   \
    for (int ii = 0; ii < nloc; ++ii) {                                        \
      int brk = fold_start_##SUF(em_x, em, ii, nnei);                          \
      for (int jj = 0; jj < nnei && jj <= brk; ++jj) {                         \
        const T* l = em + ((size_t)ii * nnei + jj) * 4;                        \
        T xx = em_x[(size_t)ii * nnei + jj], dl;                               \
        int idx;                                                               \
        locate_##SUF(info[0], info[1], info[2], info[3], info[4], &xx, &idx,   \
                     &dl);                                                     \
        for (int m = 0; m < M; ++m) {                                          \
          const T* a = table + (size_t)idx * M * 6 + 6 * m;                    \
          T g = a[1] + ((T)2. * a[2] +                                         \
                        ((T)3. * a[3] + ((T)4. * a[4] + (T)5. * a[5] * xx) *   \
                                            xx) * xx) * xx;                    \
          T v = a[0] + (a[1] + (a[2] + (a[3] + (a[4] + a[5] * xx) * xx) *      \
                                           xx) * xx) * xx;                     \
          v = v + g * dl;                                                      \
          T sc = (jj == brk) ? (T)(nnei - jj) * v : v;                         \
          for (int k = 0; k < 4; ++k)                                          \
            out[(size_t)ii * 4 * M + k * M + m] += sc * l[k];                  \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_tabulate_fusion_se_a_grad_##SUF(                                     \
      T* dy_dem_x, T* dy_dem, const T* table, const T* info, const T* em_x,    \
      const T* em, const T* dy, int nloc, int nnei, int M) {                   \
    /* source/lib/src/tabulate.cc:234-341 */                                   \
    if (nnei <= 0) return 0;                                                   \
    memset(dy_dem_x, 0, sizeof(T) * (size_t)nloc * nnei);                      \
    memset(dy_dem, 0, sizeof(T) * (size_t)nloc * nnei * 4);                    \
    for (int ii = 0; ii < nloc; ++ii) {                                        \
      int brk = fold_start_##SUF(em_x, em, ii, nnei);                          \
      for (int jj = 0; jj < nnei && jj <= brk; ++jj) {                         \
        const T* l = em + ((size_t)ii * nnei + jj) * 4;                        \
        T* o = dy_dem + ((size_t)ii * nnei + jj) * 4;                          \
        T xx = em_x[(size_t)ii * nnei + jj], dl, grad = (T)0.;                 \
        int idx;                                                               \
        locate_##SUF(info[0], info[1], info[2], info[3], info[4], &xx, &idx,   \
                     &dl);                                                     \
        T rep = (jj == brk) ? (T)(nnei - jj) : (T)1.;                          \
        for (int m = 0; m < M; ++m) {                                          \
          const T* a = table + (size_t)idx * M * 6 + 6 * m;                    \
          T r[4];                                                              \
          for (int k = 0; k < 4; ++k) r[k] = dy[(size_t)ii * 4 * M + k * M + m]; \
          T g = a[1] + ((T)2. * a[2] +                                         \
                        ((T)3. * a[3] + ((T)4. * a[4] + (T)5. * a[5] * xx) *   \
                                            xx) * xx) * xx;                    \
          T v = a[0] + (a[1] + (a[2] + (a[3] + (a[4] + a[5] * xx) * xx) *      \
                                           xx) * xx) * xx;                     \
          v = v + g * dl;                                                      \
          T dot = l[0] * r[0] + l[1] * r[1] + l[2] * r[2] + l[3] * r[3];       \
          if (jj == brk) {                                                     \
            grad += g * dot * rep;                                             \
            for (int k = 0; k < 4; ++k) o[k] += v * r[k] * rep;                \
          } else {                                                             \
            grad += g * dot;                                                   \
            for (int k = 0; k < 4; ++k) o[k] += v * r[k];                      \
          }                                                                    \
        }                                                                      \
        dy_dem_x[(size_t)ii * nnei + jj] = grad;                               \
      }                                                                        \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_tabulate_fusion_se_a_grad_grad_##SUF(                                \
      T* dz_dy, const T* table, const T* info, const T* em_x, const T* em,     \
      const T* dz_dem_x, const T* dz_dem, int nloc, int nnei, int M) {         \
    /* source/lib/src/tabulate.cc:343-449 */                                   \
    memset(dz_dy, 0, sizeof(T) * (size_t)nloc * 4 * M);                        \
    if (nnei <= 0) return 0;                                                   \
    for (int ii = 0; ii < nloc; ++ii) {                                        \
      int brk = fold_start_##SUF(em_x, em, ii, nnei);                          \
      for (int jj = 0; jj < nnei && jj <= brk; ++jj) {                         \
        const T* l = em + ((size_t)ii * nnei + jj) * 4;                        \
        const T* h = dz_dem + ((size_t)ii * nnei + jj) * 4;                    \
        T xx = em_x[(size_t)ii * nnei + jj], dl;                               \
        T dzx = dz_dem_x[(size_t)ii * nnei + jj];                              \
        int idx;                                                               \
        locate_##SUF(info[0], info[1], info[2], info[3], info[4], &xx, &idx,   \
                     &dl);                                                     \
        T sc = (jj == brk) ? (T)(nnei - jj) : (T)1.;                           \
        for (int m = 0; m < M; ++m) {                                          \
          const T* a = table + (size_t)idx * M * 6 + 6 * m;                    \
          T g = a[1] + ((T)2. * a[2] +                                         \
                        ((T)3. * a[3] + ((T)4. * a[4] + (T)5. * a[5] * xx) *   \
                                            xx) * xx) * xx;                    \
          T v = a[0] + (a[1] + (a[2] + (a[3] + (a[4] + a[5] * xx) * xx) *      \
                                           xx) * xx) * xx;                     \
          v = v + g * dl;                                                      \
          for (int k = 0; k < 4; ++k)                                          \
            dz_dy[(size_t)ii * 4 * M + k * M + m] +=                           \
                sc * (v * h[k] + (dzx * g) * l[k]);                            \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_prod_force_a_##SUF(T* force, const T* nd, const T* ed,               \
                             const int* nlist, int nloc, int nall, int nnei,   \
                             int nframes) {                                    \
    /* source/lib/src/prod_force.cc:23-72 */                                   \
    int ndes = 4 * nnei;                                                       \
    memset(force, 0, sizeof(T) * (size_t)nframes * nall * 3);                  \
    for (int i = 0; i < nframes * nloc; ++i) {                                 \
      int f = i / nloc, a = i % nloc;                                          \
      size_t ci = (size_t)f * nall + a;                                        \
      for (int aa = 0; aa < ndes; ++aa)                                        \
        for (int d = 0; d < 3; ++d)                                            \
          force[ci * 3 + d] -=                                                 \
              nd[(size_t)i * ndes + aa] * ed[(size_t)i * ndes * 3 + aa * 3 + d]; \
      for (int jj = 0; jj < nnei; ++jj) {                                      \
        int j = nlist[(size_t)i * nnei + jj];                                  \
        if (j < 0) continue;                                                   \
        for (int aa = jj * 4; aa < jj * 4 + 4; ++aa)                           \
          for (int d = 0; d < 3; ++d)                                          \
            force[((size_t)f * nall + j) * 3 + d] +=                           \
                nd[(size_t)i * ndes + aa] *                                    \
                ed[(size_t)i * ndes * 3 + aa * 3 + d];                         \
      }                                                                        \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_prod_virial_a_##SUF(T* virial, T* atom_virial, const T* nd,          \
                              const T* ed, const T* rij, const int* nlist,     \
                              int nloc, int nall, int nnei) {                  \
    /* source/lib/src/prod_virial.cc:22-69 */                                  \
    int ndes = 4 * nnei;                                                       \
    for (int k = 0; k < 9; ++k) virial[k] = (T)0.;                             \
    memset(atom_virial, 0, sizeof(T) * 9 * (size_t)nall);                      \
    for (int i = 0; i < nloc; ++i)                                             \
      for (int jj = 0; jj < nnei; ++jj) {                                      \
        int j = nlist[(size_t)i * nnei + jj];                                  \
        if (j < 0) continue;                                                   \
        for (int aa = jj * 4; aa < jj * 4 + 4; ++aa) {                         \
          T pref = (T)-1.0 * nd[(size_t)i * ndes + aa];                        \
          for (int d0 = 0; d0 < 3; ++d0)                                       \
            for (int d1 = 0; d1 < 3; ++d1) {                                   \
              T tv = pref * rij[(size_t)i * nnei * 3 + jj * 3 + d1] *          \
                     ed[(size_t)i * ndes * 3 + aa * 3 + d0];                   \
              virial[d0 * 3 + d1] -= tv;                                       \
              atom_virial[(size_t)j * 9 + d0 * 3 + d1] -= tv;                  \
            }                                                                  \
        }                                                                      \
      }                                                                        \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_prod_force_grad_a_##SUF(T* gnet, const T* grad, const T* ed,         \
                                  const int* nlist, int nloc, int nnei,        \
                                  int nframes) {                               \
    /* source/lib/src/prod_force_grad.cc:22-70: minus the center term, plus  \
       the term of the slot's neighbor (index taken modulo nloc) */           \
    int ndes = 4 * nnei;                                                       \
    for (int i = 0; i < nframes * nloc; ++i) {                                 \
      int f = i / nloc;                                                        \
      for (int aa = 0; aa < ndes; ++aa) {                                      \
        const T* e = ed + ((size_t)i * ndes + aa) * 3;                         \
        T g = (T)0.;                                                           \
        for (int d = 0; d < 3; ++d) g -= grad[(size_t)i * 3 + d] * e[d];       \
        int j = nlist[(size_t)i * nnei + aa / 4];                              \
        if (j >= nloc) j = j % nloc;                                           \
        if (j >= 0)                                                            \
          for (int d = 0; d < 3; ++d)                                          \
            g += grad[((size_t)f * nloc + j) * 3 + d] * e[d];                  \
        gnet[(size_t)i * ndes + aa] = g;                                       \
      }                                                                        \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  int orc_prod_virial_grad_a_##SUF(T* gnet, const T* grad, const T* ed,        \
                                   const T* rij, const int* nlist, int nloc,   \
                                   int nnei) {                                 \
    /* source/lib/src/prod_virial_grad.cc:21-62 */                            \
    int ndes = 4 * nnei;                                                       \
    for (int i = 0; i < nloc; ++i)                                             \
      for (int aa = 0; aa < ndes; ++aa) {                                      \
        int jj = aa / 4;                                                       \
        T g = (T)0.;                                                           \
        if (nlist[(size_t)i * nnei + jj] >= 0) {                               \
          const T* e = ed + ((size_t)i * ndes + aa) * 3;                       \
          const T* r = rij + ((size_t)i * nnei + jj) * 3;                      \
          /* the reference's literal -1.0 is a double: in the FP32 build the  \
             product and the subtraction are done in double, then rounded */  \
          for (int d0 = 0; d0 < 3; ++d0)                                       \
            for (int d1 = 0; d1 < 3; ++d1)                                     \
              g = (T)((double)g - -1.0 * (double)grad[d0 * 3 + d1] *           \
                                      (double)r[d1] * (double)e[d0]);          \
        }                                                                      \
        gnet[(size_t)i * ndes + aa] = g;                                       \
      }                                                                        \
    return 0;                                                                  \
  }

ORC_DEFINE(double, f64)
ORC_DEFINE(float, f32)
