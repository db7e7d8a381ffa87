// Runs the deepmd:: GPU drop-ins of libdpb200.so through the REFERENCE's own
// headers (source/lib/include, compiled with GOOGLE_CUDA) and compares them
// with the reference's CPU functions (its CPU library compiled from its
// sources), the way the reference's unit tests compare GPU and CPU
// (source/lib/tests/test_env_mat_a.cc:960-1029, test_coord.cc,
// test_neighbor_list.cc, test_tabulate_se_a.cc, test_prod_force_a.cc,
// test_prod_virial_a.cc).
//
// Linking against the reference headers proves the mangled names, the
// InputNlist / Region layouts and the by-value std::vector<int> sec at run
// time. Input: a binary file (see read_input); output: one JSON line per
// precision with the largest differences, which tests/test_cxx_dropin_gpu.py
// checks.
//
//   dropin_harness <input.bin>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "coord.h"
#include "errors.h"
#include "neighbor_list.h"
#include "prod_env_mat.h"
#include "prod_force.h"
#include "prod_virial.h"
#include "region.h"
#include "tabulate.h"

namespace {

struct Input {
  int nloc = 0, ntypes = 0, M = 0, nspline = 0;
  float rcut = 0.f, rcut_smth = 0.f;
  std::vector<int> sec, type;
  std::vector<double> box, coord, avg, std_, info, table;
};

// int32 nloc, ntypes, M, nspline; float32 rcut, rcut_smth; int32 sec[ntypes+1];
// f64 box[9], coord[3 nloc]; int32 type[nloc]; f64 avg, std [ntypes * nnei * 4];
// f64 table_info[6], table[nspline * 6 M]
bool read_input(const char* path, Input& in) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  auto rd = [&](void* p, size_t sz, size_t n) { return std::fread(p, sz, n, f) == n; };
  int h[4];
  float r[2];
  bool ok = rd(h, 4, 4) && rd(r, 4, 2);
  if (ok) {
    in.nloc = h[0], in.ntypes = h[1], in.M = h[2], in.nspline = h[3];
    in.rcut = r[0], in.rcut_smth = r[1];
    in.sec.resize(in.ntypes + 1);
    ok = rd(in.sec.data(), 4, in.sec.size());
  }
  if (ok) {
    const int nnei = in.sec.back();
    in.box.resize(9);
    in.coord.resize(3 * in.nloc);
    in.type.resize(in.nloc);
    in.avg.resize((size_t)in.ntypes * nnei * 4);
    in.std_.resize(in.avg.size());
    in.info.resize(6);
    in.table.resize((size_t)in.nspline * 6 * in.M);
    ok = rd(in.box.data(), 8, 9) && rd(in.coord.data(), 8, in.coord.size()) &&
         rd(in.type.data(), 4, in.type.size()) && rd(in.avg.data(), 8, in.avg.size()) &&
         rd(in.std_.data(), 8, in.std_.size()) && rd(in.info.data(), 8, 6) &&
         rd(in.table.data(), 8, in.table.size());
  }
  std::fclose(f);
  return ok;
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

template <typename T>
T* dnew(size_t n) {
  T* p = nullptr;
  ck(cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)), "cudaMalloc");
  ck(cudaMemset(p, 0, sizeof(T) * (n ? n : 1)), "cudaMemset");
  return p;
}
template <typename T>
T* dput(const std::vector<T>& v) {
  T* p = dnew<T>(v.size());
  if (!v.empty()) ck(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice), "H2D");
  return p;
}
template <typename T>
std::vector<T> dget(const T* p, size_t n) {
  std::vector<T> v(n);
  if (n) ck(cudaMemcpy(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost), "D2H");
  return v;
}
template <typename A, typename B>
double maxdiff(const std::vector<A>& a, const std::vector<B>& b, size_t n) {
  double m = 0;
  for (size_t k = 0; k < n; ++k) m = std::max(m, std::fabs((double)a[k] - (double)b[k]));
  return m;
}

template <typename T>
void run(const Input& in, const char* name) {
  const int nloc = in.nloc, nnei = in.sec.back(), M = in.M;
  std::vector<T> box(in.box.begin(), in.box.end());
  std::vector<T> coord(in.coord.begin(), in.coord.end());
  std::vector<T> avg(in.avg.begin(), in.avg.end()), sd(in.std_.begin(), in.std_.end());
  std::vector<T> info(in.info.begin(), in.info.end()), table(in.table.begin(), in.table.end());

  // ------------------------------------------------------------ CPU path
  deepmd::Region<T> region;
  deepmd::init_region_cpu(region, box.data());
  std::vector<T> cn(coord);
  deepmd::normalize_coord_cpu(cn.data(), nloc, region);
  int mem_nall = nloc * 32, nall = 0;
  std::vector<T> c_cpu;
  std::vector<int> t_cpu, map_cpu;
  for (;;) {
    c_cpu.assign(3 * (size_t)mem_nall, 0);
    t_cpu.assign(mem_nall, 0);
    map_cpu.assign(mem_nall, 0);
    if (deepmd::copy_coord_cpu(c_cpu.data(), t_cpu.data(), map_cpu.data(), &nall, cn.data(),
                               in.type.data(), nloc, mem_nall, in.rcut, region) == 0)
      break;
    mem_nall *= 2;
  }
  const int mem_size = nall;
  std::vector<int> ilist(nloc), numneigh(nloc), jrows((size_t)nloc * mem_size);
  std::vector<int*> firstneigh(nloc);
  for (int ii = 0; ii < nloc; ++ii) firstneigh[ii] = &jrows[(size_t)ii * mem_size];
  deepmd::InputNlist cpu_nl(nloc, ilist.data(), numneigh.data(), firstneigh.data());
  int max_cpu = 0;
  deepmd::build_nlist_cpu(cpu_nl, &max_cpu, c_cpu.data(), nloc, nall, mem_size, in.rcut);
  std::vector<T> em(nloc * nnei * 4), emd(nloc * nnei * 12), rij(nloc * nnei * 3);
  std::vector<int> nlist(nloc * nnei);
  deepmd::prod_env_mat_a_cpu(em.data(), emd.data(), rij.data(), nlist.data(), c_cpu.data(),
                             t_cpu.data(), cpu_nl, max_cpu, avg.data(), sd.data(), nloc, nall,
                             in.rcut, in.rcut_smth, in.sec);
  // one table call per neighbor-type section, as se_a.py:826-832 does
  std::vector<std::vector<T>> xyz_cpu;
  std::vector<std::vector<T>> ex_s, em_s;
  for (int t = 0; t < in.ntypes; ++t) {
    const int a = in.sec[t], n = in.sec[t + 1] - a;
    std::vector<T> e((size_t)nloc * n * 4), x((size_t)nloc * n);
    for (int i = 0; i < nloc; ++i)
      for (int k = 0; k < n; ++k) {
        for (int c = 0; c < 4; ++c) e[((size_t)i * n + k) * 4 + c] = em[((size_t)i * nnei + a + k) * 4 + c];
        x[(size_t)i * n + k] = e[((size_t)i * n + k) * 4];
      }
    std::vector<T> out((size_t)nloc * 4 * M);
    deepmd::tabulate_fusion_se_a_cpu(out.data(), table.data(), info.data(), x.data(), e.data(),
                                     (const T*)nullptr, nloc, n, M);
    xyz_cpu.push_back(out);
    ex_s.push_back(x);
    em_s.push_back(e);
  }
  std::vector<T> nd((size_t)nloc * nnei * 4);
  for (size_t k = 0; k < nd.size(); ++k) nd[k] = (T)(0.1 * std::sin(0.37 * (double)k));
  std::vector<T> f_cpu(3 * (size_t)nall), v_cpu(9), av_cpu(9 * (size_t)nall);
  deepmd::prod_force_a_cpu(f_cpu.data(), nd.data(), emd.data(), nlist.data(), nloc, nall, nnei, 1);
  deepmd::prod_virial_a_cpu(v_cpu.data(), av_cpu.data(), nd.data(), emd.data(), rij.data(),
                            nlist.data(), nloc, nall, nnei);

  // ------------------------------------------------- GPU drop-ins (device)
  std::vector<T> box_info(18);
  std::copy(region.boxt, region.boxt + 9, box_info.begin());
  std::copy(region.rec_boxt, region.rec_boxt + 9, box_info.begin() + 9);
  T* d_box = dput(box_info);
  deepmd::Region<T> region_dev(d_box, d_box + 9);
  T* d_coord = dput(coord);
  int* d_type = dput(in.type);
  deepmd::normalize_coord_gpu(d_coord, nloc, region_dev);
  const double norm_err = maxdiff(dget(d_coord, 3 * (size_t)nloc), cn, 3 * (size_t)nloc);
  std::vector<int> cell_info(23);
  deepmd::compute_cell_info(cell_info.data(), in.rcut, region);
  const int lc = cell_info[21], tc = cell_info[22];
  int* d_cell_info = dput(cell_info);
  int* d_int_data = dnew<int>(4 * (size_t)nloc + 2 * (size_t)lc + 7 * (size_t)tc + 2);
  int gmem = nloc * 2, gnall = 0, ret = 1;
  T* d_c = nullptr;
  int *d_t = nullptr, *d_map = nullptr;
  int retries = 0;
  while (ret != 0) {
    if (d_c) cudaFree(d_c), cudaFree(d_t), cudaFree(d_map), gmem *= 2, ++retries;
    d_c = dnew<T>(3 * (size_t)gmem);
    d_t = dnew<int>(gmem);
    d_map = dnew<int>(gmem);
    ret = deepmd::copy_coord_gpu(d_c, d_t, d_map, &gnall, d_int_data, d_coord, d_type, nloc, gmem,
                                 lc, tc, d_cell_info, region_dev);
  }
  const bool ghost_equal = gnall == nall &&
                           maxdiff(dget(d_c, 3 * (size_t)nall), c_cpu, 3 * (size_t)nall) == 0 &&
                           dget(d_t, nall) == std::vector<int>(t_cpu.begin(), t_cpu.begin() + nall) &&
                           dget(d_map, nall) == std::vector<int>(map_cpu.begin(), map_cpu.begin() + nall);
  // build_nlist_gpu into device rows of width nall
  int* d_ilist = dnew<int>(nloc);
  int* d_numneigh = dnew<int>(nloc);
  int* d_jrows = dnew<int>((size_t)nloc * mem_size);
  std::vector<int*> fn_h(nloc);
  for (int ii = 0; ii < nloc; ++ii) fn_h[ii] = d_jrows + (size_t)ii * mem_size;
  int** d_firstneigh = dput(fn_h);
  deepmd::InputNlist gpu_nl(nloc, d_ilist, d_numneigh, d_firstneigh);
  int* d_nlist_data = dnew<int>(2 * (size_t)nloc * mem_size);
  int max_gpu = 0;
  const int bret = deepmd::build_nlist_gpu(gpu_nl, &max_gpu, d_nlist_data, d_c, nloc, nall,
                                           mem_size, in.rcut);
  // prod_env_mat_a_gpu (the overload without nframes, an inline forwarder of
  // the reference header)
  T* d_avg = dput(avg);
  T* d_std = dput(sd);
  T* d_em = dnew<T>(em.size());
  T* d_emd = dnew<T>(emd.size());
  T* d_rij = dnew<T>(rij.size());
  int* d_nlist = dnew<int>(nlist.size());
  int* d_array_int = dnew<int>(in.sec.size() + (size_t)nloc * in.sec.size() + nloc);
  unsigned long long* d_array_ll = dnew<unsigned long long>((size_t)nloc * 1024 * 2);
  deepmd::prod_env_mat_a_gpu(d_em, d_emd, d_rij, d_nlist, d_c, d_t, gpu_nl, d_array_int,
                             d_array_ll, mem_size, d_avg, d_std, nloc, nall, in.rcut,
                             in.rcut_smth, in.sec);
  const bool nlist_equal = dget(d_nlist, nlist.size()) == nlist;
  const double em_err = maxdiff(dget(d_em, em.size()), em, em.size());
  const double emd_err = maxdiff(dget(d_emd, emd.size()), emd, emd.size());
  const double rij_err = maxdiff(dget(d_rij, rij.size()), rij, rij.size());
  // the host list moved to the device by convert_nlist_gpu_device, then the
  // same env mat on it
  deepmd::InputNlist gpu_nl2;
  int* d_mem = dnew<int>((size_t)nloc * max_cpu);
  deepmd::convert_nlist_gpu_device(gpu_nl2, cpu_nl, d_mem, max_cpu);
  int* d_nlist2 = dnew<int>(nlist.size());
  deepmd::prod_env_mat_a_gpu(d_em, d_emd, d_rij, d_nlist2, d_c, d_t, gpu_nl2, d_array_int,
                             d_array_ll, max_cpu, d_avg, d_std, nloc, nall, in.rcut,
                             in.rcut_smth, in.sec);
  const bool converted_equal = dget(d_nlist2, nlist.size()) == nlist &&
                               maxdiff(dget(d_em, em.size()), em, em.size()) == em_err;
  deepmd::free_nlist_gpu_device(gpu_nl2);
  bool capacity_thrown = false;
  if (max_cpu > 1) {
    deepmd::InputNlist gpu_nl3;
    try {
      deepmd::convert_nlist_gpu_device(gpu_nl3, cpu_nl, d_mem, max_cpu - 1);
    } catch (const deepmd::deepmd_exception_nlist_capacity&) {
      capacity_thrown = gpu_nl3.ilist == nullptr;  // nothing allocated before the check
    }
  }
  // use_nlist_map with a permutation of the extended atoms
  std::vector<int> perm(nall);
  for (int k = 0; k < nall; ++k) perm[k] = (int)(((long long)k * 7919 + 13) % nall);
  int* d_perm = dput(perm);
  deepmd::use_nlist_map(d_nlist2, d_perm, nloc, nnei);
  std::vector<int> mapped = dget(d_nlist2, nlist.size());
  bool map_equal = true;
  for (size_t k = 0; k < nlist.size(); ++k)
    map_equal &= mapped[k] == (nlist[k] == -1 ? -1 : perm[nlist[k]]);
  // tabulate per section
  T* d_table = dput(table);
  double tab_err = 0;
  for (int t = 0; t < in.ntypes; ++t) {
    const int n = in.sec[t + 1] - in.sec[t];
    T* d_x = dput(ex_s[t]);
    T* d_e = dput(em_s[t]);
    T* d_out = dnew<T>((size_t)nloc * 4 * M);
    deepmd::tabulate_fusion_se_a_gpu(d_out, d_table, info.data(), d_x, d_e, (const T*)nullptr,
                                     nloc, n, M);
    tab_err = std::max(tab_err, maxdiff(dget(d_out, (size_t)nloc * 4 * M), xyz_cpu[t],
                                        (size_t)nloc * 4 * M));
    cudaFree(d_x), cudaFree(d_e), cudaFree(d_out);
  }
  // force and virial from the CPU env derivative (same inputs)
  T* d_nd = dput(nd);
  T* d_emd_c = dput(emd);
  T* d_rij_c = dput(rij);
  int* d_nl_c = dput(nlist);
  T* d_f = dnew<T>(3 * (size_t)nall);
  T* d_v = dnew<T>(9);
  T* d_av = dnew<T>(9 * (size_t)nall);
  deepmd::prod_force_a_gpu(d_f, d_nd, d_emd_c, d_nl_c, nloc, nall, nnei, 1);
  deepmd::prod_virial_a_gpu(d_v, d_av, d_nd, d_emd_c, d_rij_c, d_nl_c, nloc, nall, nnei);
  const double f_err = maxdiff(dget(d_f, 3 * (size_t)nall), f_cpu, 3 * (size_t)nall);
  const double v_err = maxdiff(dget(d_v, 9), v_cpu, 9);
  const double av_err = maxdiff(dget(d_av, 9 * (size_t)nall), av_cpu, 9 * (size_t)nall);
  double f_scale = 0, v_scale = 0;
  for (T x : f_cpu) f_scale = std::max(f_scale, std::fabs((double)x));
  for (T x : v_cpu) v_scale = std::max(v_scale, std::fabs((double)x));
  std::printf(
      "{\"precision\": \"%s\", \"nloc\": %d, \"nall\": %d, \"copy_retries\": %d, "
      "\"normalize_err\": %.3e, \"ghost_equal\": %s, \"build_ret\": %d, \"max_list\": [%d, %d], "
      "\"nlist_equal\": %s, \"em_err\": %.3e, \"em_deriv_err\": %.3e, \"rij_err\": %.3e, "
      "\"converted_equal\": %s, \"capacity_thrown\": %s, \"map_equal\": %s, "
      "\"tabulate_err\": %.3e, \"force_err\": %.3e, \"force_scale\": %.3e, "
      "\"virial_err\": %.3e, \"virial_scale\": %.3e, \"atom_virial_err\": %.3e}\n",
      name, nloc, nall, retries, norm_err, ghost_equal ? "true" : "false", bret, max_cpu,
      max_gpu, nlist_equal ? "true" : "false", em_err, emd_err, rij_err,
      converted_equal ? "true" : "false", capacity_thrown ? "true" : "false",
      map_equal ? "true" : "false", tab_err, f_err, f_scale, v_err, v_scale, av_err);
  std::fflush(stdout);
  for (void* p : {(void*)d_box, (void*)d_coord, (void*)d_type, (void*)d_cell_info,
                  (void*)d_int_data, (void*)d_c, (void*)d_t, (void*)d_map, (void*)d_ilist,
                  (void*)d_numneigh, (void*)d_jrows, (void*)d_firstneigh, (void*)d_nlist_data,
                  (void*)d_avg, (void*)d_std, (void*)d_em, (void*)d_emd, (void*)d_rij,
                  (void*)d_nlist, (void*)d_array_int, (void*)d_array_ll, (void*)d_mem,
                  (void*)d_nlist2, (void*)d_perm, (void*)d_table, (void*)d_nd, (void*)d_emd_c,
                  (void*)d_rij_c, (void*)d_nl_c, (void*)d_f, (void*)d_v, (void*)d_av})
    cudaFree(p);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <input.bin>\n", argv[0]);
    return 2;
  }
  Input in;
  if (!read_input(argv[1], in)) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  try {
    run<double>(in, "double");
    run<float>(in, "float");
  } catch (const deepmd::deepmd_exception& e) {
    std::fprintf(stderr, "deepmd_exception: %s\n", e.what());
    return 1;
  }
  return 0;
}
