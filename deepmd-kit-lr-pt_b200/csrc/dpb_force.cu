// Force and virial assembly from the network derivative (prod_force_a /
// prod_virial_a).
//
// One warp per center atom, one lane per neighbor slot: the lane contracts the
// slot's 4 net_deriv values with its 4x3 em_deriv block into the pair force
// f_jj = sum_a nd[a] * ed[a, :]. The center force is -sum_jj f_jj (a warp
// butterfly, no atomics), the neighbor gets +f_jj (one atomic per component),
// and the pair virial f_jj (x) rij is reduced per block (warps stride over
// the center atoms) before one atomic per component. References: source/lib/src/prod_force.cc:23-72 and
// source/lib/src/prod_virial.cc:22-69 (sign conventions included).
#include "dpb_common.cuh"

namespace dpb {

constexpr int FW = 4;

template <typename T>
__global__ void __launch_bounds__(FW * 32)
k_prod_force(T* __restrict__ force, const T* __restrict__ nd,
             const T* __restrict__ ed, const int* __restrict__ nlist, int nloc,
             int nall, int nnei, int nrows) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * FW + w;
  if (row >= nrows) return;
  const int f = row / nloc, i = row % nloc;
  T* ff = force + (size_t)f * nall * 3;
  const T* ndr = nd + (size_t)row * nnei * 4;
  const T* edr = ed + (size_t)row * nnei * 12;
  T c0 = (T)0., c1 = (T)0., c2 = (T)0.;
  for (int jj = lane; jj < nnei; jj += 32) {
    T p[3] = {(T)0., (T)0., (T)0.};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const T n = ndr[jj * 4 + a];
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += n * edr[(jj * 4 + a) * 3 + d];
    }
    c0 += p[0];
    c1 += p[1];
    c2 += p[2];
    const int j = nlist[(size_t)row * nnei + jj];
    if (j >= 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) atomic_add(&ff[(size_t)j * 3 + d], p[d]);
    }
  }
  c0 = warp_sum(c0);
  c1 = warp_sum(c1);
  c2 = warp_sum(c2);
  if (lane == 0) {
    atomic_add(&ff[(size_t)i * 3 + 0], -c0);
    atomic_add(&ff[(size_t)i * 3 + 1], -c1);
    atomic_add(&ff[(size_t)i * 3 + 2], -c2);
  }
}

template <typename T>
__global__ void __launch_bounds__(FW * 32)
k_prod_virial(T* __restrict__ virial, T* __restrict__ atom_virial,
              const T* __restrict__ nd, const T* __restrict__ ed,
              const T* __restrict__ rij, const int* __restrict__ nlist,
              int nloc, int nnei) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T vs[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) vs[k] = (T)0.;
  for (int i = blockIdx.x * FW + w; i < nloc; i += gridDim.x * FW) {
  const T* ndr = nd + (size_t)i * nnei * 4;
  const T* edr = ed + (size_t)i * nnei * 12;
  const T* rr = rij + (size_t)i * nnei * 3;
  for (int jj = lane; jj < nnei; jj += 32) {
    const int j = nlist[(size_t)i * nnei + jj];
    if (j < 0) continue;
    T p[3] = {(T)0., (T)0., (T)0.};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const T n = ndr[jj * 4 + a];
#pragma unroll
      for (int d = 0; d < 3; ++d) p[d] += n * edr[(jj * 4 + a) * 3 + d];
    }
    const T r[3] = {rr[jj * 3 + 0], rr[jj * 3 + 1], rr[jj * 3 + 2]};
#pragma unroll
    for (int d0 = 0; d0 < 3; ++d0)
#pragma unroll
      for (int d1 = 0; d1 < 3; ++d1) {
        const T v = p[d0] * r[d1];
        vs[d0 * 3 + d1] += v;
        atomic_add(&atom_virial[(size_t)j * 9 + d0 * 3 + d1], v);
      }
  }
  }
  block_add9<FW>(vs, virial);
}

// Adjoints of prod_force_a / prod_virial_a with respect to net_deriv (the TF
// path's second derivatives), one thread per (row, descriptor element):
//   force:  g[i,a] = -sum_d grad[i,d] ed[i,a,d]
//                    + sum_d grad[f, j mod nloc, d] ed[i,a,d]   (slot a/4 -> j >= 0)
//   virial: g[i,a] = sum_{d0,d1} grad[d0,d1] rij[i,a/4,d1] ed[i,a,d0]   (j >= 0)
// with the reference's operation order (prod_force_grad.cc:22-70,
// prod_virial_grad.cc:21-62).
template <typename T>
__global__ void k_prod_force_grad(T* __restrict__ gnet, const T* __restrict__ grad,
                                  const T* __restrict__ ed, const int* __restrict__ nlist,
                                  int nloc, int nnei, long long n) {
  const int ndescrpt = nnei * 4;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    const long long row = o / ndescrpt;
    const int a = (int)(o - row * ndescrpt);
    const T* e = ed + o * 3;
    T g = (T)0.;
#pragma unroll
    for (int d = 0; d < 3; ++d) g -= grad[row * 3 + d] * e[d];
    int j = nlist[row * nnei + a / 4];
    if (j >= nloc) j = j % nloc;
    if (j >= 0) {
      const long long f = row / nloc;
#pragma unroll
      for (int d = 0; d < 3; ++d) g += grad[(f * nloc + j) * 3 + d] * e[d];
    }
    gnet[o] = g;
  }
}

template <typename T>
__global__ void k_prod_virial_grad(T* __restrict__ gnet, const T* __restrict__ grad,
                                   const T* __restrict__ ed, const T* __restrict__ rij,
                                   const int* __restrict__ nlist, int nnei, long long n) {
  const int ndescrpt = nnei * 4;
  T gv[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) gv[k] = grad[k];
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    const long long row = o / ndescrpt;
    const int a = (int)(o - row * ndescrpt);
    const int jj = a / 4;
    T g = (T)0.;
    if (nlist[row * nnei + jj] >= 0) {
      const T* e = ed + o * 3;
      const T* r = rij + (row * nnei + jj) * 3;
      // the reference's literal -1.0 is a double: in the FP32 build the
      // product and the subtraction are done in double, then rounded
#pragma unroll
      for (int d0 = 0; d0 < 3; ++d0)
#pragma unroll
        for (int d1 = 0; d1 < 3; ++d1)
          g = (T)((double)g - -1.0 * (double)gv[d0 * 3 + d1] * (double)r[d1] * (double)e[d0]);
    }
    gnet[o] = g;
  }
}

template <typename T>
static int prod_force_grad(T* gnet, const T* grad, const T* ed, const int* nlist, int nloc,
                           int nnei, int nframes, cudaStream_t st) {
  if (nloc < 0 || nnei < 0 || nframes < 1) {
    set_error("prod_force_grad_a: invalid sizes (nloc=%d nnei=%d nframes=%d)", nloc, nnei,
              nframes);
    return DPB_ERR_INVALID;
  }
  const long long n = (long long)nframes * nloc * nnei * 4;
  if (n == 0) return DPB_OK;
  k_prod_force_grad<T><<<grid_stride_blocks(n, 256), 256, 0, st>>>(gnet, grad, ed, nlist,
                                                                   nloc, nnei, n);
  DPB_CHECK_LAUNCH("prod_force_grad_a");
  return DPB_OK;
}

template <typename T>
static int prod_virial_grad(T* gnet, const T* grad, const T* ed, const T* rij,
                            const int* nlist, int nloc, int nnei, cudaStream_t st) {
  if (nloc < 0 || nnei < 0) {
    set_error("prod_virial_grad_a: invalid sizes (nloc=%d nnei=%d)", nloc, nnei);
    return DPB_ERR_INVALID;
  }
  const long long n = (long long)nloc * nnei * 4;
  if (n == 0) return DPB_OK;
  k_prod_virial_grad<T><<<grid_stride_blocks(n, 256), 256, 0, st>>>(gnet, grad, ed, rij,
                                                                    nlist, nnei, n);
  DPB_CHECK_LAUNCH("prod_virial_grad_a");
  return DPB_OK;
}

template <typename T>
static int prod_force(T* force, const T* nd, const T* ed, const int* nlist,
                      int nloc, int nall, int nnei, int nframes, cudaStream_t st) {
  if (nloc < 0 || nall < nloc || nnei < 0 || nframes < 1) {
    set_error("prod_force_a: invalid sizes (nloc=%d nall=%d nnei=%d nframes=%d)", nloc,
              nall, nnei, nframes);
    return DPB_ERR_INVALID;
  }
  if (nall > 0)
    DPB_CUDA(cudaMemsetAsync(force, 0, sizeof(T) * (size_t)nframes * nall * 3, st),
             "prod_force_a");
  const int rows = nframes * nloc;
  if (rows == 0 || nnei == 0) return DPB_OK;
  k_prod_force<T><<<ceil_div(rows, FW), FW * 32, 0, st>>>(force, nd, ed, nlist, nloc,
                                                          nall, nnei, rows);
  DPB_CHECK_LAUNCH("prod_force_a");
  return DPB_OK;
}

template <typename T>
static int prod_virial(T* virial, T* atom_virial, const T* nd, const T* ed,
                       const T* rij, const int* nlist, int nloc, int nall,
                       int nnei, cudaStream_t st) {
  if (nloc < 0 || nall < nloc || nnei < 0) {
    set_error("prod_virial_a: invalid sizes (nloc=%d nall=%d nnei=%d)", nloc, nall, nnei);
    return DPB_ERR_INVALID;
  }
  DPB_CUDA(cudaMemsetAsync(virial, 0, sizeof(T) * 9, st), "prod_virial_a");
  if (nall > 0)
    DPB_CUDA(cudaMemsetAsync(atom_virial, 0, sizeof(T) * 9 * (size_t)nall, st),
             "prod_virial_a");
  if (nloc == 0 || nnei == 0) return DPB_OK;
  k_prod_virial<T><<<grid_stride_blocks(nloc, FW), FW * 32, 0, st>>>(virial, atom_virial, nd, ed,
                                                           rij, nlist, nloc, nnei);
  DPB_CHECK_LAUNCH("prod_virial_a");
  return DPB_OK;
}

}  // namespace dpb

using namespace dpb;
extern "C" {

int dpb_prod_force_a_f64(double* force, const double* net_deriv,
                         const double* in_deriv, const int* nlist, int nloc,
                         int nall, int nnei, int nframes, dpb_stream_t stream) {
  return prod_force<double>(force, net_deriv, in_deriv, nlist, nloc, nall, nnei,
                            nframes, as_stream(stream));
}

int dpb_prod_force_a_f32(float* force, const float* net_deriv,
                         const float* in_deriv, const int* nlist, int nloc,
                         int nall, int nnei, int nframes, dpb_stream_t stream) {
  return prod_force<float>(force, net_deriv, in_deriv, nlist, nloc, nall, nnei,
                           nframes, as_stream(stream));
}

int dpb_prod_virial_a_f64(double* virial, double* atom_virial,
                          const double* net_deriv, const double* env_deriv,
                          const double* rij, const int* nlist, int nloc,
                          int nall, int nnei, dpb_stream_t stream) {
  return prod_virial<double>(virial, atom_virial, net_deriv, env_deriv, rij,
                             nlist, nloc, nall, nnei, as_stream(stream));
}

int dpb_prod_virial_a_f32(float* virial, float* atom_virial,
                          const float* net_deriv, const float* env_deriv,
                          const float* rij, const int* nlist, int nloc,
                          int nall, int nnei, dpb_stream_t stream) {
  return prod_virial<float>(virial, atom_virial, net_deriv, env_deriv, rij,
                            nlist, nloc, nall, nnei, as_stream(stream));
}

int dpb_prod_force_grad_a_f64(double* grad_net, const double* grad, const double* env_deriv,
                              const int* nlist, int nloc, int nnei, int nframes,
                              dpb_stream_t stream) {
  return prod_force_grad<double>(grad_net, grad, env_deriv, nlist, nloc, nnei, nframes,
                                 as_stream(stream));
}

int dpb_prod_force_grad_a_f32(float* grad_net, const float* grad, const float* env_deriv,
                              const int* nlist, int nloc, int nnei, int nframes,
                              dpb_stream_t stream) {
  return prod_force_grad<float>(grad_net, grad, env_deriv, nlist, nloc, nnei, nframes,
                                as_stream(stream));
}

int dpb_prod_virial_grad_a_f64(double* grad_net, const double* grad, const double* env_deriv,
                               const double* rij, const int* nlist, int nloc, int nnei,
                               dpb_stream_t stream) {
  return prod_virial_grad<double>(grad_net, grad, env_deriv, rij, nlist, nloc, nnei,
                                  as_stream(stream));
}

int dpb_prod_virial_grad_a_f32(float* grad_net, const float* grad, const float* env_deriv,
                               const float* rij, const int* nlist, int nloc, int nnei,
                               dpb_stream_t stream) {
  return prod_virial_grad<float>(grad_net, grad, env_deriv, rij, nlist, nloc, nnei,
                                 as_stream(stream));
}

}  // extern "C"
