// FP64 compression tables of the se_a embedding nets built on the device
// (the reference builds them on the host: deepmd/utils/tabulate.py:275-371
// with the network derivatives of deepmd/utils/tabulate_math.py).
//
//  k_emb_derivs : one block per grid point x: value, first and second
//                 x-derivative of every channel of one tanh embedding net by
//                 forward-mode differentiation, layer by layer in shared
//                 memory (one thread per output channel); a layer adds a
//                 residual when its width equals (x) or doubles ([x, x]) its
//                 input width (deepmd/dpmodel/utils/network.py:282-330).
//  k_hermite    : one thread per (interval, channel): the quintic matching
//                 value, slope and curvature at both ends of the interval
//                 (deepmd/utils/tabulate.py:306-349), stored as the six
//                 ascending-power coefficients of row r, channel m at
//                 table[r, 6 m + k] (source/lib/src/tabulate.cc:190-197).
#include "dpb_common.cuh"

namespace dpb {

constexpr int TB_MAXL = 8;     // layers
constexpr int TB_MAXW = 512;   // channels per layer
constexpr int TB_THREADS = 128;

struct EmbNet {
  const double* W[TB_MAXL];  // [n_in, n_out] row-major
  const double* b[TB_MAXL];  // [n_out]
  int width[TB_MAXL + 1];    // width[0] = 1
  int nlayers;
};

__global__ void __launch_bounds__(TB_THREADS)
k_emb_derivs(double* __restrict__ vv, double* __restrict__ dd, double* __restrict__ d2,
             const double* __restrict__ xx, EmbNet net) {
  __shared__ double sy[2][TB_MAXW], sdy[2][TB_MAXW], sd2[2][TB_MAXW];
  const int p = blockIdx.x;
  if (threadIdx.x == 0) {
    sy[0][0] = xx[p];
    sdy[0][0] = 1.0;
    sd2[0][0] = 0.0;
  }
  __syncthreads();
  int cur = 0;
  for (int l = 0; l < net.nlayers; ++l) {
    const int n_in = net.width[l], n_out = net.width[l + 1];
    const double* W = net.W[l];
    for (int c = threadIdx.x; c < n_out; c += blockDim.x) {
      double z = net.b[l][c], dz = 0.0, d2z = 0.0;
      for (int i = 0; i < n_in; ++i) {
        const double w = W[(size_t)i * n_out + c];
        z += sy[cur][i] * w;
        dz += sdy[cur][i] * w;
        d2z += sd2[cur][i] * w;
      }
      const double t = tanh(z);
      const double s = 1.0 - t * t;  // tanh'
      double y = t, dy = s * dz, d2y = s * d2z - 2.0 * t * s * dz * dz;
      if (n_out == n_in) {
        y += sy[cur][c];
        dy += sdy[cur][c];
        d2y += sd2[cur][c];
      } else if (n_out == 2 * n_in) {
        const int k = c % n_in;
        y += sy[cur][k];
        dy += sdy[cur][k];
        d2y += sd2[cur][k];
      }
      sy[cur ^ 1][c] = y;
      sdy[cur ^ 1][c] = dy;
      sd2[cur ^ 1][c] = d2y;
    }
    __syncthreads();
    cur ^= 1;
  }
  const int M = net.width[net.nlayers];
  for (int c = threadIdx.x; c < M; c += blockDim.x) {
    vv[(size_t)p * M + c] = sy[cur][c];
    dd[(size_t)p * M + c] = sdy[cur][c];
    d2[(size_t)p * M + c] = sd2[cur][c];
  }
}

__global__ void k_hermite(double* __restrict__ table, const double* __restrict__ vv,
                          const double* __restrict__ dd, const double* __restrict__ d2,
                          const double* __restrict__ steps, int nspline, int M) {
  const long long n = (long long)nspline * M;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n;
       o += (long long)gridDim.x * blockDim.x) {
    const long long r = o / M;
    const int m = (int)(o - r * M);
    const double h = steps[r];
    const double y0 = vv[r * M + m], y1 = vv[(r + 1) * M + m];
    const double g0 = dd[r * M + m], g1 = dd[(r + 1) * M + m];
    const double c0 = d2[r * M + m], c1 = d2[(r + 1) * M + m];
    const double dv = y1 - y0;
    const double h2 = h * h, h3 = h2 * h;
    double* out = table + r * 6 * M + 6 * m;
    out[0] = y0;
    out[1] = g0;
    out[2] = 0.5 * c0;
    out[3] = (20.0 * dv - (8.0 * g1 + 12.0 * g0) * h - (3.0 * c0 - c1) * h2) / (2.0 * h3);
    out[4] = (-30.0 * dv + (14.0 * g1 + 16.0 * g0) * h + (3.0 * c0 - 2.0 * c1) * h2) /
             (2.0 * h3 * h);
    out[5] = (12.0 * dv - 6.0 * (g1 + g0) * h + (c1 - c0) * h2) / (2.0 * h3 * h2);
  }
}

}  // namespace dpb

using namespace dpb;
extern "C" {

long long dpb_se_a_build_table_scratch_bytes(int npoints, int M) {
  if (npoints <= 0 || M <= 0) return 0;
  return 3LL * npoints * M * (long long)sizeof(double);
}

int dpb_se_a_build_table_f64(double* table, const double* xx, const double* steps, int npoints,
                             int nspline, const double* const* W, const double* const* b,
                             const int* widths, int nlayers, void* scratch,
                             long long scratch_bytes, dpb_stream_t stream) {
  if (nlayers < 1 || nlayers > TB_MAXL || nspline < 1 || npoints < nspline + 1 ||
      widths == nullptr || W == nullptr || b == nullptr || table == nullptr || xx == nullptr ||
      steps == nullptr) {
    set_error("se_a_build_table: invalid arguments (nlayers=%d npoints=%d nspline=%d)",
              nlayers, npoints, nspline);
    return DPB_ERR_INVALID;
  }
  EmbNet net{};
  net.nlayers = nlayers;
  net.width[0] = 1;
  if (widths[0] != 1) {
    set_error("se_a_build_table: the embedding net takes one input (widths[0]=%d)", widths[0]);
    return DPB_ERR_INVALID;
  }
  for (int l = 0; l < nlayers; ++l) {
    net.W[l] = W[l];
    net.b[l] = b[l];
    net.width[l + 1] = widths[l + 1];
    if (widths[l + 1] <= 0 || widths[l + 1] > TB_MAXW || W[l] == nullptr || b[l] == nullptr) {
      set_error("se_a_build_table: layer %d width %d outside [1, %d]", l, widths[l + 1],
                TB_MAXW);
      return DPB_ERR_INVALID;
    }
  }
  const int M = net.width[nlayers];
  const long long need = dpb_se_a_build_table_scratch_bytes(npoints, M);
  if (scratch == nullptr || scratch_bytes < need) {
    set_error("se_a_build_table: scratch of %lld bytes is smaller than %lld", scratch_bytes,
              need);
    return DPB_ERR_INVALID;
  }
  double* vv = reinterpret_cast<double*>(scratch);
  double* dd = vv + (size_t)npoints * M;
  double* d2 = dd + (size_t)npoints * M;
  cudaStream_t st = as_stream(stream);
  k_emb_derivs<<<npoints, TB_THREADS, 0, st>>>(vv, dd, d2, xx, net);
  DPB_CHECK_LAUNCH("se_a_build_table/derivatives");
  k_hermite<<<grid_stride_blocks((long long)nspline * M, 256), 256, 0, st>>>(table, vv, dd, d2,
                                                                           steps, nspline, M);
  DPB_CHECK_LAUNCH("se_a_build_table/hermite");
  return DPB_OK;
}

}  // extern "C"
