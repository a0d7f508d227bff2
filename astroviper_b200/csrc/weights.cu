// Natural / Briggs imaging weights (grid_imaging_weights.py:93-206, :285-443;
// briggs_weighting.py:1-31; the input preparation of
// calculate_imaging_weights.py:183-198, 228-261).
#include <math_constants.h>

#include <mutex>

#include "common.cuh"

namespace av {

// Polarisation-averaged weight of a sample, NaN where flagged
// (calculate_imaging_weights.py:185-198).
__device__ __forceinline__ double pol_avg_weight(const void *wt, int dt, const uint8_t *flag,
                                                 int64_t row, int64_t npol) {
  auto w = [&](int64_t p) {
    int64_t i = row * npol + p;
    double v = dt == AV_F32 ? (double)((const float *)wt)[i] : ((const double *)wt)[i];
    if (flag && flag[i]) v = CUDART_NAN;
    return v;
  };
  if (npol == 2) return __ddiv_rn(__dadd_rn(w(0), w(1)), 2.0);
  if (npol == 4) return __ddiv_rn(__dadd_rn(w(0), w(3)), 2.0);
  return w(0);
}

// Nearest cell of a sample in the gridder's convention (int(x + 0.5)).
__device__ __forceinline__ bool nearest_cell(double um, double vm, double f, double dl0,
                                             double dl1, int64_t n_u, int64_t n_v,
                                             long long &ui, long long &vi, long long &uic,
                                             long long &vic) {
  double us0 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, dl0), (double)n_u), C_LIGHT);
  double us1 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, dl1), (double)n_v), C_LIGHT);
  double u = __dmul_rn(um, us0), v = __dmul_rn(vm, us1);
  if (isnan(u) || isnan(v)) return false;
  double u_pos = __dadd_rn(u, (double)(n_u / 2)), v_pos = __dadd_rn(v, (double)(n_v / 2));
  double u_pc = __dadd_rn(-u, (double)(n_u / 2)), v_pc = __dadd_rn(-v, (double)(n_v / 2));
  ui = trunc_ll(__dadd_rn(u_pos, 0.5));
  vi = trunc_ll(__dadd_rn(v_pos, 0.5));
  uic = trunc_ll(__dadd_rn(u_pc, 0.5));
  vic = trunc_ll(__dadd_rn(v_pc, 0.5));
  return (ui < n_u) && (vi < n_v) && (ui >= 0) && (vi >= 0);
}

// Density grid: rows enumerated channel-major so a warp shares a channel and
// its sum_weight contribution is reduced before one atomic.
__global__ void __launch_bounds__(256) k_weight_density(double *G, double *sumw,
                                                        const double *uvw, const double *freq,
                                                        const void *wt, int dt,
                                                        const uint8_t *flag, int64_t n_u,
                                                        int64_t n_v, double dl0, double dl1,
                                                        int64_t ntb, int64_t nchan,
                                                        int64_t npol) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t total = ntb * nchan;
  double add = 0.0;
  int64_t c = -1;
  if (k < total) {
    c = k / ntb;
    int64_t tb = k - c * ntb;
    long long ui, vi, uic, vic;
    if (nearest_cell(uvw[3 * tb], uvw[3 * tb + 1], freq[c], dl0, dl1, n_u, n_v, ui, vi, uic,
                     vic)) {
      double w = pol_avg_weight(wt, dt, flag, tb * nchan + c, npol);
      if (!isnan(w)) {
        double *plane = G + c * n_u * n_v;
        atomicAdd(&plane[ui * n_v + vi], w);
        // the conjugate cell is not range-checked by the reference; it is out
        // of range only for index 0 of an even axis, skipped here
        if (uic >= 0 && uic < n_u && vic >= 0 && vic < n_v) atomicAdd(&plane[uic * n_v + vic], w);
        add = __dmul_rn(2.0, w);
      }
    }
  }
  // lanes of a warp span at most two channels: the leader of each channel
  // group sums the group's contributions and issues one atomic
  int lane = threadIdx.x & 31;
  unsigned m = __match_any_sync(0xffffffffu, (unsigned)(c + 1));
  double tot = 0.0;
  for (int l = 0; l < 32; ++l) {
    double y = __shfl_sync(0xffffffffu, add, l);
    if ((m >> l) & 1u) tot += y;
  }
  if (lane == __ffs(m) - 1 && c >= 0 && tot != 0.0) atomicAdd(&sumw[c], tot);
}

// sum(G^2) per plane: one CTA per (plane, slice), FP64 partials.
__global__ void __launch_bounds__(256) k_sum_sq(const double *G, int64_t plane_n,
                                                int slices, double *partial) {
  int64_t p = blockIdx.x / slices;
  int s = blockIdx.x - (int)p * slices;
  int64_t lo = plane_n * s / slices, hi = plane_n * (s + 1) / slices;
  const double *g = G + p * plane_n;
  double acc = 0.0;
  for (int64_t i0 = lo; i0 < hi; i0 += blockDim.x) {  // one trip count per block
    const int64_t i = i0 + threadIdx.x;
    if (i < hi) {
      double v = g[i];
      acc += v * v;
    }
  }
  __shared__ double sh[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void k_briggs_finish(const double *partial, int slices, const double *sumw,
                                int64_t nplanes, double robust, double *factors) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nplanes) return;
  double sq = 0.0;
  for (int s = 0; s < slices; ++s) sq += partial[p * slices + s];
  double r = 5.0 * pow(10.0, -robust);
  // (5 * 10^-R)^2 / (sum G^2 / sum w): NaN / inf pass through like numpy
  factors[p] = (r * r) / (sq / sumw[p]);
  factors[nplanes + p] = 1.0;
}

// Imaging weight of each sample, tiled to every polarisation
// (grid_imaging_weights.py:358-443 + calculate_imaging_weights.py:258-261).
__global__ void __launch_bounds__(256) k_briggs_apply(void *out, int out_dt, const double *G,
                                                      const double *factors, int64_t nplanes,
                                                      const double *uvw, const double *freq,
                                                      const void *wt, int dt,
                                                      const uint8_t *flag, int64_t n_u,
                                                      int64_t n_v, double dl0, double dl1,
                                                      int64_t nrows, int64_t nchan,
                                                      int64_t npol, int *err) {
  int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  int64_t tb = row / nchan, c = row - tb * nchan;
  double iw = 0.0;  // off-grid samples keep the zero the reference allocates
  long long ui, vi, uic, vic;
  if (nearest_cell(uvw[3 * tb], uvw[3 * tb + 1], freq[c], dl0, dl1, n_u, n_v, ui, vi, uic,
                   vic)) {
    double dw = pol_avg_weight(wt, dt, flag, row, npol);
    iw = dw;
    if (!isnan(dw) && dw != 0.0) {
      double gij = G[(c * n_u + ui) * n_v + vi];
      if (!isnan(gij) && gij != 0.0) {
        double f0 = factors[c], f1 = factors[nplanes + c];
        if (isnan(f0) || isnan(f1)) {
          atomicExch(err, 1);
        } else {
          double denom = __dadd_rn(__dmul_rn(f0, gij), f1);
          iw = __ddiv_rn(iw, denom);
        }
      }
    }
  }
  for (int64_t p = 0; p < npol; ++p) {
    if (out_dt == AV_F64) ((double *)out)[row * npol + p] = iw;
    else ((float *)out)[row * npol + p] = (float)iw;
  }
}

// standard_imaging_weight_degrid_jit (standard_grid.py:487-604), one thread
// per (time, baseline, channel): for a sample whose nearest cell (gridder
// convention) is on the grid, every polarisation's weight becomes its
// natural weight (the mean of polarisations 0 and 1 when there are two),
// divided by f0 * G + f1 where both the polarisation's own natural weight
// and G, the imaging-weight grid of (chan_map[c], pol_map[p]) at that cell,
// are neither NaN nor zero.  Samples off the grid (or with NaN uv) are left
// as the caller's array holds them.
__global__ void __launch_bounds__(256) k_imaging_weight_degrid(
    double *out, const void *G, int g_dt, int64_t g_chan, int64_t g_pol, const double *factors,
    const double *uvw, const double *freq, const int32_t *chan_map, const int32_t *pol_map,
    const void *wt, int dt, int64_t n_u, int64_t n_v, double dl0, double dl1, int64_t nrows,
    int64_t nchan, int64_t npol) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int64_t tb = row / nchan, c = row - tb * nchan;
  long long ui, vi, uic, vic;
  if (!nearest_cell(uvw[3 * tb], uvw[3 * tb + 1], freq[c], dl0, dl1, n_u, n_v, ui, vi, uic,
                    vic))
    return;
  auto w = [&](int64_t p) {
    const int64_t i = row * npol + p;
    return dt == AV_F32 ? (double)((const float *)wt)[i] : ((const double *)wt)[i];
  };
  const int64_t ac = chan_map[c];
  for (int64_t p = 0; p < npol; ++p) {
    const int64_t ap = pol_map[p];
    double iw = npol == 2 ? __ddiv_rn(__dadd_rn(w(0), w(1)), 2.0) : w(p);
    const double nat = w(p);
    if (!isnan(nat) && nat != 0.0) {
      const int64_t gi = ((ac * g_pol + ap) * n_u + ui) * n_v + vi;
      const double g =
          g_dt == AV_F32 ? (double)((const float *)G)[gi] : ((const double *)G)[gi];
      if (!isnan(g) && g != 0.0) {
        const int64_t fi = ac * g_pol + ap;
        const double den = __dadd_rn(__dmul_rn(factors[fi], g), factors[g_chan * g_pol + fi]);
        iw = __ddiv_rn(iw, den);
      }
    }
    out[row * npol + p] = iw;
  }
}

}  // namespace av

using namespace av;

extern "C" {

int av_weight_density(double *density, double *sum_weight, const double *uvw,
                      const double *freq, const void *wt, int wt_dtype, const uint8_t *flag,
                      int64_t n_u, int64_t n_v, double delta_l, double delta_m, int64_t nt,
                      int64_t nb, int64_t nchan, int64_t npol, void *stream) {
  clear_error();
  AV_CHECK_ARG(density && sum_weight && uvw && freq && wt, "av_weight_density: null pointer");
  AV_CHECK_ARG(wt_dtype == AV_F32 || wt_dtype == AV_F64, "av_weight_density: weight dtype");
  AV_CHECK_ARG(npol == 1 || npol == 2 || npol == 4, "av_weight_density: npol must be 1, 2 or 4");
  AV_CHECK_ARG(n_u > 0 && n_v > 0 && nt >= 0 && nb >= 0 && nchan >= 0,
               "av_weight_density: bad shape");
  int64_t total = nt * nb * nchan;
  if (total == 0) return AV_OK;
  k_weight_density<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      density, sum_weight, uvw, freq, wt, wt_dtype, flag, n_u, n_v, delta_l, delta_m, nt * nb,
      nchan, npol);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_briggs_factors_workspace_size(int64_t nplanes) {
  return Workspace::need(sizeof(double) * (size_t)nplanes * 64);
}

int av_briggs_factors(const double *density, const double *sum_weight, double *factors,
                         int64_t nplanes, int64_t n_u, int64_t n_v, double robust,
                         void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(density && sum_weight && factors, "av_briggs_factors: null pointer");
  AV_CHECK_ARG(nplanes >= 0 && n_u > 0 && n_v > 0, "av_briggs_factors: bad shape");
  if (nplanes == 0) return AV_OK;
  const int slices = 64;
  if (!workspace || workspace_bytes < av_briggs_factors_workspace_size(nplanes)) {
    set_error("av_briggs_factors: workspace too small");
    return AV_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  double *partial = (double *)workspace;
  k_sum_sq<<<(unsigned)(nplanes * slices), 256, 0, st>>>(density, n_u * n_v, slices, partial);
  AV_LAUNCH_CHECK();
  k_briggs_finish<<<(unsigned)((nplanes + 127) / 128), 128, 0, st>>>(partial, slices,
                                                                      sum_weight, nplanes,
                                                                      robust, factors);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_briggs_apply(void *out, int out_dtype, const double *density, const double *factors,
                    const double *uvw, const double *freq, const void *wt, int wt_dtype,
                    const uint8_t *flag, int64_t n_u, int64_t n_v, double delta_l,
                    double delta_m, int64_t nt, int64_t nb, int64_t nchan, int64_t npol,
                    int32_t *err_flag, void *stream) {
  clear_error();
  AV_CHECK_ARG(out && density && factors && uvw && freq && wt && err_flag,
               "av_briggs_apply: null pointer");
  AV_CHECK_ARG(out_dtype == AV_F32 || out_dtype == AV_F64, "av_briggs_apply: out dtype");
  AV_CHECK_ARG(wt_dtype == AV_F32 || wt_dtype == AV_F64, "av_briggs_apply: weight dtype");
  AV_CHECK_ARG(npol == 1 || npol == 2 || npol == 4, "av_briggs_apply: npol must be 1, 2 or 4");
  int64_t rows = nt * nb * nchan;
  if (rows == 0) return AV_OK;
  cudaStream_t st = as_stream(stream);
  k_briggs_apply<<<(unsigned)((rows + 255) / 256), 256, 0, st>>>(
      out, out_dtype, density, factors, nchan, uvw, freq, wt, wt_dtype, flag, n_u, n_v, delta_l,
      delta_m, rows, nchan, npol, err_flag);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_imaging_weight_degrid(double *imaging_weight, const void *grid_imaging_weight,
                             int grid_dtype, int64_t g_chan, int64_t g_pol,
                             const double *briggs_factors, const double *uvw, const double *freq,
                             const int32_t *chan_map, const int32_t *pol_map,
                             const void *natural_weight, int wt_dtype, int64_t n_u, int64_t n_v,
                             double delta_l, double delta_m, int64_t nt, int64_t nb,
                             int64_t nchan, int64_t npol, void *stream) {
  clear_error();
  AV_CHECK_ARG(imaging_weight && grid_imaging_weight && briggs_factors && uvw && freq &&
                   chan_map && pol_map && natural_weight,
               "av_imaging_weight_degrid: null pointer");
  AV_CHECK_ARG(grid_dtype == AV_F32 || grid_dtype == AV_F64,
               "av_imaging_weight_degrid: grid dtype");
  AV_CHECK_ARG(wt_dtype == AV_F32 || wt_dtype == AV_F64,
               "av_imaging_weight_degrid: weight dtype");
  AV_CHECK_ARG(n_u > 0 && n_v > 0 && g_chan > 0 && g_pol > 0 && nt >= 0 && nb >= 0 &&
                   nchan >= 0 && npol >= 1,
               "av_imaging_weight_degrid: bad shape");
  const int64_t rows = nt * nb * nchan;
  if (rows == 0) return AV_OK;
  k_imaging_weight_degrid<<<(unsigned)((rows + 255) / 256), 256, 0, as_stream(stream)>>>(
      imaging_weight, grid_imaging_weight, grid_dtype, g_chan, g_pol, briggs_factors, uvw, freq,
      chan_map, pol_map, natural_weight, wt_dtype, n_u, n_v, delta_l, delta_m, rows, nchan,
      npol);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"

// ------------------------------------------------- allocation-free variant --
// Some callers may not allocate device memory: a host program whose device
// buffers all come from a pool it sized at start-up and that allows no
// cudaMalloc/cudaFree while it processes (an allocation there synchronises
// the device and can fail mid-run), or a plugin called by another framework
// that owns all device memory and hands it only inputs and outputs.  For them
// av_briggs_factors_noalloc keeps the reduction's partial sums in the static
// array below instead of a caller workspace.

namespace av {

constexpr int kBriggsSlices = 64;  // partial sums per plane, as av_briggs_factors
constexpr int kMaxDevices = 64;

// The partial sums of up to AV_BRIGGS_NOALLOC_MAX_PLANES planes (512 KiB).
// The module holds one copy on every device that loads it, until the process
// exits.  In host code this name is a host-side stand-in: the device address
// comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) double
    g_briggs_scratch[(size_t)AV_BRIGGS_NOALLOC_MAX_PLANES * kBriggsSlices];

static std::mutex g_briggs_scratch_mu;
static void *g_briggs_scratch_ptr[kMaxDevices];

// Device address of the current device's copy of g_briggs_scratch, looked up
// on the first call made with that device current and cached afterwards (the
// cache does not survive cudaDeviceReset, which may move the array).  The
// stream must belong to the current device: the kernels would otherwise run
// on another device with this device's address.
static int briggs_scratch(cudaStream_t st, void **out) {
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (st != nullptr) {
    int sdev = dev;
    AV_CUDA(cudaStreamGetDevice(st, &sdev));
    if (sdev != dev) {
      set_error("av_briggs_factors_noalloc: the stream belongs to device %d, the current "
                "device is %d",
                sdev, dev);
      return AV_ERR_ARG;
    }
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("av_briggs_factors_noalloc: device %d beyond the %d this library tracks", dev,
              kMaxDevices);
    return AV_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_briggs_scratch_mu);
  if (!g_briggs_scratch_ptr[dev]) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_briggs_scratch);
    if (e != cudaSuccess || !ptr) {
      set_error("av_briggs_factors_noalloc: cudaGetSymbolAddress on device %d: %s", dev,
                cudaGetErrorString(e));
      return AV_ERR_CUDA;
    }
    g_briggs_scratch_ptr[dev] = ptr;
  }
  *out = g_briggs_scratch_ptr[dev];
  return AV_OK;
}

}  // namespace av

extern "C" {

int av_briggs_factors_noalloc(const double *density, const double *sum_weight, double *factors,
                              int64_t nplanes, int64_t n_u, int64_t n_v, double robust,
                              void *stream) {
  clear_error();
  AV_CHECK_ARG(density && sum_weight && factors, "av_briggs_factors_noalloc: null pointer");
  AV_CHECK_ARG(nplanes >= 0 && n_u > 0 && n_v > 0, "av_briggs_factors_noalloc: bad shape");
  AV_CHECK_ARG(nplanes <= AV_BRIGGS_NOALLOC_MAX_PLANES,
               "av_briggs_factors_noalloc: %lld planes exceed the static scratch's maximum of "
               "%d planes; use av_briggs_factors with a workspace",
               (long long)nplanes, AV_BRIGGS_NOALLOC_MAX_PLANES);
  static_assert(sizeof(g_briggs_scratch) ==
                    (size_t)AV_BRIGGS_NOALLOC_MAX_PLANES * kBriggsSlices * sizeof(double),
                "scratch size");
  void *scratch = nullptr;
  int rc = briggs_scratch(as_stream(stream), &scratch);
  if (rc != AV_OK) return rc;
  // every partial k_briggs_finish reads, k_sum_sq of the same call writes
  // first: nothing needs clearing between calls
  return av_briggs_factors(density, sum_weight, factors, nplanes, n_u, n_v, robust, scratch,
                           sizeof(g_briggs_scratch), stream);
}

}  // extern "C"
