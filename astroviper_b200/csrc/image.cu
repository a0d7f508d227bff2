// Image formation (grid2image_spheroid_ms4, standard_grid.py:693-708) and the
// centred FFT helpers (fft.py:5, ifft.py:5).
//
// The ifftshift is a gather in the kernel that fills the cuFFT buffer; the
// fftshift, the real part, the grid correction 1 / (grdsf(x) grdsf(y)) and
// the nx*ny / sumwt scaling are one epilogue kernel.  numpy's ifft2 carries
// 1/(nx*ny), which the reference multiplies back: the unnormalised cuFFT
// inverse is the same quantity.
#include <cufft.h>

#include <deque>
#include <mutex>

#include "common.cuh"

namespace av {

// ----------------------------------------------------------- plan cache ---
struct FftPlan {
  int dev;
  int64_t nplanes, nx, ny;
  int dbl;
  cufftHandle h;
  size_t work;
};
static std::mutex g_fft_mu;
static std::deque<FftPlan> g_fft_plans;  // stable addresses on push_back

#define AV_CUFFT(call)                                                        \
  do {                                                                        \
    cufftResult r_ = (call);                                                  \
    if (r_ != CUFFT_SUCCESS) {                                                \
      ::av::set_error("%s failed: cufftResult %d (%s:%d)", #call, (int)r_,    \
                      __FILE__, __LINE__);                                    \
      return AV_ERR_CUDA;                                                     \
    }                                                                         \
  } while (0)

// Plan for nplanes batched (nx, ny) C2C (Z2Z when dbl) transforms, without
// auto-allocated work area (the caller's workspace is attached per call).
static int get_plan(int64_t nplanes, int64_t nx, int64_t ny, int dbl, FftPlan **out) {
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_fft_mu);
  for (auto &p : g_fft_plans)
    if (p.dev == dev && p.nplanes == nplanes && p.nx == nx && p.ny == ny && p.dbl == dbl) {
      *out = &p;
      return AV_OK;
    }
  FftPlan p;
  p.dev = dev;
  p.nplanes = nplanes;
  p.nx = nx;
  p.ny = ny;
  p.dbl = dbl;
  AV_CUFFT(cufftCreate(&p.h));
  AV_CUFFT(cufftSetAutoAllocation(p.h, 0));
  long long n[2] = {nx, ny};
  size_t ws = 0;
  AV_CUFFT(cufftMakePlanMany64(p.h, 2, n, nullptr, 1, nx * ny, nullptr, 1, nx * ny,
                               dbl ? CUFFT_Z2Z : CUFFT_C2C, nplanes, &ws));
  p.work = ws;
  g_fft_plans.push_back(p);
  *out = &g_fft_plans.back();
  return AV_OK;
}

// Work-area bytes of the (cached) plan for this size.
static size_t fft_work_bytes(int64_t nplanes, int64_t nx, int64_t ny, int dbl) {
  FftPlan *p = nullptr;
  if (get_plan(nplanes, nx, ny, dbl, &p) != AV_OK) return 0;
  return p->work;
}

// ifftshift gather: buf[i, j] = in[(i + nx/2) % nx, (j + ny/2) % ny]
template <typename CT, typename IT>
__global__ void k_ishift_in(const IT *in, CT *buf, int64_t nplanes, int64_t nx, int64_t ny) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t n = nplanes * nx * ny;
  if (k >= n) return;
  int64_t p = k / (nx * ny), r = k - p * nx * ny;
  int64_t i = r / ny, j = r - i * ny;
  int64_t si = i + nx / 2;
  if (si >= nx) si -= nx;
  int64_t sj = j + ny / 2;
  if (sj >= ny) sj -= ny;
  IT v = in[p * nx * ny + si * ny + sj];
  CT o;
  o.x = v.x;
  o.y = v.y;
  buf[k] = o;
}

// fftshift of the transform + real part + grid correction + normalisation.
template <typename CT, typename OT>
__global__ void k_image_epilogue(const CT *buf, OT *img, const double *sumw, int64_t nplanes,
                                 int64_t nx, int64_t ny, int apply_corr) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t n = nplanes * nx * ny;
  if (k >= n) return;
  int64_t p = k / (nx * ny), r = k - p * nx * ny;
  int64_t i = r / ny, j = r - i * ny;
  // fftshift: out[i] = in[(i - nx/2) mod nx] = in[(i + nx - nx/2) % nx]
  int64_t si = i + (nx - nx / 2);
  if (si >= nx) si -= nx;
  int64_t sj = j + (ny - ny / 2);
  if (sj >= ny) sj -= ny;
  double v = (double)buf[p * nx * ny + si * ny + sj].x;
  if (apply_corr) {
    double cx = (double)(i - nx / 2) / (double)nx;
    double cy = (double)(j - ny / 2) / (double)ny;
    double corr = pswf_grdsf(fabs(2.0 * cx)) * pswf_grdsf(fabs(2.0 * cy));
    v = v / corr;
  }
  if (sumw) v = v / sumw[p];
  img[k] = (OT)v;
}

// Real image -> ifftshift gather into the complex FP64 transform buffer,
// divided by the grid correction grdsf(x) grdsf(y) when asked.
template <typename IT>
__global__ void k_image_prologue(const IT *img, double2 *buf, int64_t nplanes, int64_t nx,
                                 int64_t ny, int apply_corr) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t n = nplanes * nx * ny;
  if (k >= n) return;
  int64_t p = k / (nx * ny), r = k - p * nx * ny;
  int64_t i = r / ny, j = r - i * ny;
  int64_t si = i + nx / 2;
  if (si >= nx) si -= nx;
  int64_t sj = j + ny / 2;
  if (sj >= ny) sj -= ny;
  double v = (double)img[p * nx * ny + si * ny + sj];
  if (apply_corr) {
    double cx = (double)(si - nx / 2) / (double)nx;
    double cy = (double)(sj - ny / 2) / (double)ny;
    v = v / (pswf_grdsf(fabs(2.0 * cx)) * pswf_grdsf(fabs(2.0 * cy)));
  }
  buf[k] = make_double2(v, 0.0);
}

// fftshift gather of a complex result: out[i] = buf[(i + nx - nx/2) % nx].
template <typename CT, typename OT>
__global__ void k_shift_out(const CT *buf, OT *out, int64_t nplanes, int64_t nx, int64_t ny,
                            double scale) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t n = nplanes * nx * ny;
  if (k >= n) return;
  int64_t p = k / (nx * ny), r = k - p * nx * ny;
  int64_t i = r / ny, j = r - i * ny;
  int64_t si = i + (nx - nx / 2);
  if (si >= nx) si -= nx;
  int64_t sj = j + (ny - ny / 2);
  if (sj >= ny) sj -= ny;
  CT v = buf[p * nx * ny + si * ny + sj];
  OT o;
  o.x = v.x * scale;
  o.y = v.y * scale;
  out[k] = o;
}

static int run_fft(void *buf, int dbl, int64_t nplanes, int64_t nx, int64_t ny, int dir,
                   void *work, cudaStream_t st) {
  FftPlan *p = nullptr;
  int rc = get_plan(nplanes, nx, ny, dbl, &p);
  if (rc) return rc;
  AV_CUFFT(cufftSetStream(p->h, st));
  AV_CUFFT(cufftSetWorkArea(p->h, work));
  if (dbl)
    AV_CUFFT(cufftExecZ2Z(p->h, (cufftDoubleComplex *)buf, (cufftDoubleComplex *)buf, dir));
  else
    AV_CUFFT(cufftExecC2C(p->h, (cufftComplex *)buf, (cufftComplex *)buf, dir));
  return AV_OK;
}

}  // namespace av

using namespace av;

extern "C" {

size_t av_fft_workspace_size(int64_t nplanes, int64_t nx, int64_t ny, int precision) {
  int dbl = precision == AV_F64 || precision == AV_C128;
  size_t buf = (size_t)nplanes * nx * ny * (dbl ? 16 : 8);
  return Workspace::need(buf) + Workspace::need(fft_work_bytes(nplanes, nx, ny, dbl));
}

size_t av_grid_to_image_workspace_size(int64_t nplanes, int64_t nx, int64_t ny) {
  size_t buf = (size_t)nplanes * nx * ny * 16;
  return Workspace::need(buf) + Workspace::need(fft_work_bytes(nplanes, nx, ny, 1));
}

// The transform is always FP64 (Z2Z): the grid correction divides by a taper
// that is ~4e-3 at the image edges, which would amplify FP32 transform
// rounding to ~1e-4 relative error in the image.
int av_grid_to_image(const void *grid, int grid_dtype, const double *sum_weight, void *image,
                     int image_dtype, int64_t nplanes, int64_t nx, int64_t ny, int apply_corr,
                     void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(grid && image, "av_grid_to_image: null pointer");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128, "av_grid_to_image: grid dtype");
  AV_CHECK_ARG(image_dtype == AV_F32 || image_dtype == AV_F64, "av_grid_to_image: image dtype");
  AV_CHECK_ARG(nplanes >= 0 && nx > 0 && ny > 0, "av_grid_to_image: bad shape");
  if (nplanes == 0) return AV_OK;
  FftPlan *p = nullptr;
  int rc = get_plan(nplanes, nx, ny, 1, &p);
  if (rc) return rc;
  size_t bufb = (size_t)nplanes * nx * ny * 16;
  if (!workspace || workspace_bytes < Workspace::need(bufb) + Workspace::need(p->work)) {
    set_error("av_grid_to_image: workspace too small (%zu < %zu)", workspace_bytes,
              Workspace::need(bufb) + Workspace::need(p->work));
    return AV_ERR_WORKSPACE;
  }
  Workspace ws(workspace, workspace_bytes);
  double2 *buf = ws.take<double2>((size_t)nplanes * nx * ny);
  void *work = ws.take<char>(p->work > 0 ? p->work : 1);
  cudaStream_t st = as_stream(stream);
  int64_t n = nplanes * nx * ny;
  unsigned blocks = (unsigned)((n + 255) / 256);
  if (grid_dtype == AV_C128)
    k_ishift_in<double2, double2><<<blocks, 256, 0, st>>>((const double2 *)grid, buf, nplanes,
                                                         nx, ny);
  else
    k_ishift_in<double2, float2><<<blocks, 256, 0, st>>>((const float2 *)grid, buf, nplanes, nx,
                                                        ny);
  AV_LAUNCH_CHECK();
  rc = run_fft(buf, 1, nplanes, nx, ny, CUFFT_INVERSE, work, st);
  if (rc) return rc;
  if (image_dtype == AV_F64)
    k_image_epilogue<double2, double><<<blocks, 256, 0, st>>>(buf, (double *)image, sum_weight,
                                                             nplanes, nx, ny, apply_corr);
  else
    k_image_epilogue<double2, float><<<blocks, 256, 0, st>>>(buf, (float *)image, sum_weight,
                                                            nplanes, nx, ny, apply_corr);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// fft_lm_to_uv(image / corrTerm) (fft.py:5 with the grid correction of
// gcf_prolate_spheroidal.py:73-79): the forward model's image -> grid step,
// the adjoint of av_grid_to_image without sum_weight.  FP64 transform.
int av_image_to_grid(const void *image, int image_dtype, void *grid, int grid_dtype,
                     int64_t nplanes, int64_t nx, int64_t ny, int apply_corr, void *workspace,
                     size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(image && grid, "av_image_to_grid: null pointer");
  AV_CHECK_ARG(image_dtype == AV_F32 || image_dtype == AV_F64, "av_image_to_grid: image dtype");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128, "av_image_to_grid: grid dtype");
  AV_CHECK_ARG(nplanes >= 0 && nx > 0 && ny > 0, "av_image_to_grid: bad shape");
  if (nplanes == 0) return AV_OK;
  FftPlan *p = nullptr;
  int rc = get_plan(nplanes, nx, ny, 1, &p);
  if (rc) return rc;
  size_t bufb = (size_t)nplanes * nx * ny * 16;
  if (!workspace || workspace_bytes < Workspace::need(bufb) + Workspace::need(p->work)) {
    set_error("av_image_to_grid: workspace too small");
    return AV_ERR_WORKSPACE;
  }
  Workspace ws(workspace, workspace_bytes);
  double2 *buf = ws.take<double2>((size_t)nplanes * nx * ny);
  void *work = ws.take<char>(p->work > 0 ? p->work : 1);
  cudaStream_t st = as_stream(stream);
  int64_t n = nplanes * nx * ny;
  unsigned blocks = (unsigned)((n + 255) / 256);
  if (image_dtype == AV_F64)
    k_image_prologue<double><<<blocks, 256, 0, st>>>((const double *)image, buf, nplanes, nx, ny,
                                                     apply_corr);
  else
    k_image_prologue<float><<<blocks, 256, 0, st>>>((const float *)image, buf, nplanes, nx, ny,
                                                    apply_corr);
  AV_LAUNCH_CHECK();
  rc = run_fft(buf, 1, nplanes, nx, ny, CUFFT_FORWARD, work, st);
  if (rc) return rc;
  if (grid_dtype == AV_C128)
    k_shift_out<double2, double2><<<blocks, 256, 0, st>>>(buf, (double2 *)grid, nplanes, nx, ny,
                                                         1.0);
  else
    k_shift_out<double2, float2><<<blocks, 256, 0, st>>>(buf, (float2 *)grid, nplanes, nx, ny,
                                                        1.0);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_fft_shifted(const void *in, void *out, int dtype, int64_t nplanes, int64_t nx, int64_t ny,
                   int inverse, void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(in && out, "av_fft_shifted: null pointer");
  AV_CHECK_ARG(dtype == AV_C64 || dtype == AV_C128, "av_fft_shifted: dtype");
  AV_CHECK_ARG(nplanes >= 0 && nx > 0 && ny > 0, "av_fft_shifted: bad shape");
  if (nplanes == 0) return AV_OK;
  int dbl = dtype == AV_C128;
  FftPlan *p = nullptr;
  int rc = get_plan(nplanes, nx, ny, dbl, &p);
  if (rc) return rc;
  size_t bufb = (size_t)nplanes * nx * ny * (dbl ? 16 : 8);
  if (!workspace || workspace_bytes < Workspace::need(bufb) + Workspace::need(p->work)) {
    set_error("av_fft_shifted: workspace too small");
    return AV_ERR_WORKSPACE;
  }
  Workspace ws(workspace, workspace_bytes);
  void *buf = ws.take<char>(bufb);
  void *work = ws.take<char>(p->work > 0 ? p->work : 1);
  cudaStream_t st = as_stream(stream);
  int64_t n = nplanes * nx * ny;
  unsigned blocks = (unsigned)((n + 255) / 256);
  double scale = inverse ? 1.0 / ((double)nx * (double)ny) : 1.0;
  if (dbl)
    k_ishift_in<double2, double2><<<blocks, 256, 0, st>>>((const double2 *)in, (double2 *)buf,
                                                         nplanes, nx, ny);
  else
    k_ishift_in<float2, float2><<<blocks, 256, 0, st>>>((const float2 *)in, (float2 *)buf,
                                                       nplanes, nx, ny);
  AV_LAUNCH_CHECK();
  rc = run_fft(buf, dbl, nplanes, nx, ny, inverse ? CUFFT_INVERSE : CUFFT_FORWARD, work, st);
  if (rc) return rc;
  if (dbl)
    k_shift_out<double2, double2><<<blocks, 256, 0, st>>>((const double2 *)buf, (double2 *)out,
                                                         nplanes, nx, ny, scale);
  else
    k_shift_out<float2, float2><<<blocks, 256, 0, st>>>((const float2 *)buf, (float2 *)out,
                                                       nplanes, nx, ny, scale);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"
