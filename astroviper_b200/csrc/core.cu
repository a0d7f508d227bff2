// Error reporting, version, device queries and the PSWF tables.
#include <stdarg.h>
#include <string.h>

#include <atomic>

#include "common.cuh"

namespace av {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void clear_error() { g_err[0] = 0; }

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

// grdsf and (1-u^2) grdsf of gcf_prolate_spheroidal.py:102-158.
__global__ void k_pswf(const double *__restrict__ u, int64_t n, double *grdsf, double *kern) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = fabs(u[i]);
  double g = pswf_grdsf(x);
  if (grdsf) grdsf[i] = g;
  if (kern) kern[i] = __dmul_rn(__dsub_rn(1.0, __dmul_rn(x, x)), g);
}

// create_prolate_spheroidal_kernel_1D (gcf_prolate_spheroidal.py:87-99).
__global__ void k_pswf_table(double *out, int os, int sc) {
  int64_t n = (int64_t)os * sc, ntot = (int64_t)os * (sc + 1);
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  if (i >= n) {
    out[i] = 0.0;
    return;
  }
  double u = __ddiv_rn((double)i, (double)(sc * os));
  double g = pswf_grdsf(u);
  out[i] = __dmul_rn(__dsub_rn(1.0, __dmul_rn(u, u)), g);
}

// corrTerm of gcf_prolate_spheroidal.py:73-79 with coordinates() (:161).
__global__ void k_corr_term(double *out, int64_t nx, int64_t ny) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nx * ny) return;
  int64_t i = k / ny, j = k - i * ny;
  double cx = __ddiv_rn((double)(i - nx / 2), (double)nx);
  double cy = __ddiv_rn((double)(j - ny / 2), (double)ny);
  double gx = pswf_grdsf(fabs(__dmul_rn(2.0, cx)));
  double gy = pswf_grdsf(fabs(__dmul_rn(2.0, cy)));
  out[k] = __dmul_rn(gx, gy);
}

// The 4-D kernel of create_prolate_spheroidal_kernel (gcf:28-67):
// kernel[x, y, :, :] = outer(k1[x, :], k1[y, :]) for x, y < oversampling with
// k1[o, s] = (1-u^2) grdsf(u), u = ((s - sc) + (o - oc)/os) / sc; the last
// row/column (index os, even oversampling only) stays zero as in the loop
// bounds of the reference.
__global__ void k_pswf_kernel4d(double *out, int os, int support, int n_os) {
  int64_t total = (int64_t)n_os * n_os * support * support;
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= total) return;
  int s2 = (int)(k % support);
  int64_t r = k / support;
  int s1 = (int)(r % support);
  r /= support;
  int y = (int)(r % n_os);
  int x = (int)(r / n_os);
  if (x >= os || y >= os) {
    out[k] = 0.0;
    return;
  }
  int sc = support / 2, oc = os / 2;
  double ox = __ddiv_rn((double)(x - oc), (double)os);
  double oy = __ddiv_rn((double)(y - oc), (double)os);
  double ux = __ddiv_rn(__dadd_rn((double)(s1 - sc), ox), (double)sc);
  double uy = __ddiv_rn(__dadd_rn((double)(s2 - sc), oy), (double)sc);
  double kx = __dmul_rn(__dsub_rn(1.0, __dmul_rn(ux, ux)), pswf_grdsf(fabs(ux)));
  double ky = __dmul_rn(__dsub_rn(1.0, __dmul_rn(uy, uy)), pswf_grdsf(fabs(uy)));
  out[k] = __dmul_rn(kx, ky);
}

// ------------------------------------------------------------ tuning ---
constexpr int kTuneKnobs = 5;
static std::atomic<int64_t> g_tune[kTuneKnobs] = {
    {16}, {16}, {AV_GRID_LANES_AUTO}, {AV_DEGRID_LANES_AUTO}, {2000000}};

int64_t tune_value(int knob) {
  return (knob >= 0 && knob < kTuneKnobs) ? g_tune[knob].load() : 0;
}

// ------------------------------------------------------------ probes ---
// FP64 tensor rate: every warp runs four independent chains of
// mma.sync.m16n8k4.f64 (one dependent chain already keeps an SMSP's pipe
// full); thread 0 of each block writes one double to a static sink.
constexpr int kProbeIters = 4096;
constexpr int kProbeThreads = 256;
static __device__ double g_probe_sink[4096];

__global__ void __launch_bounds__(kProbeThreads) k_probe_dmma(double s) {
  double d[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.0;
  const double a0 = s + threadIdx.x * 1e-6, a1 = s * 0.5, b = s - threadIdx.x * 1e-6;
  for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
      asm volatile(
          "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
          "{%0,%1,%2,%3};\n"
          : "+d"(d[j][0]), "+d"(d[j][1]), "+d"(d[j][2]), "+d"(d[j][3])
          : "d"(a0), "d"(a1), "d"(b));
  }
  double t = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) t += d[j][0] + d[j][1] + d[j][2] + d[j][3];
  if (threadIdx.x == 0) g_probe_sink[blockIdx.x & 4095] = t;
}

}  // namespace av

using namespace av;

extern "C" {

int av_probe_fp64_mma(double *tflops, void *stream) {
  clear_error();
  AV_CHECK_ARG(tflops, "av_probe_fp64_mma: null pointer");
  cudaStream_t st = as_stream(stream);
  const int blocks = sm_count() * 8;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  AV_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    set_error("av_probe_fp64_mma: event creation failed");
    return AV_ERR_CUDA;
  }
  int rc = AV_OK;
  float ms = 0.f;
  k_probe_dmma<<<blocks, kProbeThreads, 0, st>>>(0.999);  // warm-up
  count_launch();
  cudaEventRecord(e0, st);
  for (int r = 0; r < 3; ++r) {
    k_probe_dmma<<<blocks, kProbeThreads, 0, st>>>(0.999);
    count_launch();
  }
  cudaEventRecord(e1, st);
  cudaError_t err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  if (err != cudaSuccess || ms <= 0.f) {
    set_error("av_probe_fp64_mma: %s", cudaGetErrorString(err));
    rc = AV_ERR_CUDA;
  } else {
    const double flop = 3.0 * blocks * (kProbeThreads / 32) * (double)kProbeIters * 4 * 512 * 2;
    *tflops = flop / (ms * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int av_version(void) { return 100; }

const char *av_last_error(void) { return g_err; }

int av_device_sm_count(void) { return sm_count(); }

unsigned long long av_launch_count(void) { return g_launches.load(); }

int av_tune_set(int knob, int64_t value) {
  clear_error();
  AV_CHECK_ARG(knob >= 0 && knob < kTuneKnobs, "av_tune_set: unknown knob %d", knob);
  if (knob == AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US) {
    AV_CHECK_ARG(value >= 0 && value <= 600000000,
                 "av_tune_set: AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US %lld outside [0, 600000000]",
                 (long long)value);
    g_tune[knob].store(value);
    return AV_OK;
  }
  AV_CHECK_ARG(value >= 1 && value <= 1024, "av_tune_set: value %lld outside [1, 1024]",
               (long long)value);
  AV_CHECK_ARG(knob != AV_TUNE_GRID_LANES || value <= 3,
               "av_tune_set: AV_TUNE_GRID_LANES takes 1 (mma), 2 (rows) or 3 (auto), not %lld",
               (long long)value);
  AV_CHECK_ARG(knob != AV_TUNE_DEGRID_LANES || value <= 4,
               "av_tune_set: AV_TUNE_DEGRID_LANES takes 1 (tf32), 2 (fp32), 3 (auto) or 4 "
               "(tc05), not %lld",
               (long long)value);
  g_tune[knob].store(value);
  return AV_OK;
}

int64_t av_tune_get(int knob) {
  if (knob < 0 || knob >= kTuneKnobs) return -1;
  return g_tune[knob].load();
}

int av_pswf(const double *u_in, int64_t n, double *grdsf, double *kern, void *stream) {
  clear_error();
  AV_CHECK_ARG(n >= 0 && (n == 0 || u_in), "av_pswf: bad input");
  if (n == 0) return AV_OK;
  k_pswf<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(u_in, n, grdsf, kern);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_pswf_table(double *out, int oversampling, int support, void *stream) {
  clear_error();
  AV_CHECK_ARG(out && oversampling > 0 && support >= 2, "av_pswf_table: bad arguments");
  int sc = support / 2;
  int64_t ntot = (int64_t)oversampling * (sc + 1);
  k_pswf_table<<<(unsigned)((ntot + 255) / 256), 256, 0, as_stream(stream)>>>(out, oversampling,
                                                                              sc);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_corr_term(double *out, int64_t nx, int64_t ny, void *stream) {
  clear_error();
  AV_CHECK_ARG(out && nx > 0 && ny > 0, "av_corr_term: bad arguments");
  int64_t n = nx * ny;
  k_corr_term<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(out, nx, ny);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_pswf_kernel4d(double *out, int oversampling, int support, void *stream) {
  clear_error();
  AV_CHECK_ARG(out && oversampling > 0 && support >= 2, "av_pswf_kernel4d: bad arguments");
  int n_os = (oversampling % 2 == 0) ? oversampling + 1 : oversampling;
  int64_t total = (int64_t)n_os * n_os * support * support;
  k_pswf_kernel4d<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(
      out, oversampling, support, n_os);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"
