// Shared helpers of libav200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/av200.h"

namespace av {

// ----------------------------------------------------------------- errors --
void set_error(const char *fmt, ...);
void clear_error();

#define AV_CHECK_ARG(cond, ...)        \
  do {                                 \
    if (!(cond)) {                     \
      ::av::set_error(__VA_ARGS__);    \
      return AV_ERR_ARG;               \
    }                                  \
  } while (0)

#define AV_CUDA(call)                                                               \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      ::av::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                      __FILE__, __LINE__);                                          \
      return AV_ERR_CUDA;                                                           \
    }                                                                               \
  } while (0)

// Every kernel launch of the library is followed by AV_LAUNCH_CHECK, which
// also counts it (av_launch_count).
void count_launch();
#define AV_LAUNCH_CHECK()      \
  do {                         \
    ::av::count_launch();      \
    AV_CUDA(cudaGetLastError()); \
  } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Bump allocator over a caller-supplied workspace (256-byte aligned pieces).
struct Workspace {
  char *base;
  size_t size, used;
  Workspace(void *p, size_t n) : base((char *)p), size(n), used(0) {}
  template <typename T>
  T *take(size_t count) {
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (used + bytes > size) return nullptr;
    T *p = reinterpret_cast<T *>(base + used);
    used += bytes;
    return p;
  }
  static size_t need(size_t bytes) { return (bytes + 255) & ~size_t(255); }
};

// -------------------------------------------------------------- constants --
constexpr double C_LIGHT = 299792458.0;

// ------------------------------------------------------------------- PSWF --
// d^k for k = 2, 3, 4 rounded once: the reference evaluates numpy's power,
// which is within half an ulp; products are carried as double-double pairs
// (error-free transformations with fma) and rounded at the end.
__device__ inline void pow234(double d, double &d2, double &d3, double &d4) {
  double h2 = d * d;
  double l2 = fma(d, d, -h2);           // d*d = h2 + l2 exactly
  d2 = h2;
  double p3 = h2 * d;
  double e3 = fma(h2, d, -p3);          // h2*d = p3 + e3 exactly
  d3 = p3 + (e3 + l2 * d);
  double p4 = h2 * h2;
  double e4 = fma(h2, h2, -p4);         // h2*h2 = p4 + e4 exactly
  d4 = p4 + (e4 + 2.0 * h2 * l2);
}

// Schwab's rational approximation (gcf_prolate_spheroidal.py:116-158).
__device__ inline double pswf_grdsf(double u) {
  const double P[2][5] = {{8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1},
                          {4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2}};
  const double Q[2][3] = {{1.0000000e0, 8.212018e-1, 2.078043e-1},
                          {1.0000000e0, 9.599102e-1, 2.918724e-1}};
  u = fabs(u);
  int part = 0;
  double uend = 0.0;
  if (u >= 0.0 && u < 0.75) { part = 0; uend = 0.75; }
  if (u >= 0.75 && u <= 1.0) { part = 1; uend = 1.0; }
  double d = __dsub_rn(__dmul_rn(u, u), __dmul_rn(uend, uend));
  double d2, d3, d4;
  pow234(d, d2, d3, d4);
  double top = P[part][0];
  top = __dadd_rn(top, __dmul_rn(P[part][1], d));
  top = __dadd_rn(top, __dmul_rn(P[part][2], d2));
  top = __dadd_rn(top, __dmul_rn(P[part][3], d3));
  top = __dadd_rn(top, __dmul_rn(P[part][4], d4));
  double bot = Q[part][0];
  bot = __dadd_rn(bot, __dmul_rn(Q[part][1], d));
  bot = __dadd_rn(bot, __dmul_rn(Q[part][2], d2));
  double g = 0.0;
  if (bot > 0.0) g = __ddiv_rn(top, bot);
  if (u > 1.0) g = 0.0;
  return g;
}

// ----------------------------------------------------------- index math ----
// Python int(x) of a double (truncation toward zero); magnitudes that cannot
// be grid indices map to a sentinel that fails every bounds test.
__device__ __forceinline__ long long trunc_ll(double x) {
  if (!(fabs(x) < 4.611686018427388e18)) return -(1LL << 61);
  return (long long)x;
}

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { typedef float2 type; };
template <> struct cplx_of<double> { typedef double2 type; };

// -------------------------------------------------------------- dtype size --
inline size_t dtype_size(int dt) {
  switch (dt) {
    case AV_F32: return 4;
    case AV_F64: return 8;
    case AV_C64: return 8;
    case AV_C128: return 16;
  }
  return 0;
}

// Number of SMs of the current device (cached per device).
int sm_count();

// Launch tuning knobs (av_tune_set); read at launch time.
int64_t tune_value(int knob);

}  // namespace av
