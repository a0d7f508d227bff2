// Device steps of the major/minor-cycle imager (imager.py:108-351) around
// the gridder, the degridder and Hogbom CLEAN:
//
// av_pol_transform   correlation <-> Stokes image products, pixel by pixel
//                    (corr_to_stokes.py:71-138, image_corr_to_stokes :141-305,
//                    image_stokes_to_corr :307-487)
// av_argmax          first index of the largest |x| or x (np.argmax), for the
//                    peak residuals of deconvolution.py:223-289 and the PSF
//                    peak of psf_gaussian_fit.py:62-73
// av_psf_sidelobe    max_sidelobe of extract_main_lobe (psf_gaussian_fit.py:
//                    46-126): the main lobe is the 4-connected component
//                    above threshold x peak, around the peak inside the
//                    search window, labelled in one CTA
// av_plane_sum       per-plane sums (model flux, deconvolution.py:262)
// av_vis_residual    RESIDUAL = VISIBILITY - VISIBILITY_MODEL (imager.py:82-85)
#include "common.cuh"

namespace av {

// ------------------------------------------------------ pol transform ------
struct PolMatrix {
  double re[16], im[16];  // row-major n_out x n_in
  int n_in, n_out;
};

__device__ __forceinline__ double2 load_pol(const void *p, int dt, int64_t i) {
  switch (dt) {
    case AV_F32: return make_double2((double)((const float *)p)[i], 0.0);
    case AV_F64: return make_double2(((const double *)p)[i], 0.0);
    case AV_C64: {
      const float2 v = ((const float2 *)p)[i];
      return make_double2((double)v.x, (double)v.y);
    }
    default: return ((const double2 *)p)[i];
  }
}

__device__ __forceinline__ void store_pol(void *p, int dt, int64_t i, double2 v) {
  switch (dt) {
    case AV_F32: ((float *)p)[i] = (float)v.x; break;
    case AV_F64: ((double *)p)[i] = v.x; break;
    case AV_C64: ((float2 *)p)[i] = make_float2((float)v.x, (float)v.y); break;
    default: ((double2 *)p)[i] = v; break;
  }
}

// out[o] = sum_i M[o][i] in[i] in complex arithmetic, terms with a zero
// coefficient left out and no fused multiply-add: with the coefficients of the
// reference's tables (0, +-1, +-0.5, +-i, +-0.5i) every product is exact and
// each output is one rounding of its two terms, as numpy's matmul gives.
__global__ void k_pol_transform(const void *in, int in_dt, void *out, int out_dt, PolMatrix m,
                                int64_t n_outer, int64_t n_pix) {
  const int64_t n = n_outer * n_pix;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = t / n_pix, px = t - o * n_pix;
    double2 x[4];
    for (int i = 0; i < m.n_in; ++i) x[i] = load_pol(in, in_dt, (o * m.n_in + i) * n_pix + px);
    for (int r = 0; r < m.n_out; ++r) {
      double2 acc = make_double2(0.0, 0.0);
      bool any = false;
      for (int i = 0; i < m.n_in; ++i) {
        const double cr = m.re[r * m.n_in + i], ci = m.im[r * m.n_in + i];
        if (cr == 0.0 && ci == 0.0) continue;
        const double pr = __dsub_rn(__dmul_rn(x[i].x, cr), __dmul_rn(x[i].y, ci));
        const double pi = __dadd_rn(__dmul_rn(x[i].x, ci), __dmul_rn(x[i].y, cr));
        if (!any) {
          acc = make_double2(pr, pi);
          any = true;
        } else {
          acc = make_double2(__dadd_rn(acc.x, pr), __dadd_rn(acc.y, pi));
        }
      }
      store_pol(out, out_dt, (o * m.n_out + r) * n_pix + px, acc);
    }
  }
}

// ------------------------------------------------------------- argmax ------
// np.argmax order: NaN above everything, equal values to the lower index.
struct ArgMax {
  double key;   // compared value (|x| or x)
  double val;   // signed value at idx
  int64_t idx;  // -1: none
};

__device__ __forceinline__ bool am_better(const ArgMax &a, const ArgMax &b) {
  if (a.idx < 0) return false;
  if (b.idx < 0) return true;
  const bool na = isnan(a.key), nb = isnan(b.key);
  if (na || nb) {
    if (na && nb) return a.idx < b.idx;
    return na;
  }
  if (a.key != b.key) return a.key > b.key;
  return a.idx < b.idx;
}

__device__ __forceinline__ ArgMax am_shfl(const ArgMax &a, int off) {
  ArgMax b;
  b.key = __shfl_down_sync(0xffffffffu, a.key, off);
  b.val = __shfl_down_sync(0xffffffffu, a.val, off);
  b.idx = __shfl_down_sync(0xffffffffu, a.idx, off);
  return b;
}

// Block reduction; the result is valid in thread 0.
__device__ ArgMax am_block(ArgMax a) {
  __shared__ ArgMax sh[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    const ArgMax b = am_shfl(a, off);
    if (am_better(b, a)) a = b;
  }
  if (lane == 0) sh[w] = a;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  if (w == 0) {
    ArgMax c;
    c.idx = -1;
    c.key = c.val = 0.0;
    if (lane < nw) c = sh[lane];
    for (int off = 16; off > 0; off >>= 1) {
      const ArgMax b = am_shfl(c, off);
      if (am_better(b, c)) c = b;
    }
    a = c;
  }
  __syncthreads();
  return a;
}

__device__ __forceinline__ double ld_real(const void *p, int dt, int64_t i) {
  return dt == AV_F32 ? (double)((const float *)p)[i] : ((const double *)p)[i];
}

constexpr int AM_THREADS = 256;

__global__ void __launch_bounds__(AM_THREADS) k_argmax_partial(const void *x, int dt, int64_t n,
                                                               int mode, ArgMax *part) {
  ArgMax a;
  a.idx = -1;
  a.key = a.val = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    ArgMax b;
    b.val = ld_real(x, dt, i);
    b.key = mode == 0 ? fabs(b.val) : b.val;
    b.idx = i;
    if (am_better(b, a)) a = b;
  }
  a = am_block(a);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

__global__ void __launch_bounds__(1024) k_argmax_final(const ArgMax *part, int np,
                                                       int64_t *out_idx, double *out_val) {
  ArgMax a;
  a.idx = -1;
  a.key = a.val = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x)
    if (am_better(part[i], a)) a = part[i];
  a = am_block(a);
  if (threadIdx.x == 0) {
    *out_idx = a.idx;
    *out_val = a.val;
  }
}

static int argmax_blocks(int64_t n) {
  int64_t b = (n + AM_THREADS * 8 - 1) / (AM_THREADS * 8);
  const int64_t cap = (int64_t)sm_count() * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

static size_t argmax_ws(int64_t n) {
  return Workspace::need(sizeof(ArgMax) * (size_t)argmax_blocks(n));
}

static int launch_argmax(const void *x, int dt, int64_t n, int mode, int64_t *out_idx,
                         double *out_val, ArgMax *part, cudaStream_t st) {
  const int nb = argmax_blocks(n);
  k_argmax_partial<<<nb, AM_THREADS, 0, st>>>(x, dt, n, mode, part);
  AV_LAUNCH_CHECK();
  k_argmax_final<<<1, 1024, 0, st>>>(part, nb, out_idx, out_val);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// -------------------------------------------------------- PSF sidelobe -----
// Geometry and outcome of the main-lobe labelling, in the workspace.
struct LobeInfo {
  int64_t r0, c0;  // window origin (row, column)
  int wr, wc;      // window extent
  int mode;        // 0: max over the PSF with the main lobe as 0; 1: result 0; 2: error
  int err;         // 1: threshold x peak < 0; 2: labelling did not settle
};

constexpr int LOBE_THREADS = 1024;

// One CTA.  Window rows follow the peak's column index and window columns its
// row index, as extract_main_lobe slices axis 3 with peak_x and axis 4 with
// peak_y (psf_gaussian_fit.py:78-98).
__global__ void __launch_bounds__(LOBE_THREADS) k_psf_lobe(const void *psf, int dt, int64_t ny,
                                                           int64_t nx, int win0, int win1,
                                                           double threshold,
                                                           const int64_t *peak_idx,
                                                           const double *peak_val,
                                                           LobeInfo *info, uint8_t *main_mask) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ int s_changed;
  const int64_t pidx = *peak_idx;
  const double peak = *peak_val;
  const int64_t py = pidx / nx, px = pidx - (pidx / nx) * nx;
  int64_t r0 = px - win0 / 2, r1 = px + win0 / 2, c0 = py - win1 / 2, c1 = py + win1 / 2;
  if (r0 < 0) r0 = 0;
  if (c0 < 0) c0 = 0;
  if (r1 > ny) r1 = ny;
  if (c1 > nx) c1 = nx;
  const int wr = r1 > r0 ? (int)(r1 - r0) : 0, wc = c1 > c0 ? (int)(c1 - c0) : 0;
  const int nw = wr * wc;
  const double thr = __dmul_rn(peak, threshold);
  if (threadIdx.x == 0) {
    info->r0 = r0;
    info->c0 = c0;
    info->wr = wr;
    info->wc = wc;
    info->err = 0;
    info->mode = 0;
  }
  if (peak == 0.0 || nw == 0) {  // no lobe: every product with the label mask is 0
    if (threadIdx.x == 0) info->mode = 1;
    return;
  }
  if (thr < 0.0) {  // pixels outside the window would count as above threshold
    if (threadIdx.x == 0) {
      info->mode = 2;
      info->err = 1;
    }
    return;
  }
  double *val = (double *)sm;
  int *lab = (int *)(val + nw);
  // window values, and the first window pixel holding the window maximum
  ArgMax a;
  a.idx = -1;
  a.key = a.val = 0.0;
  for (int i = threadIdx.x; i < nw; i += blockDim.x) {
    const int rr = i / wc, cc = i - (i / wc) * wc;
    const double v = ld_real(psf, dt, (r0 + rr) * nx + (c0 + cc));
    val[i] = v;
    lab[i] = v > thr ? i + 1 : 0;
    ArgMax b;
    b.key = b.val = v;
    b.idx = i;  // window order is the image's C order restricted to the window
    if (am_better(b, a)) a = b;
  }
  a = am_block(a);
  __shared__ int s_main_pos;
  __shared__ int s_none;
  if (threadIdx.x == 0) {
    s_main_pos = (int)a.idx;
    // windowed_psf is 0 outside the window: a window maximum at or below the
    // threshold leaves no pixel above it, hence no lobe
    s_none = !(a.key > thr);
  }
  __syncthreads();
  if (s_none) {
    if (threadIdx.x == 0) info->mode = 1;
    return;
  }
  // 4-connected components by minimum-label propagation (bounded)
  const int max_rounds = nw + 2;
  int rounds = 0;
  for (;;) {
    if (threadIdx.x == 0) s_changed = 0;
    __syncthreads();
    int changed = 0;
    for (int i0 = 0; i0 < nw; i0 += blockDim.x) {
      const int i = i0 + threadIdx.x;
      if (i < nw && lab[i] != 0) {
        const int rr = i / wc, cc = i - (i / wc) * wc;
        int m = lab[i];
        if (rr > 0 && lab[i - wc] != 0 && lab[i - wc] < m) m = lab[i - wc];
        if (rr + 1 < wr && lab[i + wc] != 0 && lab[i + wc] < m) m = lab[i + wc];
        if (cc > 0 && lab[i - 1] != 0 && lab[i - 1] < m) m = lab[i - 1];
        if (cc + 1 < wc && lab[i + 1] != 0 && lab[i + 1] < m) m = lab[i + 1];
        if (m < lab[i]) {
          lab[i] = m;
          changed = 1;
        }
      }
    }
    if (changed) s_changed = 1;
    __syncthreads();
    const int any = s_changed;
    __syncthreads();
    if (!any) break;
    if (++rounds > max_rounds) {
      if (threadIdx.x == 0) {
        info->mode = 2;
        info->err = 2;
      }
      return;
    }
  }
  const int main_lab = lab[s_main_pos];
  for (int i = threadIdx.x; i < nw; i += blockDim.x) main_mask[i] = lab[i] == main_lab;
}

// max over the PSF of psf x (label != main): main-lobe pixels count as +0
__global__ void __launch_bounds__(AM_THREADS) k_sidelobe_partial(const void *psf, int dt,
                                                                 int64_t ny, int64_t nx,
                                                                 const LobeInfo *info,
                                                                 const uint8_t *main_mask,
                                                                 double *part) {
  const LobeInfo li = *info;
  double m = -INFINITY;
  bool nan = false;
  if (li.mode == 0) {
    const int64_t n = ny * nx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
      double v = ld_real(psf, dt, i);
      const int64_t r = i / nx, c = i - (i / nx) * nx;
      if (r >= li.r0 && r < li.r0 + li.wr && c >= li.c0 && c < li.c0 + li.wc &&
          main_mask[(r - li.r0) * li.wc + (c - li.c0)])
        v = 0.0;
      if (isnan(v)) nan = true;
      else if (v > m) m = v;
    }
  }
  __shared__ double sh[32];
  __shared__ int shn;
  if (threadIdx.x == 0) shn = 0;
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  __syncthreads();
  if (nan) shn = 1;
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = -INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    part[blockIdx.x] = shn ? (double)NAN : r;
  }
}

__global__ void k_sidelobe_final(const double *part, int np, const LobeInfo *info,
                                 double *out) {
  if (threadIdx.x != 0) return;
  const LobeInfo li = *info;
  if (li.mode == 1) {
    out[0] = 0.0;
    out[1] = 0.0;
    return;
  }
  if (li.mode == 2) {
    out[0] = NAN;
    out[1] = (double)li.err;
    return;
  }
  double r = -INFINITY;
  bool nan = false;
  for (int i = 0; i < np; ++i) {
    if (isnan(part[i])) nan = true;
    else r = fmax(r, part[i]);
  }
  out[0] = nan ? (double)NAN : r;
  out[1] = 0.0;
}

// ----------------------------------------------------------- plane sums -----
constexpr int PS_THREADS = 256;

__global__ void __launch_bounds__(PS_THREADS) k_plane_sum_partial(const void *x, int dt,
                                                                  int64_t n_pix, double *part) {
  const int64_t plane = blockIdx.y;
  const void *base = dt == AV_F32 ? (const void *)((const float *)x + plane * n_pix)
                                  : (const void *)((const double *)x + plane * n_pix);
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pix;
       i += (int64_t)gridDim.x * blockDim.x)
    s += ld_real(base, dt, i);
  __shared__ double sh[32];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
    part[plane * gridDim.x + blockIdx.x] = r;
  }
}

__global__ void k_plane_sum_final(const double *part, int nb, int64_t n_planes, double *out) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n_planes) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[p * nb + b];
  out[p] = s;
}

static int plane_sum_blocks(int64_t n_pix) {
  int64_t b = (n_pix + PS_THREADS * 16 - 1) / (PS_THREADS * 16);
  if (b > 64) b = 64;
  if (b < 1) b = 1;
  return (int)b;
}

// ----------------------------------------------------------- residual ------
__global__ void k_vis_residual_c64(const float2 *a, const float2 *b, float2 *out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 x = a[i], y = b[i];
    out[i] = make_float2(__fsub_rn(x.x, y.x), __fsub_rn(x.y, y.y));
  }
}

__global__ void k_vis_residual_c128(const double2 *a, const double2 *b, double2 *out,
                                    int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 x = a[i], y = b[i];
    out[i] = make_double2(__dsub_rn(x.x, y.x), __dsub_rn(x.y, y.y));
  }
}

static unsigned stride_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// ------------------------------------------------ plane normalisation ---
// correct_fft_to_uv / correct_ifft_to_lm (standard_image_grid_preparation.py:
// 380-492) on x (n_planes, n_pix), real or complex, in place and in numpy's
// arithmetic for an array updated by a scalar:
//   mode 0, x /= s: a real x divided by s; a complex x (a, b) scaled as numpy
//     divides by the complex (s, 0): ((a + b*0) * r, (b - a*0) * r), r = 1/s,
//     all in the data's precision;
//   mode 1, x *= s: a real x times s; a complex x times (s, 0):
//     (a*s - b*0, a*0 + b*s), in the data's precision (s, a pixel count, is
//     exact in FP32 up to 2^24);
//   mode 2, x *= f with f = s / (corr[i] * w[plane]) rounded in FP64 and the
//     product formed in FP64 (as mode 1's formula for a complex x), then
//     rounded to the data's precision.
// The signs of zeros and the NaNs of infinite parts follow from these
// formulas, so they are written with the rounding intrinsics, uncontracted.
__device__ __forceinline__ float r_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double r_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float r_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double r_sub(double a, double b) { return __dsub_rn(a, b); }

template <typename R>
__device__ __forceinline__ void cplx_scale(R &a, R &b, R f) {
  const R z = R(0);
  const R re = r_sub(r_mul(a, f), r_mul(b, z));
  const R im = r_add(r_mul(a, z), r_mul(b, f));
  a = re;
  b = im;
}

template <typename T, int COMPS>
__global__ void __launch_bounds__(256) k_plane_rescale(T *x, int64_t n_planes, int64_t n_pix,
                                                       int mode, double s, const double *corr,
                                                       const double *w) {
  const int64_t n = n_planes * n_pix;
  const T st = (T)s;
  const T rt = r_div(T(1), st);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (COMPS == 1) {
      if (mode == 0) {
        x[e] = r_div(x[e], st);
      } else if (mode == 1) {
        x[e] = r_mul(x[e], st);
      } else {
        const int64_t pl = e / n_pix, i = e - pl * n_pix;
        const double f = __ddiv_rn(s, __dmul_rn(corr[i], w[pl]));
        x[e] = (T)__dmul_rn((double)x[e], f);
      }
    } else {
      T a = x[2 * e], b = x[2 * e + 1];
      if (mode == 0) {
        const T z = T(0);
        const T re = r_mul(r_add(a, r_mul(b, z)), rt);
        const T im = r_mul(r_sub(b, r_mul(a, z)), rt);
        a = re;
        b = im;
      } else if (mode == 1) {
        cplx_scale<T>(a, b, st);
      } else {
        const int64_t pl = e / n_pix, i = e - pl * n_pix;
        const double f = __ddiv_rn(s, __dmul_rn(corr[i], w[pl]));
        double ad = (double)a, bd = (double)b;
        cplx_scale<double>(ad, bd, f);
        a = (T)ad;
        b = (T)bd;
      }
      x[2 * e] = a;
      x[2 * e + 1] = b;
    }
  }
}

// ------------------------------------------------------ primary beam ---
// _mult_div of apply_pb (standard_image_grid_preparation.py:236-309): x
// (nt, nc, np, n_pix) times or divided by pb (pt, pc, pp, n_pix), in place;
// pb's plane is (t, c, p) with each index 0 where pb's extent differs from
// x's.  numpy's arithmetic for x op= pb: computed in P, the promoted real
// precision of the two, then rounded to x's type.  A complex x is multiplied
// as by the complex (p, 0), (a*p - b*0, a*0 + b*p), and divided by it with
// numpy's complex division, ((a + b*q) * g, (b - a*q) * g), q = 0/p,
// g = 1/(p + 0*q).  Division by a pb of 0 (either sign) leaves NaN, and
// (NaN, 0) for a complex x, as the reference's NaN fill does.
template <typename TX, typename TP, typename P, int COMPS>
__global__ void __launch_bounds__(256) k_apply_pb(TX *x, const TP *pb, int64_t nt, int64_t nc,
                                                  int64_t npl, int64_t pt, int64_t pc,
                                                  int64_t pp, int64_t n_pix, int multiply) {
  const int64_t n = nt * nc * npl * n_pix;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pl = e / n_pix, i = e - pl * n_pix;
    const int64_t p = pl % npl, tc = pl / npl;
    const int64_t c = tc % nc, t = tc / nc;
    const int64_t tu = (pt == nt) ? t : 0, cu = (pc == nc) ? c : 0, pu = (pp == npl) ? p : 0;
    const P w = (P)pb[((tu * pc + cu) * pp + pu) * n_pix + i];
    const P z = P(0);
    const bool zero_fill = !multiply && w == z;
    if (COMPS == 1) {
      const P a = (P)x[e];
      P r = multiply ? r_mul(a, w) : r_div(a, w);
      if (zero_fill) r = (P)__int_as_float(0x7fc00000);  // a quiet NaN
      x[e] = (TX)r;
    } else {
      const P a = (P)x[2 * e], b = (P)x[2 * e + 1];
      P re, im;
      if (multiply) {
        re = r_sub(r_mul(a, w), r_mul(b, z));
        im = r_add(r_mul(a, z), r_mul(b, w));
      } else if (zero_fill) {
        re = (P)__int_as_float(0x7fc00000);
        im = z;
      } else {
        const P q = r_div(z, w);
        const P g = r_div(P(1), r_add(w, r_mul(z, q)));
        re = r_mul(r_add(a, r_mul(b, q)), g);
        im = r_mul(r_sub(b, r_mul(a, q)), g);
      }
      x[2 * e] = (TX)re;
      x[2 * e + 1] = (TX)im;
    }
  }
}

template <typename TX, typename TP, typename P, int COMPS>
static void launch_apply_pb(void *x, const void *pb, int64_t nt, int64_t nc, int64_t npl,
                            int64_t pt, int64_t pc, int64_t pp, int64_t n_pix, int multiply,
                            cudaStream_t st) {
  const unsigned blocks = stride_blocks(nt * nc * npl * n_pix, 256);
  k_apply_pb<TX, TP, P, COMPS><<<blocks, 256, 0, st>>>((TX *)x, (const TP *)pb, nt, nc, npl, pt,
                                                       pc, pp, n_pix, multiply);
}

}  // namespace av

using namespace av;

extern "C" {

int av_plane_rescale(void *x, int dtype, int64_t n_planes, int64_t n_pix, int mode, double s,
                     const double *corr, const double *w, void *stream) {
  clear_error();
  AV_CHECK_ARG(x, "av_plane_rescale: null pointer");
  AV_CHECK_ARG(dtype >= AV_F32 && dtype <= AV_C128, "av_plane_rescale: dtype");
  AV_CHECK_ARG(mode >= 0 && mode <= 2, "av_plane_rescale: mode must be 0, 1 or 2");
  AV_CHECK_ARG(mode != 2 || (corr && w), "av_plane_rescale: mode 2 needs corr and w");
  AV_CHECK_ARG(n_planes >= 0 && n_pix >= 0, "av_plane_rescale: bad shape");
  const int64_t n = n_planes * n_pix;
  if (n == 0) return AV_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned blocks = stride_blocks(n, 256);
  if (dtype == AV_F32)
    k_plane_rescale<float, 1><<<blocks, 256, 0, st>>>((float *)x, n_planes, n_pix, mode, s, corr, w);
  else if (dtype == AV_F64)
    k_plane_rescale<double, 1><<<blocks, 256, 0, st>>>((double *)x, n_planes, n_pix, mode, s, corr,
                                                       w);
  else if (dtype == AV_C64)
    k_plane_rescale<float, 2><<<blocks, 256, 0, st>>>((float *)x, n_planes, n_pix, mode, s, corr, w);
  else
    k_plane_rescale<double, 2><<<blocks, 256, 0, st>>>((double *)x, n_planes, n_pix, mode, s, corr,
                                                       w);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_apply_pb(void *x, int x_dtype, int64_t nt, int64_t nc, int64_t npl, const void *pb,
                int pb_dtype, int64_t pt, int64_t pc, int64_t pp, int64_t n_pix, int multiply,
                void *stream) {
  clear_error();
  AV_CHECK_ARG(x && pb, "av_apply_pb: null pointer");
  AV_CHECK_ARG(x_dtype >= AV_F32 && x_dtype <= AV_C128, "av_apply_pb: image dtype");
  AV_CHECK_ARG(pb_dtype == AV_F32 || pb_dtype == AV_F64,
               "av_apply_pb: the primary beam must be AV_F32 or AV_F64");
  AV_CHECK_ARG(nt >= 0 && nc >= 0 && npl >= 0 && n_pix >= 0, "av_apply_pb: bad image shape");
  AV_CHECK_ARG(pt >= 1 && pc >= 1 && pp >= 1, "av_apply_pb: bad primary-beam shape");
  if (nt * nc * npl * n_pix == 0) return AV_OK;
  cudaStream_t st = as_stream(stream);
  const bool pb64 = pb_dtype == AV_F64;
  switch (x_dtype) {
    case AV_F32:
      if (pb64) launch_apply_pb<float, double, double, 1>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                          multiply, st);
      else launch_apply_pb<float, float, float, 1>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                   multiply, st);
      break;
    case AV_F64:
      if (pb64) launch_apply_pb<double, double, double, 1>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                           multiply, st);
      else launch_apply_pb<double, float, double, 1>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                     multiply, st);
      break;
    case AV_C64:
      if (pb64) launch_apply_pb<float, double, double, 2>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                          multiply, st);
      else launch_apply_pb<float, float, float, 2>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                   multiply, st);
      break;
    default:
      if (pb64) launch_apply_pb<double, double, double, 2>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                           multiply, st);
      else launch_apply_pb<double, float, double, 2>(x, pb, nt, nc, npl, pt, pc, pp, n_pix,
                                                     multiply, st);
  }
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_pol_transform(const void *in, int in_dtype, void *out, int out_dtype,
                     const double *matrix, int n_in, int n_out, int64_t n_outer, int64_t n_pix,
                     void *stream) {
  clear_error();
  AV_CHECK_ARG(in && out && matrix, "av_pol_transform: null pointer");
  AV_CHECK_ARG(n_in >= 1 && n_in <= 4 && n_out >= 1 && n_out <= 4,
               "av_pol_transform: n_in and n_out must be in [1, 4]");
  AV_CHECK_ARG(in_dtype >= AV_F32 && in_dtype <= AV_C128 && out_dtype >= AV_F32 &&
                   out_dtype <= AV_C128,
               "av_pol_transform: dtype");
  AV_CHECK_ARG(n_outer >= 0 && n_pix >= 0, "av_pol_transform: bad shape");
  if (n_outer == 0 || n_pix == 0) return AV_OK;
  PolMatrix m;
  m.n_in = n_in;
  m.n_out = n_out;
  for (int i = 0; i < 16; ++i) m.re[i] = m.im[i] = 0.0;
  for (int i = 0; i < n_in * n_out; ++i) {
    m.re[i] = matrix[2 * i];
    m.im[i] = matrix[2 * i + 1];
  }
  k_pol_transform<<<stride_blocks(n_outer * n_pix, 256), 256, 0, as_stream(stream)>>>(
      in, in_dtype, out, out_dtype, m, n_outer, n_pix);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_argmax_workspace_size(int64_t n) { return argmax_ws(n < 1 ? 1 : n); }

int av_argmax(const void *x, int dtype, int64_t n, int mode, int64_t *out_index,
              double *out_value, void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(x && out_index && out_value, "av_argmax: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_argmax: dtype must be F32 or F64");
  AV_CHECK_ARG(mode == 0 || mode == 1, "av_argmax: mode must be 0 (|x|) or 1 (x)");
  AV_CHECK_ARG(n >= 1, "av_argmax: empty input");
  Workspace ws(workspace, workspace_bytes);
  ArgMax *part = ws.take<ArgMax>(argmax_blocks(n));
  AV_CHECK_ARG(part, "av_argmax: workspace too small");
  return launch_argmax(x, dtype, n, mode, out_index, out_value, part, as_stream(stream));
}

size_t av_psf_sidelobe_workspace_size(int64_t ny, int64_t nx, int win0, int win1) {
  const int64_t n = ny * nx;
  size_t b = argmax_ws(n < 1 ? 1 : n);
  b += Workspace::need(sizeof(int64_t) + sizeof(double) * 2);
  b += Workspace::need(sizeof(LobeInfo));
  b += Workspace::need((size_t)(win0 > 0 ? win0 : 1) * (win1 > 0 ? win1 : 1));
  b += Workspace::need(sizeof(double) * (size_t)argmax_blocks(n < 1 ? 1 : n));
  return b;
}

int av_psf_sidelobe(const void *psf, int dtype, int64_t ny, int64_t nx, int win0, int win1,
                    double threshold, double *out, void *workspace, size_t workspace_bytes,
                    void *stream) {
  clear_error();
  AV_CHECK_ARG(psf && out, "av_psf_sidelobe: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_psf_sidelobe: dtype must be F32 or F64");
  AV_CHECK_ARG(ny >= 1 && nx >= 1, "av_psf_sidelobe: bad shape");
  AV_CHECK_ARG(win0 >= 1 && win1 >= 1, "av_psf_sidelobe: window must be positive");
  AV_CHECK_ARG((int64_t)(win0 / 2 * 2 + 1) * (win1 / 2 * 2 + 1) <= 16384,
               "av_psf_sidelobe: window of %d x %d exceeds the one-CTA labelling limit", win0,
               win1);
  cudaStream_t st = as_stream(stream);
  const int64_t n = ny * nx;
  Workspace ws(workspace, workspace_bytes);
  ArgMax *part = ws.take<ArgMax>(argmax_blocks(n));
  char *pk = ws.take<char>(sizeof(int64_t) + sizeof(double) * 2);
  LobeInfo *info = ws.take<LobeInfo>(1);
  uint8_t *mask = ws.take<uint8_t>((size_t)win0 * win1);
  double *spart = ws.take<double>(argmax_blocks(n));
  AV_CHECK_ARG(part && pk && info && mask && spart, "av_psf_sidelobe: workspace too small");
  int64_t *pidx = (int64_t *)pk;
  double *pval = (double *)(pk + sizeof(int64_t));
  int rc = launch_argmax(psf, dtype, n, 1, pidx, pval, part, st);
  if (rc) return rc;
  // window extent at most (win0/2*2) x (win1/2*2) pixels
  const int wmax = (win0 / 2 * 2 + 1) * (win1 / 2 * 2 + 1);
  const size_t smem = (size_t)wmax * (sizeof(double) + sizeof(int));
  if (smem > 48 * 1024)
    AV_CUDA(cudaFuncSetAttribute(k_psf_lobe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_psf_lobe<<<1, LOBE_THREADS, smem, st>>>(psf, dtype, ny, nx, win0, win1, threshold, pidx,
                                            pval, info, mask);
  AV_LAUNCH_CHECK();
  const int nb = argmax_blocks(n);
  k_sidelobe_partial<<<nb, AM_THREADS, 0, st>>>(psf, dtype, ny, nx, info, mask, spart);
  AV_LAUNCH_CHECK();
  k_sidelobe_final<<<1, 32, 0, st>>>(spart, nb, info, out);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_plane_sum_workspace_size(int64_t n_planes, int64_t n_pix) {
  return Workspace::need(sizeof(double) * (size_t)(n_planes < 1 ? 1 : n_planes) *
                         plane_sum_blocks(n_pix < 1 ? 1 : n_pix));
}

int av_plane_sum(const void *x, int dtype, int64_t n_planes, int64_t n_pix, double *out,
                 void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(x && out, "av_plane_sum: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_plane_sum: dtype must be F32 or F64");
  AV_CHECK_ARG(n_planes >= 1 && n_planes <= 65535 && n_pix >= 1, "av_plane_sum: bad shape");
  Workspace ws(workspace, workspace_bytes);
  const int nb = plane_sum_blocks(n_pix);
  double *part = ws.take<double>((size_t)n_planes * nb);
  AV_CHECK_ARG(part, "av_plane_sum: workspace too small");
  cudaStream_t st = as_stream(stream);
  k_plane_sum_partial<<<dim3(nb, (unsigned)n_planes), PS_THREADS, 0, st>>>(x, dtype, n_pix,
                                                                           part);
  AV_LAUNCH_CHECK();
  k_plane_sum_final<<<(unsigned)((n_planes + 127) / 128), 128, 0, st>>>(part, nb, n_planes,
                                                                       out);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_vis_residual(const void *vis, const void *model, void *out, int dtype, int64_t n,
                    void *stream) {
  clear_error();
  AV_CHECK_ARG(vis && model && out, "av_vis_residual: null pointer");
  AV_CHECK_ARG(dtype == AV_C64 || dtype == AV_C128, "av_vis_residual: dtype must be C64 or C128");
  AV_CHECK_ARG(n >= 0, "av_vis_residual: bad size");
  if (n == 0) return AV_OK;
  cudaStream_t st = as_stream(stream);
  if (dtype == AV_C64)
    k_vis_residual_c64<<<stride_blocks(n, 256), 256, 0, st>>>(
        (const float2 *)vis, (const float2 *)model, (float2 *)out, n);
  else
    k_vis_residual_c128<<<stride_blocks(n, 256), 256, 0, st>>>(
        (const double2 *)vis, (const double2 *)model, (double2 *)out, n);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"
