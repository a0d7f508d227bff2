// Mosaic / A-projection gridding with general convolution functions
// (mosaic_grid.py): each sample's footprint is a window of a 2-D complex
// convolution function chosen by (baseline, channel, polarisation) maps,
// premultiplied by the field's phase gradient.
//
// av_mosaic_grid      mosaic_grid_jit (mosaic_grid.py:307-486): one warp per
//                     (time, baseline, channel) sample, lanes over the
//                     support window, FP64 atomics into the grid; the
//                     window's norm is reduced in the warp for sum_weight.
// av_aperture_grid    aperture_grid_jit (mosaic_grid.py:13-153): every
//                     sample adds its function at the grid centre, so the
//                     weights are first summed per (function baseline,
//                     channel, polarisation) class and each class then adds
//                     its function once.
// av_cf_phase_product conv_kernel x phase_gradient[0] (mosaic_grid.py:384,
//                     :56-58), elementwise without fused multiply-add.
#include "plan.cuh"

namespace av {

struct MosaicArgs {
  double2 *grid;
  double *sumw;
  int do_psf;
  const double2 *vis;      // (nt, nb, nchan, npol), NULL for do_psf
  const double *wt;        // (nt, nb, nchan, npol)
  const double *uvw, *freq;
  const int32_t *chan_map, *pol_map, *cfb_map, *cfc_map, *cfp_map;
  const double2 *cf;       // (n_cfb, n_cfc, n_cfp, cu, cv), phase gradient applied
  int64_t n_cfb, n_cfc, n_cfp, cu, cv;
  const int32_t *support;  // (n_cfb, n_cfc, n_cfp, 2)
  int max_support;         // np.max(weight_support)
  int64_t n_u, n_v;
  double dl0, dl1;
  int os_u, os_v;
  int64_t nt, nb, nchan, npol, n_img_chan, n_img_pol;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// Position of a sample (mosaic_grid.py:384-405): centre cell and the offset
// index into the function; false when off the grid or NaN.
__device__ __forceinline__ bool mosaic_pos(const MosaicArgs &a, int64_t tb, int64_t c,
                                           long long &uc, long long &vc, long long &uo,
                                           long long &vo) {
  const double f = a.freq[c];
  const double s0 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, a.dl0), (double)a.n_u), C_LIGHT);
  const double s1 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, a.dl1), (double)a.n_v), C_LIGHT);
  const double u = __dmul_rn(a.uvw[3 * tb], s0), v = __dmul_rn(a.uvw[3 * tb + 1], s1);
  if (isnan(u) || isnan(v)) return false;
  const double up = __dadd_rn(u, (double)(a.n_u / 2)), vp = __dadd_rn(v, (double)(a.n_v / 2));
  uc = trunc_ll(__dadd_rn(up, 0.5));
  vc = trunc_ll(__dadd_rn(vp, 0.5));
  const long long ms = a.max_support;
  if (!(uc + ms < a.n_u && vc + ms < a.n_v && uc - ms >= 0 && vc - ms >= 0)) return false;
  uo = (long long)floor(__dadd_rn(__dmul_rn(__dsub_rn((double)uc, up), (double)a.os_u), 0.5)) +
       a.cu / 2;
  vo = (long long)floor(__dadd_rn(__dmul_rn(__dsub_rn((double)vc, vp), (double)a.os_v), 0.5)) +
       a.cv / 2;
  return true;
}

constexpr int MG_THREADS = 256;

__global__ void __launch_bounds__(MG_THREADS) k_mosaic_grid(MosaicArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t n_rows = a.nt * a.nb * a.nchan;
  for (int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; row < n_rows;
       row += n_warps) {
    const int64_t tb = row / a.nchan;
    const int64_t c = row - tb * a.nchan;
    const int64_t b = tb % a.nb;
    long long uc, vc, uo, vo;
    if (!mosaic_pos(a, tb, c, uc, vc, uo, vo)) continue;
    const int cfb = a.cfb_map[b], cfc = a.cfc_map[c], ach = a.chan_map[c];
    if (ach < 0 || ach >= a.n_img_chan || cfb < 0 || cfb >= a.n_cfb || cfc < 0 ||
        cfc >= a.n_cfc)
      continue;
    for (int64_t p = 0; p < a.npol; ++p) {
      const int64_t k = row * a.npol + p;
      const double w = a.wt[k];
      double2 wd;
      if (a.do_psf) wd = make_double2(w, 0.0);
      else {
        const double2 vv = a.vis[k];
        wd = make_double2(__dmul_rn(vv.x, w), __dmul_rn(vv.y, w));
      }
      if (isnan(wd.x) || isnan(wd.y) || (wd.x == 0.0 && wd.y == 0.0)) continue;
      const int cfp = a.cfp_map[p], apol = a.pol_map[p];
      if (cfp < 0 || cfp >= a.n_cfp || apol < 0 || apol >= a.n_img_pol) continue;
      const int64_t fidx = ((int64_t)cfb * a.n_cfc + cfc) * a.n_cfp + cfp;
      const int su = a.support[2 * fidx], sv = a.support[2 * fidx + 1];
      const int su0 = -(su / 2), sv0 = -(sv / 2);
      const double2 *f = a.cf + fidx * a.cu * a.cv;
      double2 *g = a.grid + ((int64_t)ach * a.n_img_pol + apol) * a.n_u * a.n_v;
      double2 norm = make_double2(0.0, 0.0);
      const int n_tap = su * sv;
      for (int t0 = 0; t0 < n_tap; t0 += 32) {
        const int t = t0 + lane;
        if (t >= n_tap) continue;
        const int iv = sv0 + t / su, iu = su0 + t % su;  // v outer, u inner
        const long long fu = (long long)a.os_u * iu + uo, fv = (long long)a.os_v * iv + vo;
        // a window reaching past the function (the reference reads beyond it)
        if (fu < 0 || fu >= a.cu || fv < 0 || fv >= a.cv) continue;
        const double2 conv = f[fu * a.cv + fv];
        const double2 x = cmul(conv, wd);
        double2 *cell = g + (uc + iu) * a.n_v + (vc + iv);
        atomicAdd(&cell->x, x.x);
        atomicAdd(&cell->y, x.y);
        norm.x += conv.x;
        norm.y += conv.y;
      }
      for (int off = 16; off > 0; off >>= 1) {
        norm.x += __shfl_down_sync(0xffffffffu, norm.x, off);
        norm.y += __shfl_down_sync(0xffffffffu, norm.y, off);
      }
      if (lane == 0 && a.sumw) {
        // do_psf: w Re(norm); else w Re(norm^2) (the function enters twice)
        const double re = a.do_psf ? norm.x
                                   : __dsub_rn(__dmul_rn(norm.x, norm.x), __dmul_rn(norm.y, norm.y));
        atomicAdd(&a.sumw[(int64_t)ach * a.n_img_pol + apol], __dmul_rn(w, re));
      }
    }
  }
}

// aperture_grid_jit, pass 1: weight sums per (function baseline, channel,
// polarisation) class over the samples that pass the grid bounds.
__global__ void __launch_bounds__(MG_THREADS) k_aperture_classes(MosaicArgs a, double *cls) {
  const int64_t n_rows = a.nt * a.nb * a.nchan;
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n_rows;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int64_t tb = row / a.nchan;
    const int64_t c = row - tb * a.nchan;
    const int64_t b = tb % a.nb;
    long long uc, vc, uo, vo;
    if (!mosaic_pos(a, tb, c, uc, vc, uo, vo)) continue;
    const int cfb = a.cfb_map[b];
    if (cfb < 0 || cfb >= a.n_cfb) continue;
    for (int64_t p = 0; p < a.npol; ++p) {
      const double w = a.wt[row * a.npol + p];
      if (isnan(w) || w == 0.0) continue;
      atomicAdd(&cls[((int64_t)cfb * a.nchan + c) * a.npol + p], w);
    }
  }
}

// pass 2: one block per class adds w_class x function window at the grid
// centre and w_class x Re(norm) to sum_weight.
__global__ void __launch_bounds__(MG_THREADS) k_aperture_add(MosaicArgs a, const double *cls) {
  const int64_t cl = blockIdx.x;
  const double w = cls[cl];
  if (w == 0.0) return;
  const int64_t p = cl % a.npol;
  const int64_t c = (cl / a.npol) % a.nchan;
  const int64_t cfb = cl / (a.npol * a.nchan);
  const int cfc = a.cfc_map[c], cfp = a.cfp_map[p], ach = a.chan_map[c], apol = a.pol_map[p];
  if (cfc < 0 || cfc >= a.n_cfc || cfp < 0 || cfp >= a.n_cfp || ach < 0 ||
      ach >= a.n_img_chan || apol < 0 || apol >= a.n_img_pol)
    return;
  const int64_t fidx = (cfb * a.n_cfc + cfc) * a.n_cfp + cfp;
  const int su = a.support[2 * fidx], sv = a.support[2 * fidx + 1];
  const int su0 = -(su / 2), sv0 = -(sv / 2);
  const double2 *f = a.cf + fidx * a.cu * a.cv;
  double2 *g = a.grid + ((int64_t)ach * a.n_img_pol + apol) * a.n_u * a.n_v;
  double2 norm = make_double2(0.0, 0.0);
  const int n_tap = su * sv;
  for (int t0 = 0; t0 < n_tap; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    if (t >= n_tap) continue;
    const int iv = sv0 + t / su, iu = su0 + t % su;
    const long long fu = (long long)a.os_u * iu + a.cu / 2, fv = (long long)a.os_v * iv + a.cv / 2;
    const long long gu = a.n_u / 2 + iu, gv = a.n_v / 2 + iv;
    if (fu < 0 || fu >= a.cu || fv < 0 || fv >= a.cv || gu < 0 || gu >= a.n_u || gv < 0 ||
        gv >= a.n_v)
      continue;
    const double2 conv = f[fu * a.cv + fv];
    double2 *cell = g + gu * a.n_v + gv;
    atomicAdd(&cell->x, __dmul_rn(conv.x, w));
    atomicAdd(&cell->y, __dmul_rn(conv.y, w));
    norm.x += conv.x;
  }
  __shared__ double sh[MG_THREADS / 32];
  double s = norm.x;
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0 && a.sumw) {
    double r = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
    atomicAdd(&a.sumw[(int64_t)ach * a.n_img_pol + apol], __dmul_rn(w, r));
  }
}

__global__ void k_cf_phase_product(const void *kern, int kern_complex, const double2 *pg,
                                   double2 *out, int64_t n_cf, int64_t n_pix) {
  const int64_t n = n_cf * n_pix;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double2 g = pg[i % n_pix];
    if (kern_complex) {
      out[i] = cmul(((const double2 *)kern)[i], g);
    } else {
      const double r = ((const double *)kern)[i];
      out[i] = make_double2(__dmul_rn(r, g.x), __dmul_rn(r, g.y));
    }
  }
}

// Airy-disk primary beams (make_pb_symmetric.py:1-280), one value per
// thread in the reference's operation order; J1 is CUDA's j1.
struct AiryArgs {
  double *out;
  int64_t n_dish, n_freq, nx, ny, cx, cy, n_pol;
  double cell_x, cell_y;
  int ipower, casa, rorder;
  double dish[16], block[16];
  const double *freq;
};

__global__ void k_airy_pattern(AiryArgs a) {
  const int64_t n = a.n_dish * a.n_freq * a.nx * a.ny;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t iy = t % a.ny;
    const int64_t ix = (t / a.ny) % a.nx;
    const int64_t f = (t / (a.ny * a.nx)) % a.n_freq;
    const int64_t d = t / (a.ny * a.nx * a.n_freq);
    double v = 1.0;
    if (!(ix == a.cx && iy == a.cy)) {
      const double x = __dmul_rn((double)(ix - a.cx), a.cell_x);
      const double y = __dmul_rn((double)(iy - a.cy), a.cell_y);
      const double k = __ddiv_rn(__dmul_rn(2.0 * 3.141592653589793, a.freq[f]), C_LIGHT);
      const double r = __dmul_rn(__dmul_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(x, x),
                                                                 __dmul_rn(y, y))), k),
                                 __ddiv_rn(a.dish[d], 2.0));
      const double dd = a.dish[d], bd = a.block[d];
      if (bd == 0.0) {
        v = __ddiv_rn(__dmul_rn(2.0, j1(r)), r);
      } else if (!a.casa) {
        const double e = __ddiv_rn(bd, dd);
        const double t1 = __ddiv_rn(__dmul_rn(2.0, j1(r)), r);
        const double t2 = __ddiv_rn(__dmul_rn(__dmul_rn(2.0, e), j1(__dmul_rn(r, e))), r);
        v = __ddiv_rn(__dsub_rn(t1, t2), __dsub_rn(1.0, __dmul_rn(e, e)));
      } else {
        const double lr = __ddiv_rn(dd, bd);
        const double ar = __dmul_rn(lr, lr);
        const double t1 = __ddiv_rn(__dmul_rn(__dmul_rn(ar, 2.0), j1(r)), r);
        const double rl = __dmul_rn(r, lr);
        const double t2 = __ddiv_rn(__dmul_rn(2.0, j1(rl)), rl);
        v = __ddiv_rn(__dsub_rn(t1, t2), __dsub_rn(ar, 1.0));
      }
      double p = v;
      for (int i = 1; i < a.ipower; ++i) p = __dmul_rn(p, v);
      v = a.ipower == 0 ? 1.0 : p;
    }
    for (int64_t q = 0; q < a.n_pol; ++q) {
      int64_t o;
      if (a.rorder)  // (dish, freq, pol, x, y)
        o = (((d * a.n_freq + f) * a.n_pol + q) * a.nx + ix) * a.ny + iy;
      else  // (x, y, freq, pol, dish)
        o = (((ix * a.ny + iy) * a.n_freq + f) * a.n_pol + q) * a.n_dish + d;
      a.out[o] = v;
    }
  }
}

// ----------------------------------------------------------------- tiled --
// Binned version of k_mosaic_grid: the gridder's plan (plan.cuh) with a
// footprint window of S = max_support cells and the mosaic's edge margin
// (np.max(weight_support)) holds every kept sample's cell and kernel offset;
// a persistent CTA per SM takes record chunks, keeps an FP64 complex
// sub-grid of (32 + S - 1)^2 x n_img_pol in shared memory per tile segment
// and flushes it once.  A warp takes one record at a time; its lanes cover
// the support window packed as (32 / su) rows of su columns.
constexpr int MT_THREADS = 512;
constexpr int MT_WARPS = MT_THREADS / 32;

// Unsigned 32-bit division by an invariant d (Granlund and Montgomery,
// "Division by invariant integers using multiplication", 1994): with
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, t = mulhi(m, n),
// n / d = (t + ((n - t) >> 1)) >> (l - 1); d = 1 uses m = 0 and no shifts.
struct FastDiv {
  uint32_t m;
  int s1, s2;
};

static FastDiv fast_div(uint32_t d) {
  FastDiv f{0u, 0, 0};
  if (d <= 1) return f;
  int l = 0;
  while ((1ull << l) < d) ++l;
  f.m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << l) - d)) / d + 1);
  f.s1 = 1;
  f.s2 = l - 1;
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  const uint32_t t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct MosaicTiledArgs {
  MosaicArgs m;
  FastDiv div_nchan, div_nb;  // row -> (time x baseline, channel), -> baseline
  const Rec *recs;
  const uint32_t *tile_start;
  const uint32_t *n_rec;
  uint32_t *sched;
  int64_t n_tiles, ntu, ntv, chunk;
  int S;   // footprint window (max_support)
  int W;   // sub-grid edge, TILE + S - 1
};

__global__ void __launch_bounds__(MT_THREADS, 1) k_mosaic_tiled(MosaicTiledArgs t) {
  const MosaicArgs &a = t.m;
  extern __shared__ __align__(16) unsigned char smem[];
  // real and imaginary planes [apol][W * W]: a warp's 8-byte atomics along a
  // window row fall on consecutive banks
  const int W = t.W, npg = (int)a.n_img_pol;
  const int sub_n = npg * W * W;
  double *sre = (double *)smem;
  double *sim = sre + sub_n;
  __shared__ int s_chunk;
  // lane packing of a window with sv columns: 32 / sv rows per pass, lane
  // ir = lane / sv (sv <= max_support <= 32)
  __shared__ unsigned char s_ir[33][32], s_rp[33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t n_rec = *t.n_rec;
  const int64_t n_chunks = ((int64_t)n_rec + t.chunk - 1) / t.chunk;
  const uint32_t nchan = (uint32_t)a.nchan, nb = (uint32_t)a.nb;
  for (int i = threadIdx.x; i < 33 * 32; i += MT_THREADS) {
    const int sv = i >> 5, l = i & 31;
    s_ir[sv][l] = (unsigned char)(sv ? l / sv : 0);
    if (l == 0) s_rp[sv] = (unsigned char)(sv ? 32 / sv : 0);
  }
  for (int i0 = 0; i0 < sub_n; i0 += MT_THREADS) {
    const int i = i0 + threadIdx.x;
    if (i < sub_n) {
      sre[i] = 0.0;
      sim[i] = 0.0;
    }
  }
  for (;;) {
    __syncthreads();  // sub-grid clear; previous s_chunk consumed
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(&t.sched[0], 1u);
    __syncthreads();
    const int64_t ch = s_chunk;
    if (ch >= n_chunks) break;
    const uint32_t r0 = (uint32_t)(ch * t.chunk);
    const uint32_t r1 = (uint32_t)min((int64_t)n_rec, (int64_t)r0 + t.chunk);
    int64_t lo = 0, hi = t.n_tiles;  // tile holding r0
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (t.tile_start[mid] <= r0) lo = mid; else hi = mid;
    }
    int64_t tile = lo;
    uint32_t seg_lo = r0;
    while (seg_lo < r1) {
      const uint32_t t_end = t.tile_start[tile + 1];
      const uint32_t seg_hi = min(r1, t_end);
      if (seg_hi <= seg_lo) {
        ++tile;
        continue;
      }
      const int64_t plane = tile / (t.ntu * t.ntv);
      const int64_t trem = tile - plane * t.ntu * t.ntv;
      const int tu = (int)(trem / t.ntv), tv = (int)(trem - (int64_t)tu * t.ntv);
      double swacc[4] = {0.0, 0.0, 0.0, 0.0};
      // one trip count per block: every warp reaches the barrier converged
      for (uint32_t rb = seg_lo; rb < seg_hi; rb += MT_WARPS) {
        const uint32_t r = rb + warp;
        if (r >= seg_hi) continue;
        const Rec rc = t.recs[r];
        const int64_t row = rc.row;
        const uint32_t tb = fdiv(rc.row, t.div_nchan);  // rows fit 32 bits (the plan checks)
        const uint32_t c = rc.row - tb * nchan;
        const uint32_t b = tb - fdiv(tb, t.div_nb) * nb;
        const int cfb = a.cfb_map[b], cfc = a.cfc_map[c];
        if (cfb < 0 || cfb >= a.n_cfb || cfc < 0 || cfc >= a.n_cfc) continue;
        const long long uo = (long long)rc.ou - 128 + a.cu / 2;
        const long long vo = (long long)rc.ov - 128 + a.cv / 2;
        const int cu0 = rc.du + t.S / 2, cv0 = rc.dv + t.S / 2;  // centre in the sub-grid
        // the window's norm depends on the function only (same sample): kept
        // for the next polarisation that uses the same function
        int64_t norm_fidx = -1;
        double2 norm_prev = make_double2(0.0, 0.0);
        for (int64_t p = 0; p < a.npol; ++p) {
          const int64_t k = row * a.npol + p;
          const double w = a.wt[k];
          double2 wd;
          if (a.do_psf) wd = make_double2(w, 0.0);
          else {
            const double2 vv = a.vis[k];
            wd = make_double2(__dmul_rn(vv.x, w), __dmul_rn(vv.y, w));
          }
          if (isnan(wd.x) || isnan(wd.y) || (wd.x == 0.0 && wd.y == 0.0)) continue;
          const int cfp = a.cfp_map[p], apol = a.pol_map[p];
          if (cfp < 0 || cfp >= a.n_cfp || apol < 0 || apol >= npg) continue;
          const int64_t fidx = ((int64_t)cfb * a.n_cfc + cfc) * a.n_cfp + cfp;
          const int su = a.support[2 * fidx], sv = a.support[2 * fidx + 1];
          // a window larger than the footprint the plan reserved would leave
          // the sub-grid: such functions are skipped (the host passes
          // max_support = np.max(support))
          if (su < 1 || sv < 1 || su > t.S || sv > t.S) continue;
          const double2 *f = a.cf + fidx * a.cu * a.cv;
          double *pre = sre + (size_t)apol * W * W, *pim = sim + (size_t)apol * W * W;
          // lanes along the window's v (contiguous) axis: lane = ir * sv + jv,
          // 32 / sv u-rows per pass
          const int rp = s_rp[sv];
          const int ir = s_ir[sv][lane];
          const int iv = -(sv / 2) + (lane - ir * sv);
          const long long fv = (long long)a.os_v * iv + vo;
          const bool v_ok = ir < rp && fv >= 0 && fv < a.cv;
          double2 norm = make_double2(0.0, 0.0);
          for (int iu0 = 0; iu0 < su; iu0 += rp) {
            const int iui = iu0 + ir;
            if (!v_ok || iui >= su) continue;
            const int iu = -(su / 2) + iui;
            const long long fu = (long long)a.os_u * iu + uo;
            if (fu < 0 || fu >= a.cu) continue;
            const double2 conv = __ldg(f + fu * a.cv + fv);
            const double2 x = cmul(conv, wd);
            const int cell = (cu0 + iu) * W + (cv0 + iv);
            atomicAdd(pre + cell, x.x);
            atomicAdd(pim + cell, x.y);
            norm.x += conv.x;
            norm.y += conv.y;
          }
          if (fidx == norm_fidx) {
            norm = norm_prev;
          } else {
            for (int off = 16; off > 0; off >>= 1) {
              norm.x += __shfl_down_sync(0xffffffffu, norm.x, off);
              norm.y += __shfl_down_sync(0xffffffffu, norm.y, off);
            }
            norm_fidx = fidx;
            norm_prev = norm;
          }
          const double re = a.do_psf ? norm.x
                                     : __dsub_rn(__dmul_rn(norm.x, norm.x),
                                                 __dmul_rn(norm.y, norm.y));
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q == apol) swacc[q] += __dmul_rn(w, re);
        }
      }
      if (lane == 0 && a.sumw)
        for (int q = 0; q < npg && q < 4; ++q)
          if (swacc[q] != 0.0) atomicAdd(&a.sumw[plane * npg + q], swacc[q]);
      __syncthreads();
      // flush the segment's sub-grid to the global grid and clear it
      for (int i0 = 0; i0 < sub_n; i0 += MT_THREADS) {
        const int i = i0 + threadIdx.x;
        if (i >= sub_n) continue;
        const double vr = sre[i], vi = sim[i];
        if (vr == 0.0 && vi == 0.0) continue;
        const int gp = i / (W * W);
        const int cell = i - gp * W * W;
        const int iu = cell / W, iv = cell - iu * W;
        const int64_t gu = (int64_t)tu * TILE + iu, gv = (int64_t)tv * TILE + iv;
        double2 *gd = a.grid + ((plane * npg + gp) * a.n_u + gu) * a.n_v + gv;
        atomicAdd(&gd->x, vr);
        atomicAdd(&gd->y, vi);
        sre[i] = 0.0;
        sim[i] = 0.0;
      }
      seg_lo = seg_hi;
      if (seg_hi == t_end) ++tile;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&t.sched[1], 1u) == gridDim.x - 1) {
      t.sched[0] = 0u;
      t.sched[1] = 0u;
      __threadfence();
    }
  }
}

static size_t mosaic_tiled_smem(int S, int64_t n_img_pol) {
  const int W = TILE + S - 1;
  return (size_t)W * W * (size_t)n_img_pol * sizeof(double2);
}

static int mosaic_geom(PlanGeom &g, Plan &p, int64_t n_u, int64_t n_v, int max_support,
                       int os, int64_t nt, int64_t nb, int64_t nchan, int64_t n_img_chan,
                       void *workspace, size_t workspace_bytes, const char *who) {
  AV_CHECK_ARG(max_support >= 1 && max_support <= 32, "%s: max_support must be in [1, 32]",
               who);
  AV_CHECK_ARG(os >= 1 && os <= 254, "%s: oversampling must be in [1, 254]", who);
  AV_CHECK_ARG(n_u > 2 * max_support && n_v > 2 * max_support && n_u < 131072 &&
                   n_v < 131072,
               "%s: grid size out of range", who);
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nchan >= 0 && n_img_chan >= 1, "%s: bad shape", who);
  AV_CHECK_ARG(workspace && (((uintptr_t)workspace) & 255) == 0,
               "%s: workspace must be 256-byte aligned", who);
  plan_geometry(g, nt, nb, nchan, n_img_chan, n_u, n_v, max_support, os);
  g.margin = max_support;
  g.convention = 0;
  g.chk_x = g.chk_y = 0;
  g.scale0 = g.scale1 = g.offset0 = g.offset1 = 0.0;
  const size_t need = plan_workspace_bytes(g);
  if (workspace_bytes < need) {
    set_error("%s: workspace %zu bytes < %zu needed", who, workspace_bytes, need);
    return AV_ERR_WORKSPACE;
  }
  Workspace ws(workspace, workspace_bytes);
  if (!plan_carve(g, ws, p)) {
    set_error("%s: workspace carve failed", who);
    return AV_ERR_WORKSPACE;
  }
  return AV_OK;
}

static unsigned mg_blocks(int64_t n_items, int per_block) {
  int64_t b = (n_items + per_block - 1) / per_block;
  const int64_t cap = (int64_t)sm_count() * 32;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

static int fill_mosaic(MosaicArgs &a, void *grid, double *sum_weight, int do_psf,
                       const void *vis, const double *weight, const double *uvw,
                       const double *freq, const int32_t *chan_map, const int32_t *pol_map,
                       const int32_t *cfb_map, const int32_t *cfc_map, const int32_t *cfp_map,
                       const void *cf, int64_t n_cfb, int64_t n_cfc, int64_t n_cfp,
                       int64_t conv_u, int64_t conv_v, const int32_t *support,
                       int max_support, int64_t n_u, int64_t n_v, double delta_l,
                       double delta_m, int os_u, int os_v, int64_t nt, int64_t nb,
                       int64_t nchan, int64_t npol, int64_t n_img_chan, int64_t n_img_pol) {
  a.grid = (double2 *)grid;
  a.sumw = sum_weight;
  a.do_psf = do_psf;
  a.vis = (const double2 *)vis;
  a.wt = weight;
  a.uvw = uvw;
  a.freq = freq;
  a.chan_map = chan_map;
  a.pol_map = pol_map;
  a.cfb_map = cfb_map;
  a.cfc_map = cfc_map;
  a.cfp_map = cfp_map;
  a.cf = (const double2 *)cf;
  a.n_cfb = n_cfb;
  a.n_cfc = n_cfc;
  a.n_cfp = n_cfp;
  a.cu = conv_u;
  a.cv = conv_v;
  a.support = support;
  a.max_support = max_support;
  a.n_u = n_u;
  a.n_v = n_v;
  a.dl0 = delta_l;
  a.dl1 = delta_m;
  a.os_u = os_u;
  a.os_v = os_v;
  a.nt = nt;
  a.nb = nb;
  a.nchan = nchan;
  a.npol = npol;
  a.n_img_chan = n_img_chan;
  a.n_img_pol = n_img_pol;
  return AV_OK;
}

}  // namespace av

using namespace av;

extern "C" {

int av_cf_phase_product(const void *conv_kernel, int kernel_dtype, const void *phase_gradient,
                        void *out, int64_t n_cf, int64_t conv_u, int64_t conv_v, void *stream) {
  clear_error();
  AV_CHECK_ARG(conv_kernel && phase_gradient && out, "av_cf_phase_product: null pointer");
  AV_CHECK_ARG(kernel_dtype == AV_F64 || kernel_dtype == AV_C128,
               "av_cf_phase_product: kernel must be float64 or complex128");
  AV_CHECK_ARG(n_cf >= 0 && conv_u >= 1 && conv_v >= 1, "av_cf_phase_product: bad shape");
  if (n_cf == 0) return AV_OK;
  const int64_t n = n_cf * conv_u * conv_v;
  k_cf_phase_product<<<mg_blocks(n, 256), 256, 0, as_stream(stream)>>>(
      conv_kernel, kernel_dtype == AV_C128, (const double2 *)phase_gradient, (double2 *)out,
      n_cf, conv_u * conv_v);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_airy_pattern(double *out, const double *dish_diameters, const double *blockage_diameters,
                    int64_t n_dish, const double *freq, int64_t n_freq, int64_t n_pol,
                    int64_t nx, int64_t ny, int64_t cx, int64_t cy, double cell_x,
                    double cell_y, int ipower, int casa, int rorder, void *stream) {
  clear_error();
  AV_CHECK_ARG(out && dish_diameters && blockage_diameters && freq,
               "av_airy_pattern: null pointer");
  AV_CHECK_ARG(n_dish >= 1 && n_dish <= 16, "av_airy_pattern: 1 to 16 dish types");
  AV_CHECK_ARG(n_freq >= 1 && n_pol >= 1 && nx >= 1 && ny >= 1 && ipower >= 0 && ipower <= 8,
               "av_airy_pattern: bad shape or power");
  AiryArgs a;
  a.out = out;
  a.n_dish = n_dish;
  a.n_freq = n_freq;
  a.nx = nx;
  a.ny = ny;
  a.cx = cx;
  a.cy = cy;
  a.n_pol = n_pol;
  a.cell_x = cell_x;
  a.cell_y = cell_y;
  a.ipower = ipower;
  a.casa = casa;
  a.rorder = rorder;
  a.freq = freq;
  for (int i = 0; i < 16; ++i) {
    a.dish[i] = i < n_dish ? dish_diameters[i] : 0.0;
    a.block[i] = i < n_dish ? blockage_diameters[i] : 0.0;
  }
  const int64_t n = n_dish * n_freq * nx * ny;
  k_airy_pattern<<<mg_blocks(n, 256), 256, 0, as_stream(stream)>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

#define AV_MOSAIC_PARAMS                                                                   \
  void *grid, double *sum_weight, int do_psf, const void *vis, const double *weight,       \
      const double *uvw, const double *freq, const int32_t *chan_map,                      \
      const int32_t *pol_map, const int32_t *cf_baseline_map, const int32_t *cf_chan_map,  \
      const int32_t *cf_pol_map, const void *cf, int64_t n_cf_baseline, int64_t n_cf_chan, \
      int64_t n_cf_pol, int64_t conv_u, int64_t conv_v, const int32_t *support,            \
      int max_support, int64_t n_u, int64_t n_v, double delta_l, double delta_m, int os_u, \
      int os_v, int64_t nt, int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,    \
      int64_t n_img_pol

static int check_mosaic(const char *who, AV_MOSAIC_PARAMS) {
  AV_CHECK_ARG(grid && weight && uvw && freq && chan_map && pol_map && cf_baseline_map &&
                   cf_chan_map && cf_pol_map && cf && support,
               "%s: null pointer", who);
  AV_CHECK_ARG(do_psf || vis, "%s: vis is required unless do_psf", who);
  AV_CHECK_ARG(n_cf_baseline >= 1 && n_cf_chan >= 1 && n_cf_pol >= 1 && conv_u >= 1 &&
                   conv_v >= 1,
               "%s: bad convolution-function shape", who);
  AV_CHECK_ARG(n_u >= 1 && n_v >= 1 && os_u >= 1 && os_v >= 1 && max_support >= 0,
               "%s: bad grid or oversampling", who);
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nchan >= 0 && npol >= 0 && n_img_chan >= 1 &&
                   n_img_pol >= 1,
               "%s: bad shape", who);
  return AV_OK;
}

int av_mosaic_grid(AV_MOSAIC_PARAMS, void *stream) {
  clear_error();
  int rc = check_mosaic("av_mosaic_grid", grid, sum_weight, do_psf, vis, weight, uvw, freq,
                        chan_map, pol_map, cf_baseline_map, cf_chan_map, cf_pol_map, cf,
                        n_cf_baseline, n_cf_chan, n_cf_pol, conv_u, conv_v, support,
                        max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt, nb, nchan,
                        npol, n_img_chan, n_img_pol);
  if (rc) return rc;
  const int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  MosaicArgs a;
  fill_mosaic(a, grid, sum_weight, do_psf, vis, weight, uvw, freq, chan_map, pol_map,
              cf_baseline_map, cf_chan_map, cf_pol_map, cf, n_cf_baseline, n_cf_chan, n_cf_pol,
              conv_u, conv_v, support, max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt,
              nb, nchan, npol, n_img_chan, n_img_pol);
  k_mosaic_grid<<<mg_blocks(rows, MG_THREADS / 32), MG_THREADS, 0, as_stream(stream)>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_mosaic_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u,
                                      int64_t n_v, int64_t n_img_chan, int max_support) {
  PlanGeom g;
  plan_geometry(g, nt, nb, nchan, n_img_chan, n_u, n_v, max_support < 1 ? 1 : max_support,
                100);
  return plan_workspace_bytes(g);
}

int av_mosaic_tiled_plan(const double *uvw, const double *freq, const int32_t *chan_map,
                         int64_t n_u, int64_t n_v, double delta_l, double delta_m,
                         int max_support, int oversampling, int64_t nt, int64_t nb,
                         int64_t nchan, int64_t n_img_chan, void *workspace,
                         size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(uvw && freq && chan_map, "av_mosaic_tiled_plan: null pointer");
  PlanGeom g;
  Plan p;
  int rc = mosaic_geom(g, p, n_u, n_v, max_support, oversampling, nt, nb, nchan, n_img_chan,
                       workspace, workspace_bytes, "av_mosaic_tiled_plan");
  if (rc) return rc;
  return plan_build(g, p, uvw, freq, chan_map, delta_l, delta_m, as_stream(stream));
}

int av_mosaic_tiled_execute(AV_MOSAIC_PARAMS, void *workspace, size_t workspace_bytes,
                            void *stream) {
  clear_error();
  int rc = check_mosaic("av_mosaic_tiled_execute", grid, sum_weight, do_psf, vis, weight, uvw,
                        freq, chan_map, pol_map, cf_baseline_map, cf_chan_map, cf_pol_map, cf,
                        n_cf_baseline, n_cf_chan, n_cf_pol, conv_u, conv_v, support,
                        max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt, nb, nchan,
                        npol, n_img_chan, n_img_pol);
  if (rc) return rc;
  AV_CHECK_ARG(os_u == os_v, "av_mosaic_tiled_execute: oversampling must be the same on u, v");
  AV_CHECK_ARG(n_img_pol <= 4, "av_mosaic_tiled_execute: at most 4 image polarisations");
  const size_t smem = mosaic_tiled_smem(max_support, n_img_pol);
  AV_CHECK_ARG(smem <= 220 * 1024,
               "av_mosaic_tiled_execute: sub-grid of %zu bytes exceeds shared memory", smem);
  PlanGeom g;
  Plan p;
  rc = mosaic_geom(g, p, n_u, n_v, max_support, os_u, nt, nb, nchan, n_img_chan, workspace,
                   workspace_bytes, "av_mosaic_tiled_execute");
  if (rc) return rc;
  const int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  MosaicTiledArgs t;
  fill_mosaic(t.m, grid, sum_weight, do_psf, vis, weight, uvw, freq, chan_map, pol_map,
              cf_baseline_map, cf_chan_map, cf_pol_map, cf, n_cf_baseline, n_cf_chan, n_cf_pol,
              conv_u, conv_v, support, max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt,
              nb, nchan, npol, n_img_chan, n_img_pol);
  t.recs = p.recs;
  t.tile_start = p.tile_start;
  t.n_rec = p.offs + g.n_keys();
  t.sched = p.counters;
  t.n_tiles = g.n_tiles();
  t.ntu = g.ntu;
  t.ntv = g.ntv;
  t.S = max_support;
  t.W = TILE + max_support - 1;
  t.div_nchan = fast_div((uint32_t)nchan);
  t.div_nb = fast_div((uint32_t)nb);
  const int sms = sm_count();
  int64_t chunk = (rows + (int64_t)sms * 16 - 1) / ((int64_t)sms * 16);
  if (chunk < 1024) chunk = 1024;
  t.chunk = chunk;
  int64_t nblocks = (rows + chunk - 1) / chunk;
  if (nblocks > sms) nblocks = sms;
  if (nblocks < 1) nblocks = 1;
  if (smem > 48 * 1024)
    AV_CUDA(cudaFuncSetAttribute(k_mosaic_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  k_mosaic_tiled<<<(unsigned)nblocks, MT_THREADS, smem, as_stream(stream)>>>(t);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_aperture_grid_workspace_size(int64_t n_cf_baseline, int64_t nchan, int64_t npol) {
  return Workspace::need(sizeof(double) * (size_t)(n_cf_baseline < 1 ? 1 : n_cf_baseline) *
                         (nchan < 1 ? 1 : nchan) * (npol < 1 ? 1 : npol));
}

int av_aperture_grid(AV_MOSAIC_PARAMS, void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  int rc = check_mosaic("av_aperture_grid", grid, sum_weight, 1, vis, weight, uvw, freq,
                        chan_map, pol_map, cf_baseline_map, cf_chan_map, cf_pol_map, cf,
                        n_cf_baseline, n_cf_chan, n_cf_pol, conv_u, conv_v, support,
                        max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt, nb, nchan,
                        npol, n_img_chan, n_img_pol);
  if (rc) return rc;
  const int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  const int64_t n_cls = n_cf_baseline * nchan * npol;
  AV_CHECK_ARG(n_cls <= 0x7fffffff, "av_aperture_grid: too many weight classes");
  Workspace ws(workspace, workspace_bytes);
  double *cls = ws.take<double>((size_t)n_cls);
  AV_CHECK_ARG(cls, "av_aperture_grid: workspace too small");
  MosaicArgs a;
  fill_mosaic(a, grid, sum_weight, 1, nullptr, weight, uvw, freq, chan_map, pol_map,
              cf_baseline_map, cf_chan_map, cf_pol_map, cf, n_cf_baseline, n_cf_chan, n_cf_pol,
              conv_u, conv_v, support, max_support, n_u, n_v, delta_l, delta_m, os_u, os_v, nt,
              nb, nchan, npol, n_img_chan, n_img_pol);
  cudaStream_t st = as_stream(stream);
  AV_CUDA(cudaMemsetAsync(cls, 0, sizeof(double) * (size_t)n_cls, st));
  k_aperture_classes<<<mg_blocks(rows, MG_THREADS), MG_THREADS, 0, st>>>(a, cls);
  AV_LAUNCH_CHECK();
  k_aperture_add<<<(unsigned)n_cls, MG_THREADS, 0, st>>>(a, cls);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"
