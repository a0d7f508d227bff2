/*
 * CPU oracle for the standard-gridder imaging path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C and FP64, the
 * arithmetic of astroviper's standard-gridder path so that the CUDA kernels
 * of astroviper_b200 can be checked against it.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it.  The product never calls it.
 *
 * Every function keeps the reference's operation order (no FMA contraction:
 * build with -ffp-contract=off) so that its results are bit-identical to the
 * reference's Numba / C++ code; tests/golden pins that.
 *
 * Reference files (paths inside the astroviper project):
 *   src/astroviper/core/imaging/imaging_utils/gcf_prolate_spheroidal.py
 *   src/astroviper/core/imaging/imaging_utils/standard_grid.py
 *   src/astroviper/core/imaging/imaging_utils/standard_degrid.py
 *   src/astroviper/core/imaging/imaging_weighting/grid_imaging_weights.py
 *   src/astroviper/core/imaging/deconvolvers/hogbom/src/hclean.cpp
 *   src/astroviper/core/imaging/imaging_utils/mosaic_grid.py
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

/* ---------------------------------------------------------------------------
 * PSWF rational approximation (Schwab), gcf_prolate_spheroidal.py:102-158.
 * grdsf(u) = sum_k p[part][k] d^k / sum_k q[part][k] d^k, d = u^2 - uend^2,
 * part 0 for |u| < 0.75 (uend 0.75), part 1 for 0.75 <= |u| <= 1 (uend 1),
 * 0 for |u| > 1.  Returns grdsf and (1 - u^2) grdsf.
 * ------------------------------------------------------------------------- */
static const double PSWF_P[2][5] = {
    {8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1},
    {4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2}};
static const double PSWF_Q[2][3] = {{1.0000000e0, 8.212018e-1, 2.078043e-1},
                                    {1.0000000e0, 9.599102e-1, 2.918724e-1}};

void orc_pswf(const double *u_in, int64_t n, double *grdsf_out, double *kern_out) {
  for (int64_t i = 0; i < n; ++i) {
    double u = fabs(u_in[i]);
    int part = 0;
    double uend = 0.0;
    if (u >= 0.0 && u < 0.75) { part = 0; uend = 0.75; }
    if (u >= 0.75 && u <= 1.0) { part = 1; uend = 1.0; }
    double delusq = u * u - uend * uend;
    double top = PSWF_P[part][0];
    for (int k = 1; k < 5; ++k) top += PSWF_P[part][k] * pow(delusq, (double)k);
    double bot = PSWF_Q[part][0];
    for (int k = 1; k < 3; ++k) bot += PSWF_Q[part][k] * pow(delusq, (double)k);
    double g = 0.0;
    if (bot > 0.0) g = top / bot;
    if (u > 1.0) g = 0.0;
    if (grdsf_out) grdsf_out[i] = g;
    if (kern_out) kern_out[i] = (1.0 - u * u) * g;
  }
}

/* create_prolate_spheroidal_kernel_1D, gcf_prolate_spheroidal.py:87-99:
 * out has oversampling*(support//2+1) entries; the first
 * oversampling*(support//2) are (1-u^2) grdsf(u) at u = i/(sc*os), rest 0. */
void orc_cgk_1d(int oversampling, int support, double *out) {
  int sc = support / 2;
  int64_t n = (int64_t)oversampling * sc;
  int64_t ntot = (int64_t)oversampling * (sc + 1);
  for (int64_t i = 0; i < ntot; ++i) out[i] = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double u = (double)i / (double)(sc * oversampling);
    orc_pswf(&u, 1, NULL, &out[i]);
  }
}

/* Grid-correction image of create_prolate_spheroidal_kernel,
 * gcf_prolate_spheroidal.py:73-79 (coordinates() at :161). */
void orc_corr_term(int64_t nx, int64_t ny, double *out) {
  double *gx = (double *)malloc(sizeof(double) * nx);
  double *gy = (double *)malloc(sizeof(double) * ny);
  for (int64_t i = 0; i < nx; ++i) {
    double c = (double)(i - nx / 2) / (double)nx;
    double u = fabs(2.0 * c);
    orc_pswf(&u, 1, &gx[i], NULL);
  }
  for (int64_t i = 0; i < ny; ++i) {
    double c = (double)(i - ny / 2) / (double)ny;
    double u = fabs(2.0 * c);
    orc_pswf(&u, 1, &gy[i], NULL);
  }
  for (int64_t i = 0; i < nx; ++i)
    for (int64_t j = 0; j < ny; ++j) out[i * ny + j] = gx[i] * gy[j];
  free(gx);
  free(gy);
}

/* Python int(x) of a finite double: truncation toward zero.  Values outside
 * +-2^62 cannot be inside any grid; they map to a sentinel that fails every
 * bounds test (Numba's fptosi gives INT64_MIN there). */
static inline int64_t trunc_i64(double x) {
  if (!(fabs(x) < 4.611686018427388e18)) return INT64_MIN / 2;
  return (int64_t)x;
}

/* ---------------------------------------------------------------------------
 * standard_grid_jit, standard_grid.py:246-432.
 * grid: (n_img_chan, n_img_pol, n_u, n_v), complex (is_complex=1, interleaved)
 *       or real (is_complex=0, only meaningful with do_psf).
 * vis: (nt, nb, nchan, npol) complex; weight same shape, real.
 * uvw: (nt, nb, 3).  chan_map (nchan), pol_map (npol).
 * The (t, b) range [tb_lo, tb_hi) lets the CPU baseline split work.
 * ------------------------------------------------------------------------- */
static void grid_range(void *grid, int is_complex, double *sum_weight, int do_psf,
                       int do_imaging_weight, const cplx *vis, const double *uvw,
                       const double *freq, const int64_t *chan_map,
                       const int64_t *pol_map, const double *weight, const double *cgk,
                       int64_t n_u, int64_t n_v, double dl0, double dl1, int support,
                       int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                       int64_t npol, int64_t n_img_pol, int64_t tb_lo, int64_t tb_hi) {
  const double c = 299792458.0;
  double *us0 = (double *)malloc(sizeof(double) * nchan);
  double *us1 = (double *)malloc(sizeof(double) * nchan);
  for (int64_t k = 0; k < nchan; ++k) {
    us0[k] = -(freq[k] * dl0 * (double)n_u) / c;
    us1[k] = -(freq[k] * dl1 * (double)n_v) / c;
  }
  const int64_t sc = support / 2;
  const int64_t uc0 = n_u / 2, uc1 = n_v / 2;
  const int64_t s0 = -sc, s1 = support - sc;
  cplx *gc = (cplx *)grid;
  double *gr = (double *)grid;
  (void)nt;
  for (int64_t tb = tb_lo; tb < tb_hi; ++tb) {
    const double *p_uvw = uvw + tb * 3;
    for (int64_t ic = 0; ic < nchan; ++ic) {
      int64_t a_chan = chan_map[ic];
      double u = p_uvw[0] * us0[ic];
      double v = p_uvw[1] * us1[ic];
      if (isnan(u) || isnan(v)) continue;
      double u_pos = u + (double)uc0, v_pos = v + (double)uc1;
      double u_pos_c = -u + (double)uc0, v_pos_c = -v + (double)uc1;
      int64_t ui = trunc_i64(u_pos + 0.5), vi = trunc_i64(v_pos + 0.5);
      int64_t uic = trunc_i64(u_pos_c + 0.5), vic = trunc_i64(v_pos_c + 0.5);
      if (!((ui + sc < n_u) && (vi + sc < n_v) && (ui - sc >= 0) && (vi - sc >= 0)))
        continue;
      double u_off = (double)ui - u_pos;
      int64_t uoi = (int64_t)floor(u_off * (double)oversampling + 0.5);
      double v_off = (double)vi - v_pos;
      int64_t voi = (int64_t)floor(v_off * (double)oversampling + 0.5);
      for (int64_t ip = 0; ip < npol; ++ip) {
        const int64_t idx = (tb * nchan + ic) * npol + ip;
        double sel_weight;
        cplx wd;
        if (do_psf) {
          if (npol >= 2 && do_imaging_weight) {
            const int64_t i0 = (tb * nchan + ic) * npol;
            wd.re = (weight[i0] + weight[i0 + 1]) / 2.0;
            wd.im = 0.0;
            sel_weight = wd.re;
          } else {
            sel_weight = weight[idx];
            wd.re = weight[idx];
            wd.im = 0.0;
          }
        } else {
          sel_weight = weight[idx];
          wd.re = vis[idx].re * weight[idx];
          wd.im = vis[idx].im * weight[idx];
        }
        if (isnan(wd.re) || isnan(wd.im)) continue;
        if (!(wd.re != 0.0 || wd.im != 0.0)) continue;
        int64_t a_pol = pol_map[ip];
        double norm = 0.0;
        int64_t plane = (a_chan * n_img_pol + a_pol) * n_u * n_v;
        for (int64_t iv = s0; iv < s1; ++iv) {
          int64_t v_indx = vi + iv;
          int64_t vo = oversampling * iv + voi;
          double conv_v = cgk[vo < 0 ? -vo : vo];
          int64_t v_indx_c = vic + iv;
          for (int64_t iu = s0; iu < s1; ++iu) {
            int64_t u_indx = ui + iu;
            int64_t uo = oversampling * iu + uoi;
            double conv_u = cgk[uo < 0 ? -uo : uo];
            double conv = conv_u * conv_v;
            int64_t g = plane + u_indx * n_v + v_indx;
            if (is_complex) {
              gc[g].re = gc[g].re + conv * wd.re;
              gc[g].im = gc[g].im + conv * wd.im;
            } else {
              gr[g] = gr[g] + conv * wd.re;
            }
            norm = norm + conv;
            if (do_imaging_weight) {
              int64_t u_indx_c = uic + iu;
              int64_t gg = plane + u_indx_c * n_v + v_indx_c;
              if (is_complex) {
                gc[gg].re = gc[gg].re + conv * wd.re;
                gc[gg].im = gc[gg].im + conv * wd.im;
              } else {
                gr[gg] = gr[gg] + conv * wd.re;
              }
            }
          }
        }
        int64_t sw = a_chan * n_img_pol + a_pol;
        sum_weight[sw] = sum_weight[sw] + sel_weight * norm;
        if (do_imaging_weight) sum_weight[sw] = sum_weight[sw] + sel_weight * norm;
      }
    }
  }
  free(us0);
  free(us1);
}

void orc_standard_grid(void *grid, int is_complex, double *sum_weight, int do_psf,
                       int do_imaging_weight, const cplx *vis, const double *uvw,
                       const double *freq, const int64_t *chan_map, const int64_t *pol_map,
                       const double *weight, const double *cgk, int64_t n_u, int64_t n_v,
                       double dl0, double dl1, int support, int oversampling, int64_t nt,
                       int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_pol) {
  grid_range(grid, is_complex, sum_weight, do_psf, do_imaging_weight, vis, uvw, freq,
             chan_map, pol_map, weight, cgk, n_u, n_v, dl0, dl1, support, oversampling, nt,
             nb, nchan, npol, n_img_pol, 0, nt * nb);
}

/* Multi-threaded gridding by owned grid rows (the CPU baseline and the
 * large-size parity checks).  Every image plane's u rows are cut into one
 * band per thread; a thread walks every sample in the reference's order and
 * adds only the taps whose u row lies in its band.  Each cell therefore
 * receives its addends in the serial order, and the grid is bit-identical to
 * orc_standard_grid.  sum_weight is added, per sample, by the thread owning
 * the footprint's first row, in sample order within a thread and then over
 * the threads in band order, so it can differ from the serial sum in the last
 * bits.  A first parallel pass computes every sample's cell and kernel
 * offsets once (the reference's expressions, standard_grid.py:297-352) and a
 * histogram of footprint rows; the cuts give every band about the same
 * number of taps.  No per-thread grid is allocated: the extra memory is
 * 16 bytes per (time, baseline, channel) sample.  do_imaging_weight is not
 * supported here (the serial restatement covers it).
 * Returns the number of threads used, -1 when memory runs out, -2 for a
 * support outside [1, ORC_MAX_SUPPORT]. */
typedef struct { int32_t ui, vi, uoi, voi; } orc_cell;
#define ORC_MAX_SUPPORT 64

int orc_standard_grid_mt(cplx *grid, double *sum_weight, int do_psf, const cplx *vis,
                         const double *uvw, const double *freq, const int64_t *chan_map,
                         const int64_t *pol_map, const double *weight, const double *cgk,
                         int64_t n_u, int64_t n_v, double dl0, double dl1, int support,
                         int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                         int64_t npol, int64_t n_img_chan, int64_t n_img_pol, int nthreads) {
#ifdef _OPENMP
  if (nthreads < 1) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  if (support < 1 || support > ORC_MAX_SUPPORT) return -2;
  const double c = 299792458.0;
  const int64_t sc = support / 2, s0 = -sc, s1 = support - sc;
  const int64_t uc0 = n_u / 2, uc1 = n_v / 2;
  const int64_t ntb = nt * nb, nsamp = ntb * nchan;
  const int64_t ssz = n_img_chan * n_img_pol;
  orc_cell *cells = (orc_cell *)malloc(sizeof(orc_cell) * (size_t)(nsamp > 0 ? nsamp : 1));
  double *us = (double *)malloc(sizeof(double) * 2 * (size_t)(nchan > 0 ? nchan : 1));
  int64_t *hist = (int64_t *)calloc((size_t)nthreads * (size_t)n_u, sizeof(int64_t));
  int64_t *cut = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nthreads + 1));
  double *psw = (double *)calloc((size_t)nthreads * (size_t)(ssz > 0 ? ssz : 1), sizeof(double));
  if (!cells || !us || !hist || !cut || !psw) {
    free(cells); free(us); free(hist); free(cut); free(psw);
    return -1;
  }
  for (int64_t k = 0; k < nchan; ++k) {
    us[2 * k] = -(freq[k] * dl0 * (double)n_u) / c;
    us[2 * k + 1] = -(freq[k] * dl1 * (double)n_v) / c;
  }
  /* pass 1: cells and offsets, histogram of first footprint rows */
#pragma omp parallel num_threads(nthreads)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    int64_t *h = hist + (int64_t)t * n_u;
#pragma omp for schedule(static)
    for (int64_t tb = 0; tb < ntb; ++tb) {
      const double *p_uvw = uvw + tb * 3;
      for (int64_t ic = 0; ic < nchan; ++ic) {
        orc_cell *cl = &cells[tb * nchan + ic];
        cl->ui = INT32_MIN;
        double u = p_uvw[0] * us[2 * ic];
        double v = p_uvw[1] * us[2 * ic + 1];
        if (isnan(u) || isnan(v)) continue;
        double u_pos = u + (double)uc0, v_pos = v + (double)uc1;
        int64_t ui = trunc_i64(u_pos + 0.5), vi = trunc_i64(v_pos + 0.5);
        if (!((ui + sc < n_u) && (vi + sc < n_v) && (ui - sc >= 0) && (vi - sc >= 0))) continue;
        cl->ui = (int32_t)ui;
        cl->vi = (int32_t)vi;
        cl->uoi = (int32_t)(int64_t)floor(((double)ui - u_pos) * (double)oversampling + 0.5);
        cl->voi = (int32_t)(int64_t)floor(((double)vi - v_pos) * (double)oversampling + 0.5);
        h[ui + s0] += 1;
      }
    }
  }
  /* row cuts: rows weighted by the footprints that cover them */
  {
    double total = 0.0;
    double *cover = (double *)calloc((size_t)n_u, sizeof(double));
    if (!cover) {
      free(cells); free(us); free(hist); free(cut); free(psw);
      return -1;
    }
    for (int64_t r = 0; r < n_u; ++r) {
      int64_t n0 = 0;
      for (int t = 0; t < nthreads; ++t) n0 += hist[(int64_t)t * n_u + r];
      for (int64_t d = 0; d < support && r + d < n_u; ++d) cover[r + d] += (double)n0;
      total += (double)n0 * (double)support;
    }
    cut[0] = 0;
    int k = 1;
    double acc = 0.0;
    for (int64_t r = 0; r < n_u && k < nthreads; ++r) {
      acc += cover[r];
      while (k < nthreads && acc >= total * (double)k / (double)nthreads) cut[k++] = r + 1;
    }
    while (k <= nthreads) cut[k++] = n_u;
    free(cover);
  }
  /* pass 2: every band walks all samples in order.  The tap products
   * conv = cgk[|os iu + uoi|] * cgk[|os iv + voi|] and their sum (norm, in
   * the reference's iv-outer, iu-inner order) do not depend on the
   * polarisation: they are formed once per sample, with the same operands
   * and order as the reference forms them per polarisation. */
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int t = 0; t < nthreads; ++t) {
    const int64_t lo = cut[t], hi = cut[t + 1];
    double *sw_t = psw + (int64_t)t * ssz;
    double conv[ORC_MAX_SUPPORT * ORC_MAX_SUPPORT];
    if (lo >= hi) continue;
    for (int64_t tb = 0; tb < ntb; ++tb) {
      for (int64_t ic = 0; ic < nchan; ++ic) {
        const orc_cell cl = cells[tb * nchan + ic];
        if (cl.ui == INT32_MIN) continue;
        const int64_t ui = cl.ui, vi = cl.vi;
        if (ui + s1 <= lo || ui + s0 >= hi) continue;
        const int64_t iu_lo = lo - ui > s0 ? lo - ui : s0;
        const int64_t iu_hi = hi - ui < s1 ? hi - ui : s1;
        const int owns_sw = (ui + s0 >= lo) && (ui + s0 < hi);
        const int64_t a_chan = chan_map[ic];
        double norm = 0.0;
        for (int64_t iv = s0; iv < s1; ++iv) {
          const int64_t vo = (int64_t)oversampling * iv + cl.voi;
          const double conv_v = cgk[vo < 0 ? -vo : vo];
          for (int64_t iu = s0; iu < s1; ++iu) {
            const int64_t uo = (int64_t)oversampling * iu + cl.uoi;
            const double cv = cgk[uo < 0 ? -uo : uo] * conv_v;
            conv[(iv - s0) * support + (iu - s0)] = cv;
            norm = norm + cv;
          }
        }
        for (int64_t ip = 0; ip < npol; ++ip) {
          const int64_t idx = (tb * nchan + ic) * npol + ip;
          double sel_weight = weight[idx];
          cplx wd;
          if (do_psf) {
            wd.re = weight[idx];
            wd.im = 0.0;
          } else {
            wd.re = vis[idx].re * weight[idx];
            wd.im = vis[idx].im * weight[idx];
          }
          if (isnan(wd.re) || isnan(wd.im)) continue;
          if (!(wd.re != 0.0 || wd.im != 0.0)) continue;
          const int64_t a_pol = pol_map[ip];
          cplx *plane = grid + (a_chan * n_img_pol + a_pol) * n_u * n_v;
          for (int64_t iv = s0; iv < s1; ++iv) {
            const double *crow = conv + (iv - s0) * support - s0;
            cplx *grow = plane + (vi + iv);
            for (int64_t iu = iu_lo; iu < iu_hi; ++iu) {
              cplx *g = grow + (ui + iu) * n_v;
              g->re = g->re + crow[iu] * wd.re;
              g->im = g->im + crow[iu] * wd.im;
            }
          }
          if (owns_sw) sw_t[a_chan * n_img_pol + a_pol] += sel_weight * norm;
        }
      }
    }
  }
  for (int64_t s = 0; s < ssz; ++s)
    for (int t = 0; t < nthreads; ++t) sum_weight[s] += psw[(int64_t)t * ssz + s];
  free(cells);
  free(us);
  free(hist);
  free(cut);
  free(psw);
  return nthreads;
}

/* ---------------------------------------------------------------------------
 * dgrid_numba, standard_degrid.py:388-485.
 * values (nt, nb, nvchan, nvpol) complex, += ; flag same shape (uint8).
 * grid (nchan, npol, gx, gy) complex; the bounds test uses the reference's
 * own nx = shape[3], ny = shape[2] (standard_degrid.py:407,457-462); a sample
 * that passes it but would still index outside the array is skipped here.
 * ------------------------------------------------------------------------- */
static void dgrid_range(const double *uvw, const double *dphase, cplx *values,
                        const uint8_t *flag, const double *scale, const double *offset,
                        const cplx *grid, int64_t g_nchan, int64_t g_npol, int64_t g_n2,
                        int64_t g_n3, const double *freq, double c, int support, int sampling,
                        const double *convFunc, const int64_t *chanmap, const int64_t *polmap,
                        int64_t nt, int64_t nb, int64_t nvchan, int64_t nvpol, int64_t t_lo,
                        int64_t t_hi) {
  const int64_t nx = g_n3, ny = g_n2; /* as named in the reference */
  const int64_t supp_centre = support / 2;
  const int64_t supp_beg = -supp_centre, supp_end = supp_beg + support;
  (void)nt;
  /* The reference loops polarisation outside channel; every value is
   * computed on its own, so the walk here takes the channel outside and
   * forms the position, the phasor and the tap products wt = wtx * wty (and
   * their sum, norm, in the reference's ix-outer, iy-inner order) once for
   * all polarisations: same operands, same order, same results. */
  double *wt = (double *)malloc(sizeof(double) * (size_t)support * (size_t)support);
  if (!wt) return;
  for (int64_t t = t_lo; t < t_hi; ++t) {
    for (int64_t b = 0; b < nb; ++b) {
      const double *p_uvw = uvw + (t * nb + b) * 3;
      for (int64_t ichan = 0; ichan < nvchan; ++ichan) {
        int64_t achan = chanmap[ichan];
        if (!(0 <= achan && achan < g_nchan)) continue;
        double pos0 = scale[0] * p_uvw[0] * freq[ichan] / c + offset[0];
        double pos1 = scale[1] * p_uvw[1] * freq[ichan] / c + offset[1];
        double r0 = nearbyint(pos0), r1 = nearbyint(pos1);
        /* loc and off are stored in int32 arrays by the reference
         * (standard_degrid.py:413-414): keep its wrap-around. */
        int64_t loc0 = (int32_t)(uint32_t)(uint64_t)trunc_i64(r0);
        int64_t loc1 = (int32_t)(uint32_t)(uint64_t)trunc_i64(r1);
        int64_t off0 = (int32_t)(uint32_t)(uint64_t)trunc_i64(
            nearbyint(((double)loc0 - pos0) * (double)sampling));
        int64_t off1 = (int32_t)(uint32_t)(uint64_t)trunc_i64(
            nearbyint(((double)loc1 - pos1) * (double)sampling));
        int64_t x0 = loc0, y0 = loc1;
        if (!((x0 + supp_beg >= 0) && ((x0 + supp_end - 1) < nx) && (y0 + supp_beg >= 0) &&
              ((y0 + supp_end - 1) < ny)))
          continue;
        if (x0 + supp_end - 1 >= g_n2 || y0 + supp_end - 1 >= g_n3) continue;
        int any = 0;
        for (int64_t ipol = 0; ipol < nvpol && !any; ++ipol) {
          int64_t apol = polmap[ipol];
          int64_t vidx = ((t * nb + b) * nvchan + ichan) * nvpol + ipol;
          any = (0 <= apol && apol < g_npol) && !flag[vidx];
        }
        if (!any) continue;
        double phase = -2.0 * M_PI * dphase[t * nb + b] * freq[ichan] / c;
        double ph_re = cos(phase), ph_im = sin(phase);
        double norm = 0.0;
        for (int64_t ix = supp_beg; ix < supp_end; ++ix) {
          int64_t i1 = sampling * ix + off0;
          double wtx = convFunc[i1 < 0 ? -i1 : i1];
          for (int64_t iy = supp_beg; iy < supp_end; ++iy) {
            int64_t i2 = sampling * iy + off1;
            double w = wtx * convFunc[i2 < 0 ? -i2 : i2];
            wt[(ix - supp_beg) * support + (iy - supp_beg)] = w;
            norm += w;
          }
        }
        if (norm == 0.0) continue;
        for (int64_t ipol = 0; ipol < nvpol; ++ipol) {
          int64_t apol = polmap[ipol];
          if (!(0 <= apol && apol < g_npol)) continue;
          int64_t vidx = ((t * nb + b) * nvchan + ichan) * nvpol + ipol;
          if (flag[vidx]) continue;
          double nv_re = 0.0, nv_im = 0.0;
          const cplx *plane = grid + (achan * g_npol + apol) * g_n2 * g_n3;
          for (int64_t ix = supp_beg; ix < supp_end; ++ix) {
            const cplx *grow = plane + (x0 + ix) * g_n3 + y0;
            const double *wrow = wt + (ix - supp_beg) * support - supp_beg;
            for (int64_t iy = supp_beg; iy < supp_end; ++iy) {
              cplx gv = grow[iy];
              nv_re = nv_re + wrow[iy] * gv.re;
              nv_im = nv_im + wrow[iy] * gv.im;
            }
          }
          /* nvalue * conj(phasor), then / norm (component-wise for a real
           * divisor, as the complex quotient reduces to it). */
          double cr = ph_re, ci = -ph_im;
          double pr = nv_re * cr - nv_im * ci;
          double pi = nv_re * ci + nv_im * cr;
          values[vidx].re = values[vidx].re + pr / norm;
          values[vidx].im = values[vidx].im + pi / norm;
        }
      }
    }
  }
  free(wt);
}

void orc_dgrid(const double *uvw, const double *dphase, cplx *values, const uint8_t *flag,
               const double *scale, const double *offset, const cplx *grid, int64_t g_nchan,
               int64_t g_npol, int64_t g_n2, int64_t g_n3, const double *freq, double c,
               int support, int sampling, const double *convFunc, const int64_t *chanmap,
               const int64_t *polmap, int64_t nt, int64_t nb, int64_t nvchan, int64_t nvpol,
               int nthreads) {
#ifdef _OPENMP
  if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    int t = omp_get_thread_num(), T = omp_get_num_threads();
    int64_t lo = nt * t / T, hi = nt * (t + 1) / T;
    dgrid_range(uvw, dphase, values, flag, scale, offset, grid, g_nchan, g_npol, g_n2, g_n3,
                freq, c, support, sampling, convFunc, chanmap, polmap, nt, nb, nvchan, nvpol,
                lo, hi);
  }
#else
  (void)nthreads;
  dgrid_range(uvw, dphase, values, flag, scale, offset, grid, g_nchan, g_npol, g_n2, g_n3, freq,
              c, support, sampling, convFunc, chanmap, polmap, nt, nb, nvchan, nvpol, 0, nt);
#endif
}

/* Transpose of dgrid_numba (standard_degrid.py:388-485): for every sample the
 * degridder reads, grid[c, p, x0+ix, y0+iy] += wt * phasor * values / norm
 * (same positions, taps, maps and flags, FP64).  Used to check the adjoint
 * kernels of the degridding forward model. */
void orc_dgrid_adjoint(const double *uvw, const double *dphase, const cplx *values,
                       const uint8_t *flag, const double *scale, const double *offset,
                       cplx *grid, int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                       const double *freq, double c, int support, int sampling,
                       const double *convFunc, const int64_t *chanmap, const int64_t *polmap,
                       int64_t nt, int64_t nb, int64_t nvchan, int64_t nvpol) {
  const int64_t nx = g_n3, ny = g_n2;
  const int64_t supp_beg = -(support / 2), supp_end = supp_beg + support;
  for (int64_t t = 0; t < nt; ++t)
    for (int64_t b = 0; b < nb; ++b) {
      const double *p_uvw = uvw + (t * nb + b) * 3;
      for (int64_t ipol = 0; ipol < nvpol; ++ipol) {
        int64_t apol = polmap[ipol];
        if (!(0 <= apol && apol < g_npol)) continue;
        for (int64_t ichan = 0; ichan < nvchan; ++ichan) {
          int64_t achan = chanmap[ichan];
          int64_t vidx = ((t * nb + b) * nvchan + ichan) * nvpol + ipol;
          if (!(0 <= achan && achan < g_nchan) || (flag && flag[vidx])) continue;
          double pos0 = scale[0] * p_uvw[0] * freq[ichan] / c + offset[0];
          double pos1 = scale[1] * p_uvw[1] * freq[ichan] / c + offset[1];
          int64_t x0 = (int32_t)(uint32_t)(uint64_t)trunc_i64(nearbyint(pos0));
          int64_t y0 = (int32_t)(uint32_t)(uint64_t)trunc_i64(nearbyint(pos1));
          int64_t off0 = (int32_t)(uint32_t)(uint64_t)trunc_i64(
              nearbyint(((double)x0 - pos0) * (double)sampling));
          int64_t off1 = (int32_t)(uint32_t)(uint64_t)trunc_i64(
              nearbyint(((double)y0 - pos1) * (double)sampling));
          if (!((x0 + supp_beg >= 0) && ((x0 + supp_end - 1) < nx) && (y0 + supp_beg >= 0) &&
                ((y0 + supp_end - 1) < ny)))
            continue;
          if (x0 + supp_end - 1 >= g_n2 || y0 + supp_end - 1 >= g_n3) continue;
          double norm = 0.0;
          for (int64_t ix = supp_beg; ix < supp_end; ++ix) {
            int64_t i1 = sampling * ix + off0;
            for (int64_t iy = supp_beg; iy < supp_end; ++iy) {
              int64_t i2 = sampling * iy + off1;
              norm += convFunc[i1 < 0 ? -i1 : i1] * convFunc[i2 < 0 ? -i2 : i2];
            }
          }
          if (norm == 0.0) continue;
          double phase = dphase ? -2.0 * M_PI * dphase[t * nb + b] * freq[ichan] / c : 0.0;
          double pr = cos(phase), pi = sin(phase);
          double vr = values[vidx].re * pr - values[vidx].im * pi;
          double vi = values[vidx].re * pi + values[vidx].im * pr;
          cplx *plane = grid + (achan * g_npol + apol) * g_n2 * g_n3;
          for (int64_t ix = supp_beg; ix < supp_end; ++ix) {
            int64_t i1 = sampling * ix + off0;
            double wtx = convFunc[i1 < 0 ? -i1 : i1];
            for (int64_t iy = supp_beg; iy < supp_end; ++iy) {
              int64_t i2 = sampling * iy + off1;
              double wt = wtx * convFunc[i2 < 0 ? -i2 : i2];
              cplx *g = &plane[(x0 + ix) * g_n3 + (y0 + iy)];
              g->re += wt * vr / norm;
              g->im += wt * vi / norm;
            }
          }
        }
      }
    }
}

/* ---------------------------------------------------------------------------
 * grid_imaging_weights_jit, grid_imaging_weights.py:93-206.
 * grid (n_chan, n_gpol, n_u, n_v) real; data_weights (nt, nb, nchan, npol).
 * ------------------------------------------------------------------------- */
void orc_grid_imaging_weights(double *grid, int64_t n_gpol, double *sum_weight,
                              const double *uvw, const double *freq, const int64_t *chan_map,
                              const double *data_weights, int64_t n_u, int64_t n_v, double dl0,
                              double dl1, int64_t nt, int64_t nb, int64_t nchan, int64_t npol) {
  const double c = 299792458.0;
  const int64_t uc0 = n_u / 2, uc1 = n_v / 2;
  for (int64_t tb = 0; tb < nt * nb; ++tb) {
    for (int64_t ic = 0; ic < nchan; ++ic) {
      int64_t a_chan = chan_map[ic];
      double us0 = -(freq[ic] * dl0 * (double)n_u) / c;
      double us1 = -(freq[ic] * dl1 * (double)n_v) / c;
      double u = uvw[tb * 3 + 0] * us0, v = uvw[tb * 3 + 1] * us1;
      if (isnan(u) || isnan(v)) continue;
      double u_pos = u + (double)uc0, v_pos = v + (double)uc1;
      double u_pos_c = -u + (double)uc0, v_pos_c = -v + (double)uc1;
      int64_t ui = trunc_i64(u_pos + 0.5), vi = trunc_i64(v_pos + 0.5);
      int64_t uic = trunc_i64(u_pos_c + 0.5), vic = trunc_i64(v_pos_c + 0.5);
      if (!((ui < n_u) && (vi < n_v) && (ui >= 0) && (vi >= 0))) continue;
      double w = data_weights[(tb * nchan + ic) * npol + 0];
      if (isnan(w)) continue;
      double *plane = grid + (a_chan * n_gpol + 0) * n_u * n_v;
      plane[ui * n_v + vi] = plane[ui * n_v + vi] + w;
      /* the conjugate cell is not bounds-checked by the reference; for a
       * grid of even size it is in range whenever the direct cell is,
       * except at index 0 where it would be n (skipped here). */
      if (uic >= 0 && uic < n_u && vic >= 0 && vic < n_v)
        plane[uic * n_v + vic] = plane[uic * n_v + vic] + w;
      sum_weight[a_chan * n_gpol + 0] = sum_weight[a_chan * n_gpol + 0] + 2.0 * w;
    }
  }
}

/* degrid_imaging_weights_jit, grid_imaging_weights.py:285-443.
 * imaging_weight must be zero-initialised by the caller (the reference wrapper
 * allocates np.zeros, :266). */
int orc_degrid_imaging_weights(double *imaging_weight, const double *grid, int64_t n_gchan,
                               int64_t n_gpol, const double *briggs_factors,
                               const double *uvw, const double *freq, const int64_t *chan_map,
                               const int64_t *pol_map, int64_t n_pol_map,
                               const double *data_weight, int64_t n_u, int64_t n_v, double dl0,
                               double dl1, int64_t nt, int64_t nb, int64_t nchan,
                               int64_t npol) {
  const double c = 299792458.0;
  const int64_t uc0 = n_u / 2, uc1 = n_v / 2;
  for (int64_t tb = 0; tb < nt * nb; ++tb) {
    for (int64_t ic = 0; ic < nchan; ++ic) {
      int64_t a_chan = chan_map[ic];
      double us0 = -(freq[ic] * dl0 * (double)n_u) / c;
      double us1 = -(freq[ic] * dl1 * (double)n_v) / c;
      double u = uvw[tb * 3 + 0] * us0, v = uvw[tb * 3 + 1] * us1;
      if (isnan(u) || isnan(v)) continue;
      double u_pos = u + (double)uc0, v_pos = v + (double)uc1;
      int64_t ui = trunc_i64(u_pos + 0.5), vi = trunc_i64(v_pos + 0.5);
      if (!((ui < n_u) && (vi < n_v) && (ui >= 0) && (vi >= 0))) continue;
      for (int64_t ip = 0; ip < n_pol_map; ++ip) {
        int64_t a_pol = pol_map[ip];
        int64_t idx = (tb * nchan + ic) * npol + ip;
        double dw = data_weight[idx];
        imaging_weight[idx] = dw;
        if (!isnan(dw) && dw != 0.0) {
          double gij = grid[((a_chan * n_gpol + a_pol) * n_u + ui) * n_v + vi];
          if (!isnan(gij) && gij != 0.0) {
            double f0 = briggs_factors[(0 * n_gchan + a_chan) * n_gpol + a_pol];
            double f1 = briggs_factors[(1 * n_gchan + a_chan) * n_gpol + a_pol];
            if (isnan(f0) || isnan(f1)) return -1;
            double denom = f0 * gij + f1;
            imaging_weight[idx] = imaging_weight[idx] / denom;
          }
        }
      }
    }
  }
  return 0;
}

/* standard_imaging_weight_degrid_jit, standard_grid.py:487-604.  Per
 * polarisation: the natural weight (pols 0 and 1 averaged when n_pol == 2),
 * divided by f0 * G + f1 where the polarisation's own natural weight and G
 * are neither NaN nor zero; samples off the grid are not written. */
void orc_imaging_weight_degrid(double *imaging_weight, const double *grid, int64_t n_gchan,
                               int64_t n_gpol, const double *briggs_factors, const double *uvw,
                               const double *freq, const int64_t *chan_map,
                               const int64_t *pol_map, const double *natural, int64_t n_u,
                               int64_t n_v, double dl0, double dl1, int64_t nt, int64_t nb,
                               int64_t nchan, int64_t npol) {
  const double c = 299792458.0;
  const int64_t uc0 = n_u / 2, uc1 = n_v / 2;
  for (int64_t tb = 0; tb < nt * nb; ++tb) {
    for (int64_t ic = 0; ic < nchan; ++ic) {
      const int64_t a_chan = chan_map[ic];
      const double us0 = -(freq[ic] * dl0 * (double)n_u) / c;
      const double us1 = -(freq[ic] * dl1 * (double)n_v) / c;
      const double u = uvw[tb * 3 + 0] * us0, v = uvw[tb * 3 + 1] * us1;
      if (isnan(u) || isnan(v)) continue;
      const double u_pos = u + (double)uc0, v_pos = v + (double)uc1;
      const int64_t ui = trunc_i64(u_pos + 0.5), vi = trunc_i64(v_pos + 0.5);
      if (!((ui < n_u) && (vi < n_v) && (ui >= 0) && (vi >= 0))) continue;
      const double *nw = natural + (tb * nchan + ic) * npol;
      for (int64_t ip = 0; ip < npol; ++ip) {
        const int64_t a_pol = pol_map[ip];
        double *out = imaging_weight + (tb * nchan + ic) * npol + ip;
        *out = npol == 2 ? (nw[0] + nw[1]) / 2.0 : nw[ip];
        if (!isnan(nw[ip]) && nw[ip] != 0.0) {
          const double g = grid[((a_chan * n_gpol + a_pol) * n_u + ui) * n_v + vi];
          if (!isnan(g) && g != 0.0) {
            const double f0 = briggs_factors[(0 * n_gchan + a_chan) * n_gpol + a_pol];
            const double f1 = briggs_factors[(1 * n_gchan + a_chan) * n_gpol + a_pol];
            *out = *out / (f0 * g + f1);
          }
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------------
 * Hogbom CLEAN, hclean.cpp:51-81 (maximg) and :106-210 (clean).
 * Generalised to a PSF of size (pny, pnx) >= (ny, nx) with centre
 * (pny/2, pnx/2): with pnx = nx, pny = ny this is the reference exactly.
 * comps (optional, 3 x niter): px, py and the component value pv per
 * iteration, for position checks.
 * ------------------------------------------------------------------------- */
#define HOGBOM_BODY(T, ABS, POW)                                                              \
  int yes = 0;                                                                                \
  T maxval = 0, absval = 0;                                                                   \
  int px = 0, py = 0;                                                                         \
  int iter;                                                                                   \
  int ncomp = 0;                                                                              \
  for (iter = siter; iter < niter; ++iter) {                                                  \
    absval = (T)0;                                                                            \
    for (int iy = ybeg; iy < yend; ++iy)                                                      \
      for (int ix = xbeg; ix < xend; ++ix) {                                                  \
        if (domask == 0 || lmask[(int64_t)iy * nx + ix] > (T)0.5) {                           \
          T val = ABS(limagestep[(int64_t)iy * nx + ix]);                                     \
          if (val > absval) { px = ix; py = iy; absval = val; }                               \
        }                                                                                     \
      }                                                                                       \
    maxval = limagestep[(int64_t)py * nx + px];                                               \
    T cthres;                                                                                 \
    if (cspeedup > (T)0) cthres = thres * POW((T)2, (T)(iter - siter) / cspeedup);            \
    else cthres = thres;                                                                      \
    if (yes == 1 || absval < cthres) break;                                                   \
    int x1 = px - pnx / 2 > 0 ? px - pnx / 2 : 0;                                             \
    int y1 = py - pny / 2 > 0 ? py - pny / 2 : 0;                                             \
    int x2 = px + pnx / 2 - 1 < nx - 1 ? px + pnx / 2 - 1 : nx - 1;                           \
    int y2 = py + pny / 2 - 1 < ny - 1 ? py + pny / 2 - 1 : ny - 1;                           \
    T pv = gain * maxval;                                                                     \
    limage[(int64_t)py * nx + px] += pv;                                                      \
    if (comps) {                                                                              \
      comps[3 * ncomp + 0] = (double)px;                                                      \
      comps[3 * ncomp + 1] = (double)py;                                                      \
      comps[3 * ncomp + 2] = (double)pv;                                                      \
    }                                                                                         \
    ++ncomp;                                                                                  \
    for (int iy = y1; iy <= y2; ++iy)                                                         \
      for (int ix = x1; ix <= x2; ++ix) {                                                     \
        int psf_x = pnx / 2 + ix - px, psf_y = pny / 2 + iy - py;                             \
        if (psf_x < 0 || psf_x >= pnx || psf_y < 0 || psf_y >= pny) continue;                 \
        limagestep[(int64_t)iy * nx + ix] -= pv * lpsf[(int64_t)psf_y * pnx + psf_x];         \
      }                                                                                       \
  }                                                                                           \
  if (iter > niter) iter = niter;                                                             \
  out_peak[0] = px;                                                                           \
  out_peak[1] = py;                                                                           \
  *out_maxval = (double)maxval;                                                               \
  return iter;

int orc_hogbom_f32(float *limage, float *limagestep, const float *lpsf, int pnx, int pny,
                   int domask, const float *lmask, int nx, int ny, int xbeg, int xend, int ybeg,
                   int yend, int niter, int siter, float gain, float thres, float cspeedup,
                   double *comps, int *out_peak, double *out_maxval) {
  HOGBOM_BODY(float, fabsf, powf)
}

int orc_hogbom_f64(double *limage, double *limagestep, const double *lpsf, int pnx, int pny,
                   int domask, const double *lmask, int nx, int ny, int xbeg, int xend,
                   int ybeg, int yend, int niter, int siter, double gain, double thres,
                   double cspeedup, double *comps, int *out_peak, double *out_maxval) {
  HOGBOM_BODY(double, fabs, pow)
}

void orc_maximg_f32(const float *img, int domask, const float *mask, int nx, int ny,
                    float *fmin, float *fmax) {
  float mn = 1e20f, mx = -1e20f;
  for (int64_t i = 0; i < (int64_t)nx * ny; ++i)
    if (domask == 0 || mask[i] > 0.5f) {
      float w = img[i];
      if (w > mx) mx = w;
      if (w < mn) mn = w;
    }
  *fmin = mn;
  *fmax = mx;
}

void orc_maximg_f64(const double *img, int domask, const double *mask, int nx, int ny,
                    double *fmin, double *fmax) {
  double mn = 1e20, mx = -1e20;
  for (int64_t i = 0; i < (int64_t)nx * ny; ++i)
    if (domask == 0 || mask[i] > 0.5) {
      double w = img[i];
      if (w > mx) mx = w;
      if (w < mn) mn = w;
    }
  *fmin = mn;
  *fmax = mx;
}

/* ---------------------------------------------------------------------------
 * Mosaic gridder, mosaic_grid_jit (mosaic_grid.py:307-486): each sample's
 * window of the convolution function cf (n_cfb, n_cfc, n_cfp, cu, cv),
 * phase gradient already applied, v outer and u inner, in sample order.
 * grid (n_img_chan, n_img_pol, n_u, n_v) and sum_weight (n_img_chan,
 * n_img_pol) are accumulated.  Window taps outside cf (the reference reads
 * past the array there) are left out.
 * ------------------------------------------------------------------------- */
static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

void orc_mosaic_grid(cplx *grid, double *sum_weight, int do_psf, const cplx *vis,
                     const double *uvw, const double *freq, const int64_t *chan_map,
                     const int64_t *pol_map, const int64_t *cfb_map, const int64_t *cfc_map,
                     const int64_t *cfp_map, const double *weight, const cplx *cf, int64_t n_cfc,
                     int64_t n_cfp, int64_t cu, int64_t cv, const int64_t *support,
                     int64_t max_support, int64_t n_u, int64_t n_v, double dl0, double dl1,
                     int64_t os_u, int64_t os_v, int64_t nt, int64_t nb, int64_t nchan,
                     int64_t npol, int64_t n_img_pol) {
  const double c = 299792458.0;
  for (int64_t t = 0; t < nt; ++t)
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t cfb = cfb_map[b];
      for (int64_t ch = 0; ch < nchan; ++ch) {
        const double s0 = -(freq[ch] * dl0 * (double)n_u) / c;
        const double s1 = -(freq[ch] * dl1 * (double)n_v) / c;
        const int64_t tb = t * nb + b;
        const double u = uvw[3 * tb] * s0, v = uvw[3 * tb + 1] * s1;
        if (isnan(u) || isnan(v)) continue;
        const double up = u + (double)(n_u / 2), vp = v + (double)(n_v / 2);
        const int64_t uc = trunc_i64(up + 0.5), vc = trunc_i64(vp + 0.5);
        if (!(uc + max_support < n_u && vc + max_support < n_v && uc - max_support >= 0 &&
              vc - max_support >= 0))
          continue;
        const int64_t uo = (int64_t)floor(((double)uc - up) * (double)os_u + 0.5) + cu / 2;
        const int64_t vo = (int64_t)floor(((double)vc - vp) * (double)os_v + 0.5) + cv / 2;
        const int64_t cfc = cfc_map[ch], ach = chan_map[ch];
        for (int64_t p = 0; p < npol; ++p) {
          const int64_t k = (tb * nchan + ch) * npol + p;
          const double w = weight[k];
          cplx wd;
          if (do_psf) {
            wd.re = w;
            wd.im = 0.0;
          } else {
            wd.re = vis[k].re * w;
            wd.im = vis[k].im * w;
          }
          if (isnan(wd.re) || isnan(wd.im) || (wd.re == 0.0 && wd.im == 0.0)) continue;
          const int64_t cfp = cfp_map[p], apol = pol_map[p];
          const int64_t fidx = (cfb * n_cfc + cfc) * n_cfp + cfp;
          const int64_t su = support[2 * fidx], sv = support[2 * fidx + 1];
          const cplx *f = cf + fidx * cu * cv;
          cplx *g = grid + (ach * n_img_pol + apol) * n_u * n_v;
          cplx norm = {0.0, 0.0};
          for (int64_t iv = -(sv / 2); iv < sv - sv / 2; ++iv) {
            const int64_t fv = os_v * iv + vo;
            for (int64_t iu = -(su / 2); iu < su - su / 2; ++iu) {
              const int64_t fu = os_u * iu + uo;
              if (fu < 0 || fu >= cu || fv < 0 || fv >= cv) continue;
              const cplx cw = f[fu * cv + fv];
              const cplx x = cmul(cw, wd);
              cplx *cell = g + (uc + iu) * n_v + (vc + iv);
              cell->re += x.re;
              cell->im += x.im;
              norm.re += cw.re;
              norm.im += cw.im;
            }
          }
          const double re = do_psf ? norm.re : norm.re * norm.re - norm.im * norm.im;
          sum_weight[ach * n_img_pol + apol] += w * re;
        }
      }
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
