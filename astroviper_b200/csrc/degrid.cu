// Convolutional degridding (dgrid_numba, standard_degrid.py:388-485).
//
// av_degrid_plain: one thread per (sample, polarisation), FP64, the
//   reference's tap order and summation order: bit-identical to it.
// av_degrid_tiled: FP32 over a cell-sorted plan (plan.cuh).  Each CTA stages
//   a tile's sub-grid (all image polarisations) in shared memory and gives
//   one record to each thread; consecutive threads hold samples of the same
//   cell, so the sub-grid reads are broadcasts.  The separable kernel is
//   applied as row sums (sum_j cv_j G_ij, then sum_i cu_i row_i) with packed
//   FP32 FMAs; the normalisation sum_k w_k is (sum_i cu_i)(sum_j cv_j) from
//   FP64 per-offset row sums.
#include "plan.cuh"
#include "umma.cuh"

namespace av {

struct DegridArgs {
  const double *uvw, *dphase;
  void *values;
  int values_c128;
  const uint8_t *flag;
  double scale0, scale1, offset0, offset1;
  const void *grid;
  int grid_c128;
  int64_t g_nchan, g_npol, g_n2, g_n3;
  const double *freq;
  double c;
  int support, sampling;
  const double *cf;
  const int32_t *chanmap, *polmap;
  int64_t nt, nb, nvchan, nvpol;
};

// ---------------------------------------------------------------- plain ----
__global__ void __launch_bounds__(256) k_degrid_plain(DegridArgs a) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t total = a.nt * a.nb * a.nvchan * a.nvpol;
  if (k >= total) return;
  int64_t row = k / a.nvpol;
  int ipol = (int)(k - row * a.nvpol);
  int64_t tb = row / a.nvchan;
  int ichan = (int)(row - tb * a.nvchan);
  int apol = a.polmap[ipol];
  if (!(0 <= apol && apol < a.g_npol)) return;
  int achan = a.chanmap[ichan];
  if (!(0 <= achan && achan < a.g_nchan)) return;
  if (a.flag && a.flag[k]) return;
  const double f = a.freq[ichan];
  double p0 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(a.scale0, a.uvw[3 * tb]), f), a.c), a.offset0);
  double p1 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(a.scale1, a.uvw[3 * tb + 1]), f), a.c), a.offset1);
  int x0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p0));
  int y0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p1));
  int o0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(__dmul_rn(__dsub_rn((double)x0, p0), (double)a.sampling)));
  int o1 = (int)(unsigned)(unsigned long long)trunc_ll(rint(__dmul_rn(__dsub_rn((double)y0, p1), (double)a.sampling)));
  const long long beg = -(a.support / 2), end = beg + a.support;
  // the reference's nx = shape[3], ny = shape[2] (standard_degrid.py:407)
  if (!(((long long)x0 + beg >= 0) && ((long long)x0 + end - 1 < a.g_n3) &&
        ((long long)y0 + beg >= 0) && ((long long)y0 + end - 1 < a.g_n2)))
    return;
  if (!((long long)x0 + end - 1 < a.g_n2 && (long long)y0 + end - 1 < a.g_n3)) return;
  double ph_re = 1.0, ph_im = 0.0;
  double phase = 0.0;
  if (a.dphase) {
    phase = __ddiv_rn(__dmul_rn(__dmul_rn(-2.0 * 3.141592653589793, a.dphase[tb]), f), a.c);
    sincos(phase, &ph_im, &ph_re);
  } else {
    phase = __ddiv_rn(__dmul_rn(__dmul_rn(-2.0 * 3.141592653589793, 0.0), f), a.c);
    ph_re = 1.0;
    ph_im = phase;  // sin(+-0) = +-0
  }
  double nv_re = 0.0, nv_im = 0.0, norm = 0.0;
  const int64_t plane = ((int64_t)achan * a.g_npol + apol) * a.g_n2 * a.g_n3;
  for (long long ix = beg; ix < end; ++ix) {
    long long i1 = (long long)a.sampling * ix + o0;
    double wtx = a.cf[i1 < 0 ? -i1 : i1];
    for (long long iy = beg; iy < end; ++iy) {
      long long i2 = (long long)a.sampling * iy + o1;
      double wty = a.cf[i2 < 0 ? -i2 : i2];
      double wt = __dmul_rn(wtx, wty);
      norm = __dadd_rn(norm, wt);
      int64_t gi = plane + ((int64_t)x0 + ix) * a.g_n3 + ((int64_t)y0 + iy);
      double gr, gim;
      if (a.grid_c128) {
        double2 gv = ((const double2 *)a.grid)[gi];
        gr = gv.x; gim = gv.y;
      } else {
        float2 gv = ((const float2 *)a.grid)[gi];
        gr = gv.x; gim = gv.y;
      }
      nv_re = __dadd_rn(nv_re, __dmul_rn(wt, gr));
      nv_im = __dadd_rn(nv_im, __dmul_rn(wt, gim));
    }
  }
  if (norm != 0.0) {
    double cr = ph_re, ci = -ph_im;
    double pr = __dsub_rn(__dmul_rn(nv_re, cr), __dmul_rn(nv_im, ci));
    double pi = __dadd_rn(__dmul_rn(nv_re, ci), __dmul_rn(nv_im, cr));
    if (a.values_c128) {
      double2 *o = (double2 *)a.values + k;
      double2 cur = *o;
      *o = make_double2(__dadd_rn(cur.x, __ddiv_rn(pr, norm)), __dadd_rn(cur.y, __ddiv_rn(pi, norm)));
    } else {
      float2 *o = (float2 *)a.values + k;
      float2 cur = *o;
      *o = make_float2((float)((double)cur.x + pr / norm), (float)((double)cur.y + pi / norm));
    }
  }
}

// Adjoint of k_degrid_plain: grid[c, p, x, y] += w / norm * phasor * values
// for each unflagged sample (FP64, atomics), with the degridder's exact
// positions - the gradient of the degridder for finite-difference checks.
__global__ void __launch_bounds__(256) k_degrid_adjoint_plain(DegridArgs a) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t total = a.nt * a.nb * a.nvchan * a.nvpol;
  if (k >= total) return;
  int64_t row = k / a.nvpol;
  int ipol = (int)(k - row * a.nvpol);
  int64_t tb = row / a.nvchan;
  int ichan = (int)(row - tb * a.nvchan);
  int apol = a.polmap[ipol];
  if (!(0 <= apol && apol < a.g_npol)) return;
  int achan = a.chanmap[ichan];
  if (!(0 <= achan && achan < a.g_nchan)) return;
  if (a.flag && a.flag[k]) return;
  const double f = a.freq[ichan];
  double p0 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(a.scale0, a.uvw[3 * tb]), f), a.c), a.offset0);
  double p1 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(a.scale1, a.uvw[3 * tb + 1]), f), a.c), a.offset1);
  int x0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p0));
  int y0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p1));
  int o0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(__dmul_rn(__dsub_rn((double)x0, p0), (double)a.sampling)));
  int o1 = (int)(unsigned)(unsigned long long)trunc_ll(rint(__dmul_rn(__dsub_rn((double)y0, p1), (double)a.sampling)));
  const long long beg = -(a.support / 2), end = beg + a.support;
  if (!(((long long)x0 + beg >= 0) && ((long long)x0 + end - 1 < a.g_n3) &&
        ((long long)y0 + beg >= 0) && ((long long)y0 + end - 1 < a.g_n2)))
    return;
  if (!((long long)x0 + end - 1 < a.g_n2 && (long long)y0 + end - 1 < a.g_n3)) return;
  double norm = 0.0;
  for (long long ix = beg; ix < end; ++ix) {
    long long i1 = (long long)a.sampling * ix + o0;
    double wtx = a.cf[i1 < 0 ? -i1 : i1];
    for (long long iy = beg; iy < end; ++iy) {
      long long i2 = (long long)a.sampling * iy + o1;
      norm = __dadd_rn(norm, __dmul_rn(wtx, a.cf[i2 < 0 ? -i2 : i2]));
    }
  }
  if (norm == 0.0) return;
  double vr, vi;
  if (a.values_c128) {
    double2 v = ((const double2 *)a.values)[k];
    vr = v.x; vi = v.y;
  } else {
    float2 v = ((const float2 *)a.values)[k];
    vr = v.x; vi = v.y;
  }
  if (a.dphase) {
    double phase = __ddiv_rn(__dmul_rn(__dmul_rn(-2.0 * 3.141592653589793, a.dphase[tb]), f), a.c);
    double s, c;
    sincos(phase, &s, &c);
    double r = vr * c - vi * s, i = vr * s + vi * c;  // values * phasor
    vr = r;
    vi = i;
  }
  vr /= norm;
  vi /= norm;
  const int64_t plane = ((int64_t)achan * a.g_npol + apol) * a.g_n2 * a.g_n3;
  for (long long ix = beg; ix < end; ++ix) {
    long long i1 = (long long)a.sampling * ix + o0;
    double wtx = a.cf[i1 < 0 ? -i1 : i1];
    for (long long iy = beg; iy < end; ++iy) {
      long long i2 = (long long)a.sampling * iy + o1;
      double wt = wtx * a.cf[i2 < 0 ? -i2 : i2];
      int64_t gi = plane + ((int64_t)x0 + ix) * a.g_n3 + ((int64_t)y0 + iy);
      if (a.grid_c128) {
        atomicAdd(&((double2 *)a.grid)[gi].x, wt * vr);
        atomicAdd(&((double2 *)a.grid)[gi].y, wt * vi);
      } else {
        atomicAdd(&((float2 *)a.grid)[gi].x, (float)(wt * vr));
        atomicAdd(&((float2 *)a.grid)[gi].y, (float)(wt * vi));
      }
    }
  }
}

// ---------------------------------------------------------------- tiled ----
constexpr int DT_THREADS = 256;

struct TiledDegridArgs {
  const Rec *recs;
  const uint32_t *tile_start;
  const uint32_t *n_rec;    // device: usable records (offs[n_keys])
  const uint32_t *exc_mark; // device: a shared plan's marks (zero otherwise)
  int64_t n_rows;           // all samples (the plan also lists skipped ones)
  int64_t n_tiles, ntu, ntv, chunk;
  DegridArgs d;
  int cgk_len;
  uint32_t *sched;          // device: [0] next chunk, [1] CTAs done (0 between launches)
  int accumulate;           // 1: values +=, 0: values = (skipped samples get 0)
  // complex64 store mode, 4 visibility polarisations, no flags, no phase,
  // values 32-byte aligned: a sample's 4 values go out as two 16-byte stores
  int fast_out;
};

template <int S, int NPG>
struct DSmem {
  static constexpr int W = TILE + S - 1;
  static constexpr int RW = (S + 3) & ~3;  // tap-table row (floats)
  static constexpr size_t tab_bytes = 256 * RW * sizeof(float);
  static constexpr size_t rs_bytes = 256 * sizeof(double);
  static constexpr size_t sub_bytes = (size_t)W * W * NPG * sizeof(float2);  // [cell][pol]
  static constexpr size_t total = tab_bytes + rs_bytes + sub_bytes;
};

template <int S, int RW>
__device__ void build_tap_tables_d(float *tab, double *rs, const double *cgk, int cgk_len,
                                   int os) {
  for (int o = threadIdx.x; o < 256; o += blockDim.x) {
    int off = o - 128;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < RW; ++i) {
      double v = 0.0;
      if (i < S) {
        int k = os * (i - S / 2) + off;
        k = k < 0 ? -k : k;
        v = (k < cgk_len) ? cgk[k] : 0.0;
        s += v;
      }
      tab[o * RW + i] = (float)v;
    }
    rs[o] = s;
  }
}

// Taps of offset o - 128 (the reference's kernel indices |sampling ix + off|,
// standard_degrid.py:466-469) divided by their FP64 sum, so that the product
// of a sample's row and column taps carries its 1 / norm (the reference's
// norm, the sum of the 2-D taps, standard_degrid.py:464-485, is the product
// of the two sums); a zero sum gives zero taps (and a zero value, as norm ==
// 0 does in the reference).  tab[o * RW + i], zero past the support.
template <int S, int RW>
__device__ void build_norm_tap_tables(float *tab, const double *cgk, int cgk_len, int os) {
  for (int o = threadIdx.x; o < 256; o += blockDim.x) {
    const int off = o - 128;
    double v[RW], s = 0.0;
#pragma unroll
    for (int i = 0; i < RW; ++i) {
      v[i] = 0.0;
      if (i < S) {
        int k = os * (i - S / 2) + off;
        k = k < 0 ? -k : k;
        v[i] = (k < cgk_len) ? cgk[k] : 0.0;
        s += v[i];
      }
    }
#pragma unroll
    for (int i = 0; i < RW; ++i) tab[o * RW + i] = s != 0.0 ? (float)(v[i] / s) : 0.f;
  }
}

__device__ __forceinline__ void put_value(const DegridArgs &d, int accumulate, int64_t k,
                                          double vr, double vi) {
  if (d.values_c128) {
    double2 *o = (double2 *)d.values + k;
    if (accumulate) {
      double2 cur = *o;
      vr += cur.x;
      vi += cur.y;
    }
    *o = make_double2(vr, vi);
  } else {
    float2 *o = (float2 *)d.values + k;
    float2 v = make_float2((float)vr, (float)vi);
    if (accumulate) {
      float2 cur = *o;
      v.x += cur.x;
      v.y += cur.y;
    }
    *o = v;
  }
}

// Writes one sample's degridded values (all visibility polarisations):
// normalised by sum_k w_k, phase-rotated when dphase is given, zeros in store
// mode for flagged, unmapped and zero-norm samples.
template <int NPG>
__device__ __forceinline__ void degrid_write(const TiledDegridArgs &a, const DegridArgs &d,
                                             const double *rs, const int (&pmv)[8],
                                             const Rec &rc, bool marked,
                                             const float2 (&acc)[NPG]) {
  const double norm = rs[rc.ou] * rs[rc.ov];
  const int64_t row_i = rc.row;
  if (marked) {
    // a shared plan's sample whose degridder convention differs: zeros in
    // store mode (k_degrid_exceptions then writes the ones the degridder
    // keeps), nothing when accumulating
    if (!a.accumulate) {
      if (a.fast_out) {
        float4 *o = (float4 *)((float2 *)d.values + row_i * 4);
        o[0] = make_float4(0.f, 0.f, 0.f, 0.f);
        o[1] = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        for (int p = 0; p < d.nvpol; ++p) put_value(d, 0, row_i * d.nvpol + p, 0.0, 0.0);
      }
    }
    return;
  }
  if (a.fast_out) {
    // 1 / norm in FP64, the scaling in FP32 (one more rounding, ~6e-8)
    const float inv = norm != 0.0 ? (float)(1.0 / norm) : 0.f;
    float2 v[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int apol = pmv[p];
      float2 x = make_float2(0.f, 0.f);
#pragma unroll
      for (int gp = 0; gp < NPG; ++gp)
        if (apol == gp) x = acc[gp];
      // zero-norm samples and unmapped polarisations get 0, as in store mode
      v[p] = (apol >= 0 && norm != 0.0) ? make_float2(__fmul_rn(x.x, inv), __fmul_rn(x.y, inv))
                                        : make_float2(0.f, 0.f);
    }
    float4 *o = (float4 *)((float2 *)d.values + row_i * 4);
    o[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    o[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
    return;
  }
  if (norm == 0.0) {  // the reference leaves such samples untouched
    if (!a.accumulate)
      for (int p = 0; p < d.nvpol; ++p) put_value(d, 0, row_i * d.nvpol + p, 0.0, 0.0);
    return;
  }
  double ph_re = 1.0, ph_im = 0.0;
  if (d.dphase) {
    const int64_t tb = row_i / d.nvchan;
    const int ichan = (int)(row_i - tb * d.nvchan);
    double phase = (-2.0 * 3.141592653589793 * d.dphase[tb]) * d.freq[ichan] / d.c;
    sincos(phase, &ph_im, &ph_re);
  }
  const double inv = 1.0 / norm;
  for (int p = 0; p < d.nvpol; ++p) {
    const int64_t k = row_i * d.nvpol + p;
    const int apol = p < 8 ? pmv[p] : -1;
    if (apol < 0 || (d.flag && d.flag[k])) {
      if (!a.accumulate) put_value(d, 0, k, 0.0, 0.0);
      continue;
    }
    float2 v = acc[0];
#pragma unroll
    for (int gp = 1; gp < NPG; ++gp)
      if (apol == gp) v = acc[gp];
    double vr = v.x, vi = v.y;
    if (d.dphase) {
      const double cr = ph_re, ci = -ph_im;
      const double pr = vr * cr - vi * ci, pi = vr * ci + vi * cr;
      vr = pr;
      vi = pi;
    }
    put_value(d, a.accumulate, k, vr * inv, vi * inv);
  }
}

// Stages a tile's sub-grid (W x W cells from tile (tu, tv) of `plane`, the
// NPG grid polarisations interleaved per cell, zero outside the grid) into
// shared memory as float2.  SUB_UNROLL loads per thread are issued before
// their stores, so a thread has several grid reads in flight.  The loop trip
// count is the same for the whole block.
constexpr int SUB_UNROLL = 4;

template <int W, int NPG, int THREADS>
__device__ __forceinline__ void stage_subgrid(const DegridArgs &d, float2 *sub, int64_t plane,
                                              int tu, int tv, int64_t gplane) {
  constexpr int N = W * W * NPG;
  for (int i0 = 0; i0 < N; i0 += THREADS * SUB_UNROLL) {
    float2 v[SUB_UNROLL];
#pragma unroll
    for (int k = 0; k < SUB_UNROLL; ++k) {
      const int i = i0 + k * THREADS + (int)threadIdx.x;
      v[k] = make_float2(0.f, 0.f);
      const int cell = i / NPG, gp = i - cell * NPG;
      const int iu = cell / W, iv = cell - iu * W;
      const int64_t gu = (int64_t)tu * TILE + iu, gv = (int64_t)tv * TILE + iv;
      if (i < N && gp < d.g_npol && gu < d.g_n2 && gv < d.g_n3) {
        const int64_t gi = (plane * d.g_npol + gp) * gplane + gu * d.g_n3 + gv;
        if (d.grid_c128) {
          const double2 x = ((const double2 *)d.grid)[gi];
          v[k] = make_float2((float)x.x, (float)x.y);
        } else {
          v[k] = ((const float2 *)d.grid)[gi];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < SUB_UNROLL; ++k) {
      const int i = i0 + k * THREADS + (int)threadIdx.x;
      if (i < N) sub[i] = v[k];
    }
  }
}

template <int S, int NPG>
__global__ void __launch_bounds__(DT_THREADS) k_degrid_tiled(TiledDegridArgs a) {
  using M = DSmem<S, NPG>;
  constexpr int W = M::W, RW = M::RW;
  extern __shared__ __align__(16) unsigned char smem[];
  float *tab = (float *)smem;
  double *rs = (double *)(smem + M::tab_bytes);
  float2 *sub = (float2 *)(smem + M::tab_bytes + M::rs_bytes);
  const DegridArgs &d = a.d;

  __shared__ int s_chunk;
  const uint32_t n_rec = *a.n_rec;
  const uint32_t n_all = a.accumulate ? n_rec : (uint32_t)a.n_rows;
  const int64_t n_chunks = ((int64_t)n_all + a.chunk - 1) / a.chunk;
  build_tap_tables_d<S, RW>(tab, rs, d.cf, a.cgk_len, d.sampling);
  int pmv[8];
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    int v = p < d.nvpol ? d.polmap[p] : -1;
    pmv[p] = (v >= 0 && v < NPG && v < d.g_npol) ? v : -1;
  }
  const int64_t gplane = d.g_n2 * d.g_n3;

  // persistent: chunks of records from a.sched[0] until none are left
  for (;;) {
  __syncthreads();  // tables built; the previous chunk is done with sub and s_chunk
  if (threadIdx.x == 0) s_chunk = (int)atomicAdd(&a.sched[0], 1u);
  __syncthreads();
  const int64_t ch = s_chunk;
  if (ch >= n_chunks) break;
  const uint32_t r0 = (uint32_t)(ch * a.chunk);
  const uint32_t r1 = (uint32_t)min((int64_t)n_all, (int64_t)r0 + a.chunk);
  // store mode: skipped samples (after the usable records) get zeros
  if (!a.accumulate && r1 > n_rec) {
    const uint32_t z0 = max(r0, n_rec);
    for (uint32_t rb = z0; rb < r1; rb += DT_THREADS) {
      const uint32_t r = rb + threadIdx.x;
      if (r >= r1) continue;
      const int64_t row = a.recs[r].row;
      for (int p = 0; p < d.nvpol; ++p) put_value(d, 0, row * d.nvpol + p, 0.0, 0.0);
    }
  }
  const uint32_t v1 = min(r1, n_rec);
  if (r0 >= v1) continue;

  int t = find_tile_warp(a.tile_start, a.n_tiles, r0);
  uint32_t seg_lo = r0;
  while (seg_lo < v1) {
    uint32_t t_end = a.tile_start[t + 1];
    uint32_t seg_hi = min(v1, t_end);
    if (seg_hi <= seg_lo) {
      ++t;
      continue;
    }
    const int64_t plane = t / (a.ntu * a.ntv);
    const int64_t trem = t - plane * a.ntu * a.ntv;
    const int tu = (int)(trem / a.ntv), tv = (int)(trem - (int64_t)tu * a.ntv);
    __syncthreads();  // previous segment's readers are done with sub
    stage_subgrid<W, NPG, DT_THREADS>(d, sub, plane, tu, tv, gplane);
    __syncthreads();
    // each thread takes a pair of consecutive records: cell-sorted records
    // usually share the cell, and then one read of the footprint serves
    // both samples; a pair that straddles two cells reads the second
    // footprint with loads predicated on the lanes that need it
    // records (and whether a shared plan marks them for the degridder's FP64
    // pass) are loaded one step ahead
    Rec nxa, nxb;
    bool nma = false, nmb = false;
    {
      const uint32_t r = seg_lo + 2 * threadIdx.x;
      if (r < seg_hi) {
        nxa = a.recs[r];
        nma = degrid_marked(a.exc_mark, r);
      }
      if (r + 1 < seg_hi) {
        nxb = a.recs[r + 1];
        nmb = degrid_marked(a.exc_mark, r + 1);
      }
    }
    // one trip count per block, so every warp reaches the next barrier converged
    for (uint32_t rb = seg_lo; rb < seg_hi; rb += 2 * DT_THREADS) {
      const uint32_t r = rb + 2 * threadIdx.x;
      const Rec ra = nxa, rbx = nxb;
      const bool ma = nma, mb = nmb;
      {
        const uint32_t rn = r + 2 * DT_THREADS;
        if (rn < seg_hi) {
          nxa = a.recs[rn];
          nma = degrid_marked(a.exc_mark, rn);
        }
        if (rn + 1 < seg_hi) {
          nxb = a.recs[rn + 1];
          nmb = degrid_marked(a.exc_mark, rn + 1);
        }
      }
      if (r >= seg_hi) continue;
      const bool has_b = r + 1 < seg_hi;
      const Rec rcb = has_b ? rbx : ra;
      float cua[RW], cva[RW], cub[RW], cvb[RW];
#pragma unroll
      for (int k = 0; k < RW; k += 4) {
        const float4 a4 = *(const float4 *)&tab[ra.ou * RW + k];
        const float4 b4 = *(const float4 *)&tab[ra.ov * RW + k];
        const float4 c4 = *(const float4 *)&tab[rcb.ou * RW + k];
        const float4 d4 = *(const float4 *)&tab[rcb.ov * RW + k];
        cua[k] = a4.x; cua[k + 1] = a4.y; cua[k + 2] = a4.z; cua[k + 3] = a4.w;
        cva[k] = b4.x; cva[k + 1] = b4.y; cva[k + 2] = b4.z; cva[k + 3] = b4.w;
        cub[k] = c4.x; cub[k + 1] = c4.y; cub[k + 2] = c4.z; cub[k + 3] = c4.w;
        cvb[k] = d4.x; cvb[k + 1] = d4.y; cvb[k + 2] = d4.z; cvb[k + 3] = d4.w;
      }
      const bool same = rcb.du == ra.du && rcb.dv == ra.dv;
      float2 acca[NPG], accb[NPG];
#pragma unroll
      for (int gp = 0; gp < NPG; ++gp) {
        acca[gp] = make_float2(0.f, 0.f);
        accb[gp] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < S; ++i) {
        float2 rowa[NPG], rowb[NPG];
#pragma unroll
        for (int gp = 0; gp < NPG; ++gp) {
          rowa[gp] = make_float2(0.f, 0.f);
          rowb[gp] = make_float2(0.f, 0.f);
        }
        const float2 *pa = sub + ((ra.du + i) * W + ra.dv) * NPG;
        const float2 *pb = sub + ((rcb.du + i) * W + rcb.dv) * NPG;
#pragma unroll
        for (int j = 0; j < S; ++j) {
          float2 ga[NPG], gb[NPG];
          if (NPG >= 2) {
#pragma unroll
            for (int gp = 0; gp < NPG; gp += 2) {
              const float4 qa = *(const float4 *)(pa + j * NPG + gp);
              float4 qb = qa;
              if (!same) qb = *(const float4 *)(pb + j * NPG + gp);
              ga[gp] = make_float2(qa.x, qa.y);
              ga[(gp + 1) % NPG] = make_float2(qa.z, qa.w);
              gb[gp] = make_float2(qb.x, qb.y);
              gb[(gp + 1) % NPG] = make_float2(qb.z, qb.w);
            }
          } else {
            ga[0] = pa[j];
            gb[0] = ga[0];
            if (!same) gb[0] = pb[j];
          }
#pragma unroll
          for (int gp = 0; gp < NPG; ++gp) {
            rowa[gp] = __ffma2_rn(make_float2(cva[j], cva[j]), ga[gp], rowa[gp]);
            rowb[gp] = __ffma2_rn(make_float2(cvb[j], cvb[j]), gb[gp], rowb[gp]);
          }
        }
#pragma unroll
        for (int gp = 0; gp < NPG; ++gp) {
          acca[gp] = __ffma2_rn(make_float2(cua[i], cua[i]), rowa[gp], acca[gp]);
          accb[gp] = __ffma2_rn(make_float2(cub[i], cub[i]), rowb[gp], accb[gp]);
        }
      }
      degrid_write<NPG>(a, d, rs, pmv, ra, ma, acca);
      if (has_b) degrid_write<NPG>(a, d, rs, pmv, rcb, mb, accb);
    }
    seg_lo = seg_hi;
    if (seg_hi == t_end) ++t;
  }
  }
  // every CTA has taken its last chunk: the last one to get here re-arms
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.sched[1], 1u) == gridDim.x - 1) {
      a.sched[0] = 0u;
      a.sched[1] = 0u;
      __threadfence();
    }
  }
}

// ------------------------------------------------------- tensor cores ----
// k_degrid_tc: the tiled degridder's fast store path (complex64 values, 4
// visibility and 4 grid polarisations, no flags, no phase) on the TF32 tensor
// path.  For one cell, 16 samples and each footprint row r, the column sums
// are a matrix product,
//   D_r[m][q] = sum over c of cv_m[c] P[q][r][c],
// with cv_m the sample's column taps and P[q][r][c] the cell's footprint value
// at row r, column c for output q = (output polarisation, real | imaginary):
// one mma.sync.m16n8k8.tf32 per row (n = 8 outputs, k = 8 columns), rows at
// or past the support skipped.  Then V[m][q] = sum over r of cu_m[r]
// D_r[m][q] accumulates on the FP32 pipe in the lane that holds D_r[m][q]
// (row and column taps come divided by their tap sums, so V carries
// 1 / norm).  TF32 keeps 11 significant bits, so both operands are split into
// a TF32 high part and the TF32-rounded remainder (the taps once, in a table;
// the patch once per cell) and the products hi.hi, hi.lo and lo.hi are
// accumulated in FP32: what is left out is below 2^-22 of each product.
// Fragment layout (lane = 4 g + t): a = cv[g][t], cv[g + 8][t], cv[g][t + 4],
// cv[g + 8][t + 4] (samples g and g + 8); b = P[q = g][r][t], P[g][r][t + 4]
// (output g, read from grid polarisation polmap[g / 2]); d = D_r[g][2t],
// D_r[g][2t + 1], D_r[g + 8][2t], D_r[g + 8][2t + 1].  Lane (g, t) thus owns
// the real and imaginary parts of output polarisation t of samples g and
// g + 8, sums them over the rows with its row taps, and writes them: no
// shuffles.
constexpr int TC_THREADS = 256;
constexpr int TC_ROUND = 64;  // records a warp stages per round (two per lane)

template <int S>
struct TCSmem {
  static constexpr int W = TILE + S - 1;
  static constexpr int RW = 8;  // taps 0-7 of a row, zero past the support
  static constexpr size_t tab_bytes = 256 * RW * sizeof(float);
  // the same taps split into TF32 (high, remainder) pairs
  static constexpr size_t tabs_bytes = 256 * RW * sizeof(uint2);
  static constexpr size_t rec_bytes = (size_t)(TC_THREADS / 32) * TC_ROUND * sizeof(Rec);
  static constexpr size_t off_tabs = tab_bytes;
  static constexpr size_t off_rec = off_tabs + tabs_bytes;
  static constexpr size_t off_sub = off_rec + rec_bytes;
  static constexpr size_t sub_bytes = (size_t)W * W * 4 * sizeof(float2);  // [cell][pol]
  static constexpr size_t total = off_sub + sub_bytes;
  static_assert(off_sub % 16 == 0, "alignment");
  static_assert(S <= 8, "an 8 x 8 footprint");
};

// x rounded to TF32 (10 stored mantissa bits), to nearest with ties away
// from zero, as a float bit pattern whose low 13 bits are zero: the same
// result as cvt.rna.tf32.f32, computed on the integer pipe (the conversion
// unit's throughput is far lower).  Adding half a TF32 unit to the magnitude
// bits and truncating rounds the magnitude up at a tie; a carry into the
// exponent gives the next binade, or infinity past the largest value.  NaN
// becomes the canonical NaN (its payload could otherwise carry into the sign).
__device__ __forceinline__ uint32_t tf32_rna(float x) {
  const uint32_t b = __float_as_uint(x);
  const uint32_t r = (b + 0x1000u) & 0xFFFFE000u;
  return (b & 0x7FFFFFFFu) > 0x7F800000u ? 0x7FFFFFFFu : r;
}

// x = hi + lo, both TF32 (lo: the remainder rounded to TF32)
__device__ __forceinline__ void tf32_split(float x, uint32_t &hi, uint32_t &lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int S>
__global__ void __launch_bounds__(TC_THREADS, 2) k_degrid_tc(TiledDegridArgs a) {
  using M = TCSmem<S>;
  constexpr int W = M::W, RW = M::RW, WARPS = TC_THREADS / 32;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  float *tab = (float *)smem;
  uint2 *tabs = (uint2 *)(smem + M::off_tabs);
  Rec *st_rec = (Rec *)(smem + M::off_rec);
  float2 *sub = (float2 *)(smem + M::off_sub);
  const DegridArgs &d = a.d;

  __shared__ int s_chunk;
  const uint32_t n_rec = *a.n_rec;
  const uint32_t n_all = (uint32_t)a.n_rows;  // store mode: every sample is written
  const int64_t n_chunks = ((int64_t)n_all + a.chunk - 1) / a.chunk;
  // row and column taps over their sums: the products carry 1 / norm
  build_norm_tap_tables<S, RW>(tab, d.cf, a.cgk_len, d.sampling);
  __syncthreads();
  for (int i = threadIdx.x; i < 256 * RW; i += TC_THREADS) {
    uint2 hl;
    tf32_split(tab[i], hl.x, hl.y);
    tabs[i] = hl;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  // this lane writes output polarisation t (from grid polarisation polmap[t]);
  // its B column is output q = g: polarisation g / 2 (from grid polarisation
  // bsrc), real or imaginary part g % 2
  int src = -1, bsrc = -1;
  {
    const int v = d.polmap[t];
    if (v >= 0 && v < 4 && v < d.g_npol) src = v;
    const int u = d.polmap[g >> 1];
    if (u >= 0 && u < 4 && u < d.g_npol) bsrc = u;
  }
  const int64_t gplane = d.g_n2 * d.g_n3;

  for (;;) {
    __syncthreads();  // tables built; the previous chunk is done with sub and s_chunk
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(&a.sched[0], 1u);
    __syncthreads();
    const int64_t ch = s_chunk;
    if (ch >= n_chunks) break;
    const uint32_t r0 = (uint32_t)(ch * a.chunk);
    const uint32_t r1 = (uint32_t)min((int64_t)n_all, (int64_t)r0 + a.chunk);
    if (r1 > n_rec) {  // skipped samples (after the usable records) get zeros
      const uint32_t z0 = max(r0, n_rec);
      for (uint32_t rb = z0; rb < r1; rb += TC_THREADS) {
        const uint32_t r = rb + threadIdx.x;
        if (r >= r1) continue;
        const int64_t row = a.recs[r].row;
        for (int p = 0; p < 4; ++p) put_value(d, 0, row * 4 + p, 0.0, 0.0);
      }
    }
    const uint32_t v1 = min(r1, n_rec);
    if (r0 >= v1) continue;

    int tt = find_tile_warp(a.tile_start, a.n_tiles, r0);
    uint32_t seg_lo = r0;
    while (seg_lo < v1) {
      const uint32_t t_end = a.tile_start[tt + 1];
      const uint32_t seg_hi = min(v1, t_end);
      if (seg_hi <= seg_lo) {
        ++tt;
        continue;
      }
      const int64_t plane = tt / (a.ntu * a.ntv);
      const int64_t trem = tt - plane * a.ntu * a.ntv;
      const int tu = (int)(trem / a.ntv), tv = (int)(trem - (int64_t)tu * a.ntv);
      __syncthreads();  // previous segment's readers are done with sub
      stage_subgrid<W, 4, TC_THREADS>(d, sub, plane, tu, tv, gplane);
      __syncthreads();

      // this warp's slice of the segment, in rounds of 64 records (two per
      // lane): records go to the warp's staging area, from which the lanes of
      // a group read the samples they need
      const uint32_t seg_n = seg_hi - seg_lo;
      const uint32_t w_lo = seg_lo + (uint32_t)(((uint64_t)seg_n * warp) / WARPS);
      const uint32_t w_hi = seg_lo + (uint32_t)(((uint64_t)seg_n * (warp + 1)) / WARPS);
      const int n_rounds = (int)((w_hi - w_lo + TC_ROUND - 1) / TC_ROUND);
      Rec *wrec = st_rec + warp * TC_ROUND;
      int cur = -1;
      // patch fragments of the current cell, one k x n tile per footprint
      // row r: b = P[q = g][r][c = t, t + 4]
      uint32_t bh[8][2], bl[8][2];
#pragma unroll
      for (int q = 0; q < 8; ++q) bh[q][0] = bh[q][1] = bl[q][0] = bl[q][1] = 0u;
      // records and their mark words (a shared plan's samples marked for
      // the degridder's FP64 pass) are loaded one round ahead
      Rec na, nb;
      uint32_t nma = 0u, nmb = 0u;
      if (w_lo + lane < w_hi) {
        na = a.recs[w_lo + lane];
        nma = __ldg(a.exc_mark + ((w_lo + lane) >> 5));
      }
      if (w_lo + 32 + lane < w_hi) {
        nb = a.recs[w_lo + 32 + lane];
        nmb = __ldg(a.exc_mark + ((w_lo + 32 + lane) >> 5));
      }
      for (int rd = 0; rd < n_rounds; ++rd) {
        const uint32_t r = w_lo + (uint32_t)rd * TC_ROUND + lane;
        const bool va = r < w_hi, vb = r + 32 < w_hi;
        const Rec ra = na, rb = nb;
        const uint32_t ma = nma, mb = nmb;
        if (r + TC_ROUND < w_hi) {
          na = a.recs[r + TC_ROUND];
          nma = __ldg(a.exc_mark + ((r + TC_ROUND) >> 5));
        }
        if (r + TC_ROUND + 32 < w_hi) {
          nb = a.recs[r + TC_ROUND + 32];
          nmb = __ldg(a.exc_mark + ((r + TC_ROUND + 32) >> 5));
        }
        const int ka = va ? ((int)ra.du | ((int)ra.dv << 8)) : -1;
        const int kb = vb ? ((int)rb.du | ((int)rb.dv << 8)) : -1;
        __syncwarp();  // the previous round's groups are done with the staging area
        // staged records carry a shared plan's mark in the row's top bit (the
        // host runs this kernel only for fewer than 2^31 rows)
        if (va) {
          Rec x = ra;
          if ((ma >> (r & 31u)) & 1u) x.row |= REC_DEGRID_EXC;
          wrec[lane] = x;
        }
        if (vb) {
          Rec x = rb;
          if ((mb >> ((r + 32) & 31u)) & 1u) x.row |= REC_DEGRID_EXC;
          wrec[lane + 32] = x;
        }
        int pa = __shfl_up_sync(FULL, ka, 1);
        if (lane == 0) pa = cur;
        int pb = __shfl_up_sync(FULL, kb, 1);
        const int ka_last = __shfl_sync(FULL, ka, 31);
        if (lane == 0) pb = ka_last;
        const unsigned long long starts =
            (unsigned long long)__ballot_sync(FULL, ka >= 0 && ka != pa) |
            ((unsigned long long)__ballot_sync(FULL, kb >= 0 && kb != pb) << 32);
        __syncwarp();
        const int jn = (int)min((uint32_t)TC_ROUND, w_hi - (w_lo + (uint32_t)rd * TC_ROUND));
        // a run starts at sample j: its cell's patch, split, into bh / bl
        // (this lane: output q = g, footprint rows 0 .. S - 1, columns t and
        // t + 4; the real or imaginary part of grid polarisation bsrc)
        auto load_patch = [&](const int j) {
          const Rec rj = wrec[j];
          cur = (int)rj.du | ((int)rj.dv << 8);
          const int du = rj.du, dv = rj.dv;
          const float *sf = (const float *)sub + (g & 1);
#pragma unroll
          for (int r = 0; r < S; ++r) {
            float x0 = 0.f, x1 = 0.f;
            if (bsrc >= 0) {
              const int e = ((du + r) * W + dv + t) * 4 + bsrc;
              if (t < S) x0 = sf[2 * e];
              if (t + 4 < S) x1 = sf[2 * (e + 16)];  // 4 columns on
            }
            tf32_split(x0, bh[r][0], bl[r][0]);
            tf32_split(x1, bh[r][1], bl[r][1]);
          }
        };
        // one group of 16 samples [j0, j0 + 16) of a run ending at j1
        auto group = [&](const int j0, const int j1) {
          // samples j0 + g and j0 + g + 8 of the round (an empty slot reads
          // sample j0 and contributes a zero row of W)
          const int sg = j0 + g, sh = j0 + g + 8;
          const bool vg = sg < j1, vh = sh < j1;
          const Rec recg = wrec[vg ? sg : j0], rech = wrec[vh ? sh : j0];
          const int oug = recg.ou, ovg = recg.ov, ouh = rech.ou, ovh = rech.ov;
          // A = the column taps of samples g and g + 8 (columns t, t + 4),
          // split in the table; an empty slot is a zero row
          const uint2 z = make_uint2(0u, 0u);
          const uint2 ag0 = vg ? tabs[ovg * RW + t] : z, ag1 = vg ? tabs[ovg * RW + t + 4] : z;
          const uint2 ah0 = vh ? tabs[ovh * RW + t] : z, ah1 = vh ? tabs[ovh * RW + t + 4] : z;
          // row taps of samples g and g + 8
          const float4 cg0 = *(const float4 *)&tab[oug * RW];
          const float4 cg1 = *(const float4 *)&tab[oug * RW + 4];
          const float4 ch0 = *(const float4 *)&tab[ouh * RW];
          const float4 ch1 = *(const float4 *)&tab[ouh * RW + 4];
          const float cug[8] = {cg0.x, cg0.y, cg0.z, cg0.w, cg1.x, cg1.y, cg1.z, cg1.w};
          const float cuh[8] = {ch0.x, ch0.y, ch0.z, ch0.w, ch1.x, ch1.y, ch1.z, ch1.w};
          // per footprint row r: D_r[m][q] = sum_c cv_m[c] P[q][r][c] (three
          // TF32 products), of which this lane holds outputs q = 2t, 2t + 1
          // (polarisation t, real and imaginary) of samples g and g + 8, and
          // V[m][q] = sum_r cu_m[r] D_r[m][q] accumulates in the lane
          float xgre = 0.f, xgim = 0.f, xhre = 0.f, xhim = 0.f;
  #pragma unroll
          for (int r = 0; r < S; ++r) {
            float dr[4] = {0.f, 0.f, 0.f, 0.f};
            mma_tf32(dr, ag0.y, ah0.y, ag1.y, ah1.y, bh[r][0], bh[r][1]);
            mma_tf32(dr, ag0.x, ah0.x, ag1.x, ah1.x, bl[r][0], bl[r][1]);
            mma_tf32(dr, ag0.x, ah0.x, ag1.x, ah1.x, bh[r][0], bh[r][1]);
            xgre = __fmaf_rn(cug[r], dr[0], xgre);
            xgim = __fmaf_rn(cug[r], dr[1], xgim);
            xhre = __fmaf_rn(cuh[r], dr[2], xhre);
            xhim = __fmaf_rn(cuh[r], dr[3], xhim);
          }
          // a shared plan's marked sample gets 0 here (k_degrid_exceptions
          // writes the ones the degridder keeps)
          float2 *out = (float2 *)d.values;
          const bool ug = (recg.row & REC_DEGRID_EXC) == 0u;
          const bool uh = (rech.row & REC_DEGRID_EXC) == 0u;
          if (vg)
            out[(int64_t)(recg.row & ~REC_DEGRID_EXC) * 4 + t] =
                (src >= 0 && ug) ? make_float2(xgre, xgim)
                                 : make_float2(0.f, 0.f);
          if (vh)
            out[(int64_t)(rech.row & ~REC_DEGRID_EXC) * 4 + t] =
                (src >= 0 && uh) ? make_float2(xhre, xhim)
                                 : make_float2(0.f, 0.f);
        };
        int j = 0;
        // a round of one run: its four groups with the run's end known (no
        // empty-slot selects)
        if (starts <= 1ull && jn == TC_ROUND) {
          if (starts) load_patch(0);
#pragma unroll 1
          for (int j0 = 0; j0 < TC_ROUND; j0 += 16) group(j0, TC_ROUND);
          j = jn;
        }
        while (j < jn) {
          if ((starts >> j) & 1ull) load_patch(j);
          const unsigned long long later = j < 63 ? (starts & (~1ull << j)) : 0ull;
          const int j1 = later ? min(jn, __ffsll((long long)later) - 1) : jn;
          for (int j0 = j; j0 < j1; j0 += 16) group(j0, j1);
          j = j1;
        }
      }
      seg_lo = seg_hi;
      if (seg_hi == t_end) ++tt;
    }
  }
  // every CTA has taken its last chunk: the last one to get here re-arms
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.sched[1], 1u) == gridDim.x - 1) {
      a.sched[0] = 0u;
      a.sched[1] = 0u;
      __threadfence();
    }
  }
}

// ------------------------------------------- fifth-generation tensor cores --
// k_degrid_umma: the same fast store path as k_degrid_tc on tcgen05.  A
// warpgroup (128 threads) takes tiles of up to 128 consecutive records of one
// cell and computes the row sums
//   D[m][(p, re|im, r)] = sum over c of cv_m[c] P[(p, re|im, r)][c]
// for the tile's samples in one MMA chain: M = 128 samples, N = 64, K = 8
// columns, TF32 operands from shared memory, FP32 accumulators in tensor
// memory.  Operands are split into TF32 high parts and TF32-rounded
// remainders as in k_degrid_tc; the products lo.hi, hi.lo and hi.hi
// accumulate into the same columns.  Sample m (tensor-memory lane m, thread m
// of the warpgroup) then reads its row of D and forms
//   V[m][p] = sum over r of cu_m[r] D[m][(p, re|im, r)]
// with its row taps: no shuffles, one 32-byte store per sample.  Row and
// column taps come divided by their offsets' tap sums, so V carries the
// sample's 1 / norm (the reference's norm, the sum of the 2-D taps,
// standard_degrid.py:464-485, is the product of the two sums).
//
// Layouts.  Row n of the B operand (output polarisation p, real or imaginary
// part, footprint row r) is n = 16 p + 8 (re|im) + r and reads grid
// polarisation polmap[p].  A and B are stored K-major in 8-row x 16-byte core
// matrices: element (m, c) at byte (m % 8) 16 + (m / 8) 256 + (c / 4) 128 +
// (c % 4) 4.  The sub-grid is staged as one plane per grid polarisation,
// rows RS float2 apart (RS = 8 mod 16: the 16 lanes of a half-warp reading 8
// columns of 2 rows hit distinct banks).
//
// Schedule.  Each window of up to UM_WIN records of a segment (one chunk's
// records in one grid tile) first gets a bitmap of where cells change, so
// every thread finds its tiles' ends alone.  Within a tile the four warps
// work independently: warp j writes its 32 samples' A rows and the B rows of
// output polarisation j, then arrives on the stage's `full` mbarrier; thread
// 0 issues the MMAs when all four have arrived and commits them to the
// stage's `done` mbarrier; each warp then finishes the previous tile from its
// own quarter of the tensor-memory lanes.  Two stages of operands and
// accumulators per warpgroup: the MMA of tile i runs while the warps finish
// tile i - 1 and build tile i + 1.  One CTA of four warpgroups per SM holds
// all 512 tensor-memory columns (4 x 2 stages x 64).  Every wait is bounded: a
// wait that gives up sets g_degrid_fault and the warpgroup's fault word,
// after which its warps stop taking tiles (their remaining samples stay
// unwritten) and the CTA waits once more, bounded, before it frees the
// tensor memory.
constexpr int UM_THREADS = 512;
constexpr int UM_WG = UM_THREADS / 128;
constexpr int UM_SPIN = 1 << 21;     // mbarrier probes before a wait gives up
constexpr uint32_t UM_SLEEP_NS = 1000; // each probe sleeps at most this long (~2 s in all)
constexpr uint32_t UM_STAGE = 12288; // per stage: A hi | A lo | B hi | B lo
constexpr int UM_WIN = 16384;        // records per bitmap window
// set (sticky) when a wait of k_degrid_umma gave up; av_degrid_fault_read
// reads and clears it
__device__ uint32_t g_degrid_fault = 0u;

template <int S>
struct UMSmem {
  static constexpr int W = TILE + S - 1;
  static constexpr int RS = ((W + 7) / 16) * 16 + 8;  // plane row stride, 8 mod 16
  // 256 x 8 FP32 taps, each divided by its offset's tap sum (so that the
  // products of a row's and a column's taps carry 1 / norm), their TF32 high
  // parts and remainders
  static constexpr size_t off_tab = 0;
  static constexpr size_t off_tabh = off_tab + 256 * 8 * 4;
  static constexpr size_t off_tabl = off_tabh + 256 * 8 * 4;
  static constexpr size_t off_ops = off_tabl + 256 * 8 * 4;
  static constexpr size_t off_sub = off_ops + (size_t)UM_WG * 2 * UM_STAGE;
  static constexpr size_t sub_bytes = (size_t)4 * W * RS * sizeof(float2);  // [pol][row][col]
  static constexpr size_t total = off_sub + sub_bytes;
  static_assert(RS >= W && RS % 16 == 8, "plane rows");
  static_assert(off_ops % 1024 == 0 && off_sub % 16 == 0, "alignment");
  // more than half of an SM's shared memory: one CTA (and its 512 tensor-
  // memory columns) per SM
  static_assert(total > 116 * 1024 && total + UM_WIN / 8 + 1024 <= 227 * 1024,
                "one CTA per SM");
  static_assert(S <= 8, "an 8 x 8 footprint");
};

__device__ __forceinline__ uint32_t um_kmaj(int n, int c) {
  return (uint32_t)((n & 7) * 16 + (n >> 3) * 256 + (c >> 2) * 128 + (c & 3) * 4);
}

// The bounded wait of one thread for an mbarrier phase; false: it gave up.
__device__ __forceinline__ bool um_wait(uint64_t *mbar, uint32_t parity) {
  for (int it = 0; it < UM_SPIN; ++it)
    if (umma::mbar_try_wait_sleep(mbar, parity, UM_SLEEP_NS)) return true;
  return false;
}

__device__ __forceinline__ void um_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(umma::smem_addr(mbar))
               : "memory");
}

// The sub-grid of tile (plane, tu, tv) as planes [pol][row][col] of float2,
// rows RS apart (zeros outside the grid or past g_npol).
template <int W, int RS, int THREADS>
__device__ __forceinline__ void stage_subgrid_planes(const DegridArgs &d, float2 *sub,
                                                     int64_t plane, int tu, int tv,
                                                     int64_t gplane) {
  constexpr int N = 4 * W * W;
  for (int i0 = 0; i0 < N; i0 += THREADS * SUB_UNROLL) {
    float2 v[SUB_UNROLL];
    int dst[SUB_UNROLL];
#pragma unroll
    for (int k = 0; k < SUB_UNROLL; ++k) {
      const int i = i0 + k * THREADS + (int)threadIdx.x;
      v[k] = make_float2(0.f, 0.f);
      const int gp = i / (W * W), rem = i - gp * (W * W);
      const int iu = rem / W, iv = rem - iu * W;
      dst[k] = (gp * W + iu) * RS + iv;
      const int64_t gu = (int64_t)tu * TILE + iu, gv = (int64_t)tv * TILE + iv;
      if (i < N && gp < d.g_npol && gu < d.g_n2 && gv < d.g_n3) {
        const int64_t gi = (plane * d.g_npol + gp) * gplane + gu * d.g_n3 + gv;
        if (d.grid_c128) {
          const double2 x = ((const double2 *)d.grid)[gi];
          v[k] = make_float2((float)x.x, (float)x.y);
        } else {
          v[k] = ((const float2 *)d.grid)[gi];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < SUB_UNROLL; ++k) {
      const int i = i0 + k * THREADS + (int)threadIdx.x;
      if (i < N) sub[dst[k]] = v[k];
    }
  }
}

template <int S>
__global__ void __launch_bounds__(UM_THREADS, 1) k_degrid_umma(TiledDegridArgs a) {
  using M = UMSmem<S>;
  constexpr int W = M::W, RS = M::RS;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  float *tab = (float *)(smem + M::off_tab);
  uint32_t *tabh = (uint32_t *)(smem + M::off_tabh);
  uint32_t *tabl = (uint32_t *)(smem + M::off_tabl);
  float2 *sub = (float2 *)(smem + M::off_sub);
  __shared__ __align__(8) uint64_t s_full[UM_WG][2];
  __shared__ __align__(8) uint64_t s_done[UM_WG][2];
  __shared__ uint32_t s_bits[UM_WIN / 32];
  __shared__ int s_fault[UM_WG];
  __shared__ uint32_t s_taddr;
  __shared__ int s_chunk;
  const DegridArgs &d = a.d;
  const int tid = threadIdx.x, wg = tid >> 7, t = tid & 127, j = t >> 5, lane = tid & 31;
  const int gwarp = tid >> 5;

  // row and column taps over their sums (the products carry 1 / norm), and
  // their TF32 splits
  build_norm_tap_tables<S, 8>(tab, d.cf, a.cgk_len, d.sampling);
  __syncthreads();
  for (int i = tid; i < 256 * 8; i += UM_THREADS) tf32_split(tab[i], tabh[i], tabl[i]);
  if (gwarp == 0) {
    umma::tmem_alloc(&s_taddr, 512);
    umma::tmem_relinquish();
  }
  if (tid < UM_WG) {
    for (int x = 0; x < 2; ++x) {
      umma::mbar_init(&s_full[tid][x], 4);  // one arrival per warp
      umma::mbar_init(&s_done[tid][x], 1);  // the MMA commit
    }
    s_fault[tid] = 0;
  }
  umma::mbar_init_fence();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = s_taddr + (uint32_t)(wg * 128);  // two stages of 64 columns
  unsigned char *ops = smem + M::off_ops + (size_t)wg * 2 * UM_STAGE;
  const uint32_t ops_s = umma::smem_addr(ops);
  // this warp's B rows: output polarisation j from grid polarisation bsrc
  // (-1: zeros); lane (br, bc) takes footprint rows br and br + 4, column bc
  const int br = lane >> 3, bc = lane & 7;
  int bsrc = -1;
  {
    const int v = d.polmap[j];
    if (v >= 0 && v < 4 && v < d.g_npol) bsrc = v;
  }
  const uint32_t aoff = (uint32_t)((t & 7) * 16 + (t >> 3) * 256);
  const int64_t gplane = d.g_n2 * d.g_n3;
  const uint32_t n_rec = *a.n_rec;
  const uint32_t n_all = (uint32_t)a.n_rows;
  const int64_t n_chunks = ((int64_t)n_all + a.chunk - 1) / a.chunk;
  const uint32_t idesc = umma::idesc_tf32(128, 64);
  uint32_t tiles = 0;           // this warpgroup's tiles so far: stage = tiles & 1
  uint32_t fph = 0u, dph = 0u;  // bit s: the parity of stage s's next full / done phase
  int bkey0 = -1, bkey1 = -1;   // the cell whose footprint each stage's B holds
  int stuck = -1;               // the stage whose done phase this thread gave up on
  // the tile whose MMA is in flight: its samples, stage and length
  bool pend = false;
  int pL = 0, ps = 0;
  uint32_t prow = 0u, pmk = 0u;
  int pou = 0;

  // waits for the pending tile's MMA, then each of this warp's samples reads
  // its row of D, weights it with its row taps and writes its 4 values
  auto finish = [&]() {
    if (um_wait(&s_done[wg][ps], (dph >> ps) & 1u)) {
      dph ^= 1u << ps;
    } else {
      stuck = ps;
      s_fault[wg] = 1;
      atomicExch(&g_degrid_fault, 1u);
    }
    umma::fence_after_sync();
    if (32 * j < pL) {
      const float4 c0 = *(const float4 *)(tab + pou * 8);
      const float4 c1 = *(const float4 *)(tab + pou * 8 + 4);
      const float cu[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
      const uint32_t ta = tmem + (uint32_t)(ps * 64) + ((uint32_t)(32 * j) << 16);
      float4 *out = (float4 *)d.values + (int64_t)prow * 2;
      // columns [32 h, 32 h + 32): polarisations 2 h and 2 h + 1
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        uint32_t dr[32];
        umma::ld_32x32b_x32(ta + (uint32_t)(32 * h), dr);
        umma::wait_ld(dr);
        float v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float s = __fmul_rn(cu[0], __uint_as_float(dr[q * 8]));
#pragma unroll
          for (int r = 1; r < S; ++r) s = __fmaf_rn(cu[r], __uint_as_float(dr[q * 8 + r]), s);
          v[q] = s;
        }
        if (t < pL)
          out[h] = pmk ? make_float4(0.f, 0.f, 0.f, 0.f) : make_float4(v[0], v[1], v[2], v[3]);
      }
    }
    umma::fence_before_sync();
    pend = false;
  };

  for (;;) {
    __syncthreads();
    if (tid == 0) s_chunk = (int)atomicAdd(&a.sched[0], 1u);
    __syncthreads();
    const int64_t ch = s_chunk;
    if (ch >= n_chunks) break;
    const uint32_t r0 = (uint32_t)(ch * a.chunk);
    const uint32_t r1 = (uint32_t)min((int64_t)n_all, (int64_t)r0 + a.chunk);
    if (r1 > n_rec) {  // skipped samples (after the usable records) get zeros
      const uint32_t z0 = max(r0, n_rec);
      for (uint32_t rb = z0; rb < r1; rb += UM_THREADS) {
        const uint32_t r = rb + tid;
        if (r >= r1) continue;
        const int64_t row = a.recs[r].row;
        for (int p = 0; p < 4; ++p) put_value(d, 0, row * 4 + p, 0.0, 0.0);
      }
    }
    const uint32_t v1 = min(r1, n_rec);
    if (r0 >= v1) continue;

    int tt = find_tile_warp(a.tile_start, a.n_tiles, r0);
    uint32_t seg_lo = r0;
    while (seg_lo < v1) {
      const uint32_t t_end = a.tile_start[tt + 1];
      const uint32_t seg_hi = min(v1, t_end);
      if (seg_hi <= seg_lo) {
        ++tt;
        continue;
      }
      const int64_t plane = tt / (a.ntu * a.ntv);
      const int64_t trem = tt - plane * a.ntu * a.ntv;
      const int tu = (int)(trem / a.ntv), tv = (int)(trem - (int64_t)tu * a.ntv);
      __syncthreads();  // every warp has built its B rows from the previous sub
      stage_subgrid_planes<W, RS, UM_THREADS>(d, sub, plane, tu, tv, gplane);
      bkey0 = bkey1 = -1;  // a new sub-grid: no footprint is current

      for (uint32_t x0 = seg_lo; x0 < seg_hi; x0 += UM_WIN) {
        const uint32_t x1 = min(seg_hi, x0 + (uint32_t)UM_WIN);
        if (x0 != seg_lo) __syncthreads();  // every warp is done with the last bitmap
        // bit i of the window: a cell starts at record x0 + i (each warp
        // loads 8 words' records before it compares them)
        {
          constexpr int NW = UM_THREADS / 32, BATCH = 8;
          const uint32_t nwords = (x1 - x0 + 31u) >> 5;
          for (uint32_t w0 = (uint32_t)gwarp; w0 < nwords; w0 += NW * BATCH) {
            uint32_t ky[BATCH], pk[BATCH];
#pragma unroll
            for (int b = 0; b < BATCH; ++b) {
              const uint32_t wi = w0 + (uint32_t)(b * NW);
              const uint32_t r = x0 + wi * 32u + (uint32_t)lane;
              ky[b] = r < x1 ? ((const uint2 *)(a.recs + r))->y : 0xFFFFFFFFu;
              pk[b] = (lane == 0 && wi > 0 && wi < nwords) ? ((const uint2 *)(a.recs + r - 1))->y
                                                          : 0xFFFFFFFEu;
            }
#pragma unroll
            for (int b = 0; b < BATCH; ++b) {
              const uint32_t wi = w0 + (uint32_t)(b * NW);
              if (wi >= nwords) break;  // uniform across the warp
              const int key = ky[b] == 0xFFFFFFFFu ? -1 : (int)(ky[b] & 0xFFFFu);
              int prev = __shfl_up_sync(FULL, key, 1);
              if (lane == 0) prev = wi == 0 ? -2 : (int)(pk[b] & 0xFFFFu);
              const uint32_t m = __ballot_sync(FULL, key >= 0 && key != prev);
              if (lane == 0) s_bits[wi] = m;
            }
          }
        }
        __syncthreads();  // the bitmap (and, in the first window, the sub-grid)

        // this warpgroup's slice of the window, in tiles of one cell
        const uint32_t n = x1 - x0;
        const uint32_t w_lo = x0 + (uint32_t)(((uint64_t)n * wg) / UM_WG);
        const uint32_t w_hi = x0 + (uint32_t)(((uint64_t)n * (wg + 1)) / UM_WG);
        // the tile from base: up to 128 records, ending before the next cell
        auto tile_len = [&](uint32_t base) -> int {
          int L = (int)min(128u, w_hi - base);
          uint32_t i = base - x0 + 1u;                    // first bit to look at
          const uint32_t iend = base - x0 + (uint32_t)L;  // one past the last
          while (i < iend) {
            const uint32_t m = s_bits[i >> 5] >> (i & 31u);
            if (m) {
              const uint32_t pos = i + (uint32_t)(__ffs((int)m) - 1);
              if (pos < iend) L = (int)(pos - (base - x0));
              break;
            }
            i = (i | 31u) + 1u;
          }
          return L;
        };
        uint32_t base = w_lo;
        uint2 raw = make_uint2(0u, 0u);
        uint32_t mword = 0u, kraw = 0u;
        if (base < w_hi) {
          const uint32_t r = base + (uint32_t)t;
          if (r < w_hi) {
            raw = *(const uint2 *)(a.recs + r);
            mword = __ldg(a.exc_mark + (r >> 5));
          }
          kraw = ((const uint2 *)(a.recs + base))->y;
        }
        int L = base < w_hi ? tile_len(base) : 0;
        while (base < w_hi) {
          if (*(volatile int *)&s_fault[wg]) break;
          const uint32_t r = base + (uint32_t)t;
          const uint32_t row = raw.x;
          const int ou = (int)((raw.y >> 16) & 0xFFu), ov = (int)(raw.y >> 24);
          const uint32_t mk = (mword >> (r & 31u)) & 1u;
          const int kx = (int)(kraw & 0xFFFFu);
          // the next tile and its records
          const uint32_t nbase = base + (uint32_t)L;
          int nL = 0;
          if (nbase < w_hi) {
            const uint32_t rn = nbase + (uint32_t)t;
            if (rn < w_hi) {
              raw = *(const uint2 *)(a.recs + rn);
              mword = __ldg(a.exc_mark + (rn >> 5));
            }
            kraw = ((const uint2 *)(a.recs + nbase))->y;
            nL = tile_len(nbase);
          }
          const int s = (int)(tiles & 1u);
          unsigned char *st = ops + s * UM_STAGE;
          // A: this sample's column taps (row t), high parts and remainders
          if (t < L) {
            const uint4 *th = (const uint4 *)(tabh + ov * 8);
            const uint4 *tl = (const uint4 *)(tabl + ov * 8);
            *(uint4 *)(st + aoff) = th[0];
            *(uint4 *)(st + aoff + 128) = th[1];
            *(uint4 *)(st + 4096 + aoff) = tl[0];
            *(uint4 *)(st + 4096 + aoff + 128) = tl[1];
          }
          // B: output polarisation j's rows of the cell's footprint, split
          // (kept from two tiles back when the cell is the same)
          if ((s ? bkey1 : bkey0) != kx) {
            if (s)
              bkey1 = kx;
            else
              bkey0 = kx;
            const int du = kx & 255, dv = kx >> 8;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int rr = br + 4 * h;
              float2 v = make_float2(0.f, 0.f);
              if (bsrc >= 0 && rr < S && bc < S) v = sub[(bsrc * W + du + rr) * RS + dv + bc];
              uint32_t rh, rl, ih, il;
              tf32_split(v.x, rh, rl);
              tf32_split(v.y, ih, il);
              const uint32_t o_re = 8192 + um_kmaj(16 * j + rr, bc);
              *(uint32_t *)(st + o_re) = rh;
              *(uint32_t *)(st + 2048 + o_re) = rl;
              *(uint32_t *)(st + o_re + 256) = ih;  // row + 8: the next 8-row group
              *(uint32_t *)(st + 2048 + o_re + 256) = il;
            }
          }
          // this warp's operands are written: tell the MMA thread
          umma::fence_proxy_async();
          umma::fence_before_sync();
          __syncwarp();
          if (lane == 0) um_arrive(&s_full[wg][s]);
          if (t == 0) {
            if (um_wait(&s_full[wg][s], (fph >> s) & 1u)) {
              fph ^= 1u << s;
              umma::fence_after_sync();
              const uint32_t sa = ops_s + (uint32_t)(s * UM_STAGE);
              const uint64_t ah = umma::desc_kmajor(sa, 128, 256);
              const uint64_t al = umma::desc_kmajor(sa + 4096, 128, 256);
              const uint64_t bh = umma::desc_kmajor(sa + 8192, 128, 256);
              const uint64_t bl = umma::desc_kmajor(sa + 10240, 128, 256);
              const uint32_t td = tmem + (uint32_t)(s * 64);
              umma::mma_tf32(td, al, bh, idesc, false);
              umma::mma_tf32(td, ah, bl, idesc, true);
              umma::mma_tf32(td, ah, bh, idesc, true);
              umma::commit(&s_done[wg][s]);
            } else {
              s_fault[wg] = 1;
              atomicExch(&g_degrid_fault, 1u);
            }
          }
          __syncwarp();
          // the previous tile, while this one's MMA runs
          if (pend) finish();
          pend = true;
          pL = L;
          ps = s;
          prow = row;
          pmk = mk;
          pou = ou;
          ++tiles;
          base = nbase;
          L = nL;
        }
      }
      seg_lo = seg_hi;
      if (seg_hi == t_end) ++tt;
    }
  }
  // the last tile; after a wait that gave up, one more bounded wait for each
  // commit still outstanding before the columns are freed
  const bool faulted = *(volatile int *)&s_fault[wg] != 0;
  if (pend && !faulted) finish();
  if (faulted && lane == 0) {
    if (stuck >= 0) um_wait(&s_done[wg][stuck], (dph >> stuck) & 1u);
    if (pend) um_wait(&s_done[wg][ps], (dph >> ps) & 1u);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (gwarp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(s_taddr, 512);
  }
  // every CTA has taken its last chunk: the last one to get here re-arms
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&a.sched[1], 1u) == gridDim.x - 1) {
      a.sched[0] = 0u;
      a.sched[1] = 0u;
      __threadfence();
    }
  }
}

// ------------------------------------------------- shared-plan exceptions --
// The samples a shared plan lists for the degridder (plan.cuh): each in the
// degridder's own convention (sample_pos_degrid, standard_degrid.py:435-462)
// and in FP64, the reference's tap and summation order, one thread per
// sample, all visibility polarisations.  Runs after the tiled kernel, which
// left zeros there in store mode.  Reads the plan's copies of u, v, the
// frequencies, the channel map and the degridder's scale / offset.
struct ExcArgs {
  const uint32_t *count, *rows;
  const double2 *uv;
  const double *freq;
  const int32_t *chan_map;
  const double *dpar;
  PlanGeom g;  // the degridder's geometry (scale / offset come from dpar)
  DegridArgs d;
  int accumulate;
};

__global__ void __launch_bounds__(128) k_degrid_exceptions(ExcArgs e) {
  const uint32_t n = *e.count;
  if (n == 0u) return;
  const DegridArgs &d = e.d;
  PlanGeom g = e.g;
  g.scale0 = e.dpar[0];
  g.scale1 = e.dpar[1];
  g.offset0 = e.dpar[2];
  g.offset1 = e.dpar[3];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t row = e.rows[i];
    const int64_t tb = row / d.nvchan;
    const int ichan = (int)(row - tb * d.nvchan);
    const int achan = e.chan_map[ichan];
    const double f = e.freq[ichan];
    const double2 uv = e.uv[tb];
    int fu, fv, o0, o1;
    if (achan < 0 || achan >= d.g_nchan || !sample_pos_degrid(uv.x, uv.y, f, g, fu, fv, o0, o1))
      continue;  // not listed by the plan; kept for safety
    const long long beg = -(d.support / 2), end = beg + d.support;
    const long long x0 = (long long)fu - beg, y0 = (long long)fv - beg;
    double norm = 0.0;
    for (long long ix = beg; ix < end; ++ix) {
      const long long i1 = (long long)d.sampling * ix + o0;
      const double wtx = d.cf[i1 < 0 ? -i1 : i1];
      for (long long iy = beg; iy < end; ++iy) {
        const long long i2 = (long long)d.sampling * iy + o1;
        norm = __dadd_rn(norm, __dmul_rn(wtx, d.cf[i2 < 0 ? -i2 : i2]));
      }
    }
    double ph_re = 1.0, ph_im = 0.0;
    if (d.dphase) {
      const double phase =
          __ddiv_rn(__dmul_rn(__dmul_rn(-2.0 * 3.141592653589793, d.dphase[tb]), f), d.c);
      sincos(phase, &ph_im, &ph_re);
    }
    for (int p = 0; p < d.nvpol; ++p) {
      const int64_t k = (int64_t)row * d.nvpol + p;
      const int apol = d.polmap[p];
      if (apol < 0 || apol >= d.g_npol || (d.flag && d.flag[k]) || norm == 0.0) {
        if (!e.accumulate) put_value(d, 0, k, 0.0, 0.0);
        continue;
      }
      const int64_t plane = ((int64_t)achan * d.g_npol + apol) * d.g_n2 * d.g_n3;
      double nv_re = 0.0, nv_im = 0.0;
      for (long long ix = beg; ix < end; ++ix) {
        const long long i1 = (long long)d.sampling * ix + o0;
        const double wtx = d.cf[i1 < 0 ? -i1 : i1];
        for (long long iy = beg; iy < end; ++iy) {
          const long long i2 = (long long)d.sampling * iy + o1;
          const double wt = __dmul_rn(wtx, d.cf[i2 < 0 ? -i2 : i2]);
          const int64_t gi = plane + (x0 + ix) * d.g_n3 + (y0 + iy);
          double gr, gim;
          if (d.grid_c128) {
            const double2 gv = ((const double2 *)d.grid)[gi];
            gr = gv.x;
            gim = gv.y;
          } else {
            const float2 gv = ((const float2 *)d.grid)[gi];
            gr = gv.x;
            gim = gv.y;
          }
          nv_re = __dadd_rn(nv_re, __dmul_rn(wt, gr));
          nv_im = __dadd_rn(nv_im, __dmul_rn(wt, gim));
        }
      }
      const double cr = ph_re, ci = -ph_im;
      const double pr = __dsub_rn(__dmul_rn(nv_re, cr), __dmul_rn(nv_im, ci));
      const double pi = __dadd_rn(__dmul_rn(nv_re, ci), __dmul_rn(nv_im, cr));
      put_value(d, e.accumulate, k, __ddiv_rn(pr, norm), __ddiv_rn(pi, norm));
    }
  }
}

template <int S>
static int launch_degrid_tc(const TiledDegridArgs &a, int64_t nblocks, cudaStream_t st) {
  size_t smem = TCSmem<S>::total;
  static int resident[64] = {0};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("av_degrid_tiled: device %d beyond the 64 this library tracks", dev);
    return AV_ERR_UNSUPPORTED;
  }
  if (resident[dev] == 0) {
    if (smem > 48 * 1024)
      AV_CUDA(cudaFuncSetAttribute(k_degrid_tc<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    int per_sm = 0;
    AV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_degrid_tc<S>, TC_THREADS,
                                                          smem));
    resident[dev] = (per_sm > 0 ? per_sm : 1) * sm_count();
  }
  if (nblocks > resident[dev]) nblocks = resident[dev];
  k_degrid_tc<S><<<(unsigned)nblocks, TC_THREADS, smem, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

template <int S>
static int launch_degrid_umma(const TiledDegridArgs &a, int64_t nblocks, cudaStream_t st) {
  const size_t smem = UMSmem<S>::total;
  static bool attr[64] = {false};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("av_degrid_tiled: device %d beyond the 64 this library tracks", dev);
    return AV_ERR_UNSUPPORTED;
  }
  if (!attr[dev]) {
    AV_CUDA(cudaFuncSetAttribute(k_degrid_umma<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    attr[dev] = true;
  }
  // one CTA per SM (its shared memory rules out a second, and it holds all
  // 512 tensor-memory columns)
  const int64_t sms = sm_count();
  if (nblocks > sms) nblocks = sms;
  k_degrid_umma<S><<<(unsigned)nblocks, UM_THREADS, smem, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

template <int S, int NPG>
static int launch_degrid_tiled(const TiledDegridArgs &a, int64_t nblocks, cudaStream_t st) {
  // persistent CTAs: at most as many as are resident at once
  size_t smem = DSmem<S, NPG>::total;
  static int resident[64] = {0};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("av_degrid_tiled: device %d beyond the 64 this library tracks", dev);
    return AV_ERR_UNSUPPORTED;
  }
  if (resident[dev] == 0) {
    if (smem > 48 * 1024)
      AV_CUDA(cudaFuncSetAttribute(k_degrid_tiled<S, NPG>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    AV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_degrid_tiled<S, NPG>,
                                                          DT_THREADS, smem));
    resident[dev] = (per_sm > 0 ? per_sm : 1) * sm_count();
  }
  if (nblocks > resident[dev]) nblocks = resident[dev];
  k_degrid_tiled<S, NPG><<<(unsigned)nblocks, DT_THREADS, smem, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// The TF32 tensor-core kernel for the fast store path with 4 grid
// polarisations as AV_TUNE_DEGRID_LANES says (automatically for every support
// it covers, 3-8, where it is the faster), the FP32 kernel otherwise.
template <int S>
static int degrid_dispatch_npg(const TiledDegridArgs &a, int npg, int64_t nb, cudaStream_t st) {
  if (npg == 1) return launch_degrid_tiled<S, 1>(a, nb, st);
  if (npg == 2) return launch_degrid_tiled<S, 2>(a, nb, st);
  if constexpr (S <= 8) {
    const int64_t lanes = tune_value(AV_TUNE_DEGRID_LANES);
    if (a.fast_out && a.d.g_npol == 4 && lanes == AV_DEGRID_LANES_TC05)
      return launch_degrid_umma<S>(a, nb, st);
    const bool tf32 = lanes == AV_DEGRID_LANES_TF32 || lanes == AV_DEGRID_LANES_AUTO;
    // the TF32 kernel keeps a shared plan's marks in the staged rows' top bit
    if (a.fast_out && a.d.g_npol == 4 && tf32 && a.n_rows < (int64_t)REC_DEGRID_EXC)
      return launch_degrid_tc<S>(a, nb, st);
  }
  return launch_degrid_tiled<S, 4>(a, nb, st);
}

static int degrid_dispatch(const TiledDegridArgs &a, int support, int npg, int64_t nb,
                           cudaStream_t st) {
  switch (support) {
    case 3: return degrid_dispatch_npg<3>(a, npg, nb, st);
    case 4: return degrid_dispatch_npg<4>(a, npg, nb, st);
    case 5: return degrid_dispatch_npg<5>(a, npg, nb, st);
    case 6: return degrid_dispatch_npg<6>(a, npg, nb, st);
    case 7: return degrid_dispatch_npg<7>(a, npg, nb, st);
    case 8: return degrid_dispatch_npg<8>(a, npg, nb, st);
    case 9: return degrid_dispatch_npg<9>(a, npg, nb, st);
  }
  set_error("av_degrid_tiled: support %d not in [3, 9]", support);
  return AV_ERR_UNSUPPORTED;
}

static int fill_degrid_args(DegridArgs &a, const double *uvw, const double *dphase, void *values,
                            int values_dtype, const uint8_t *flag, double scale_x, double scale_y,
                            double offset_x, double offset_y, const void *grid, int grid_dtype,
                            int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                            const double *freq, double c, int support, int sampling,
                            const double *convFunc, const int32_t *chanmap,
                            const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                            int64_t nvpol, const char *who) {
  AV_CHECK_ARG(uvw && values && grid && freq && convFunc && chanmap && polmap,
               "%s: null pointer", who);
  AV_CHECK_ARG(values_dtype == AV_C64 || values_dtype == AV_C128, "%s: values dtype", who);
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128, "%s: grid dtype", who);
  AV_CHECK_ARG(support >= 1 && sampling >= 1, "%s: bad kernel sizes", who);
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nvchan >= 0 && nvpol >= 0 && g_nchan >= 0 && g_npol >= 0 &&
                   g_n2 >= 0 && g_n3 >= 0, "%s: bad shape", who);
  a.scale0 = scale_x; a.scale1 = scale_y; a.offset0 = offset_x; a.offset1 = offset_y;
  a.uvw = uvw; a.dphase = dphase; a.values = values; a.values_c128 = values_dtype == AV_C128;
  a.flag = flag;
  a.grid = grid; a.grid_c128 = grid_dtype == AV_C128;
  a.g_nchan = g_nchan; a.g_npol = g_npol; a.g_n2 = g_n2; a.g_n3 = g_n3;
  a.freq = freq; a.c = c; a.support = support; a.sampling = sampling; a.cf = convFunc;
  a.chanmap = chanmap; a.polmap = polmap; a.nt = nt; a.nb = nb; a.nvchan = nvchan; a.nvpol = nvpol;
  return AV_OK;
}

}  // namespace av

using namespace av;

extern "C" {

int av_degrid_plain(const double *uvw, const double *dphase, void *values, int values_dtype,
                    const uint8_t *flag, double scale_x, double scale_y, double offset_x, double offset_y,
                    const void *grid, int grid_dtype, int64_t g_nchan, int64_t g_npol,
                    int64_t g_n2, int64_t g_n3, const double *freq, double c, int support,
                    int sampling, const double *convFunc, const int32_t *chanmap,
                    const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                    int64_t nvpol, void *stream) {
  clear_error();
  DegridArgs a;
  int rc = fill_degrid_args(a, uvw, dphase, values, values_dtype, flag, scale_x, scale_y, offset_x, offset_y, grid,
                            grid_dtype, g_nchan, g_npol, g_n2, g_n3, freq, c, support, sampling,
                            convFunc, chanmap, polmap, nt, nb, nvchan, nvpol, "av_degrid_plain");
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  int64_t total = nt * nb * nvchan * nvpol;
  if (total == 0) return AV_OK;
  k_degrid_plain<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_degrid_plain_adjoint(const double *uvw, const double *dphase, const void *values,
                            int values_dtype, const uint8_t *flag, double scale_x, double scale_y,
                            double offset_x, double offset_y, void *grid, int grid_dtype,
                            int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                            const double *freq, double c, int support, int sampling,
                            const double *convFunc, const int32_t *chanmap,
                            const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                            int64_t nvpol, void *stream) {
  clear_error();
  DegridArgs a;
  int rc = fill_degrid_args(a, uvw, dphase, (void *)values, values_dtype, flag, scale_x, scale_y,
                            offset_x, offset_y, grid, grid_dtype, g_nchan, g_npol, g_n2, g_n3,
                            freq, c, support, sampling, convFunc, chanmap, polmap, nt, nb, nvchan,
                            nvpol, "av_degrid_plain_adjoint");
  if (rc) return rc;
  int64_t total = nt * nb * nvchan * nvpol;
  if (total == 0) return AV_OK;
  k_degrid_adjoint_plain<<<(unsigned)((total + 255) / 256), 256, 0, as_stream(stream)>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_degrid_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nvchan, int64_t g_n2,
                                      int64_t g_n3, int64_t g_nchan, int support) {
  PlanGeom g;
  plan_geometry(g, nt, nb, nvchan, g_nchan, g_n2, g_n3, support, 100);
  return plan_workspace_bytes(g);
}

static int degrid_geom_checked(PlanGeom &g, Plan &p, double scale_x, double scale_y,
                               double offset_x, double offset_y, int64_t g_nchan, int64_t g_n2,
                               int64_t g_n3, int support, int sampling, int64_t nt, int64_t nb,
                               int64_t nvchan, void *workspace, size_t workspace_bytes,
                               const char *who) {
  AV_CHECK_ARG(support >= 3 && support <= 9, "%s: support must be in [3, 9]", who);
  AV_CHECK_ARG(sampling >= 1 && sampling <= 254, "%s: sampling must be in [1, 254]", who);
  AV_CHECK_ARG(g_n2 >= support && g_n3 >= support && g_n2 < 131072 && g_n3 < 131072,
               "%s: grid size out of range", who);
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nvchan >= 0 && g_nchan >= 0, "%s: bad shape", who);
  AV_CHECK_ARG(workspace && (((uintptr_t)workspace) & 255) == 0,
               "%s: workspace must be 256-byte aligned", who);
  plan_geometry(g, nt, nb, nvchan, g_nchan > 0 ? g_nchan : 1, g_n2, g_n3, support, sampling);
  g.convention = 1;
  g.chk_x = g_n3;
  g.chk_y = g_n2;
  g.scale0 = scale_x;
  g.scale1 = scale_y;
  g.offset0 = offset_x;
  g.offset1 = offset_y;
  size_t need = plan_workspace_bytes(g);
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

int av_degrid_tiled_plan(const double *uvw, const double *freq, const int32_t *chanmap,
                         double scale_x, double scale_y, double offset_x, double offset_y,
                         int64_t g_nchan, int64_t g_n2, int64_t g_n3, int support, int sampling,
                         int64_t nt, int64_t nb, int64_t nvchan, void *workspace,
                         size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(uvw && freq && chanmap, "av_degrid_tiled_plan: null pointer");
  PlanGeom g;
  Plan p;
  int rc = degrid_geom_checked(g, p, scale_x, scale_y, offset_x, offset_y, g_nchan, g_n2, g_n3,
                               support, sampling, nt, nb, nvchan, workspace, workspace_bytes,
                               "av_degrid_tiled_plan");
  if (rc) return rc;
  return plan_build(g, p, uvw, freq, chanmap, 0.0, 0.0, as_stream(stream));
}

int av_degrid_tiled_execute(const double *dphase, void *values, int values_dtype,
                            int accumulate, const uint8_t *flag, const void *grid, int grid_dtype,
                            int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                            const double *freq, int support, int sampling,
                            const double *convFunc, const int32_t *polmap, int64_t nt,
                            int64_t nb, int64_t nvchan, int64_t nvpol, void *workspace,
                            size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(values && grid && freq && convFunc && polmap,
               "av_degrid_tiled_execute: null pointer");
  AV_CHECK_ARG(values_dtype == AV_C64 || values_dtype == AV_C128,
               "av_degrid_tiled_execute: values dtype");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_degrid_tiled_execute: grid dtype");
  AV_CHECK_ARG(g_npol >= 1 && g_npol <= 4, "av_degrid_tiled_execute: grid pols must be in [1, 4]");
  AV_CHECK_ARG(nvpol >= 0, "av_degrid_tiled_execute: bad shape");
  PlanGeom g;
  Plan p;
  int rc = degrid_geom_checked(g, p, 0.0, 0.0, 0.0, 0.0, g_nchan, g_n2, g_n3, support, sampling,
                               nt, nb, nvchan, workspace, workspace_bytes,
                               "av_degrid_tiled_execute");
  if (rc) return rc;
  AV_CHECK_ARG(nvpol <= 8, "av_degrid_tiled_execute: at most 8 visibility polarisations");
  int64_t rows = nt * nb * nvchan;
  if (rows == 0 || nvpol == 0) return AV_OK;
  DegridArgs d;
  d.uvw = nullptr;
  d.dphase = dphase;
  d.values = values;
  d.values_c128 = values_dtype == AV_C128;
  d.flag = flag;
  d.scale0 = d.scale1 = d.offset0 = d.offset1 = 0.0;
  d.grid = grid;
  d.grid_c128 = grid_dtype == AV_C128;
  d.g_nchan = g_nchan; d.g_npol = g_npol; d.g_n2 = g_n2; d.g_n3 = g_n3;
  d.freq = freq; d.c = C_LIGHT; d.support = support; d.sampling = sampling; d.cf = convFunc;
  d.chanmap = nullptr; d.polmap = polmap; d.nt = nt; d.nb = nb; d.nvchan = nvchan;
  d.nvpol = nvpol;
  TiledDegridArgs a;
  a.recs = p.recs;
  a.tile_start = p.tile_start;
  a.n_rec = p.offs + g.n_keys();
  a.exc_mark = p.exc_mark;
  a.n_tiles = g.n_tiles();
  a.ntu = g.ntu;
  a.ntv = g.ntv;
  int sms = sm_count();
  const int64_t per_sm = tune_value(AV_TUNE_DEGRID_CHUNKS_PER_SM);
  int64_t chunk = (rows + (int64_t)sms * per_sm - 1) / ((int64_t)sms * per_sm);
  if (chunk < 1024) chunk = 1024;
  a.chunk = chunk;
  a.d = d;
  a.cgk_len = sampling * (support / 2 + 1);
  a.sched = p.counters + 2;
  a.accumulate = accumulate ? 1 : 0;
  a.n_rows = rows;
  a.fast_out = (!accumulate && values_dtype == AV_C64 && nvpol == 4 && flag == nullptr &&
                dphase == nullptr && (((uintptr_t)values) & 31) == 0) ? 1 : 0;
  int npg = g_npol <= 1 ? 1 : (g_npol <= 2 ? 2 : 4);
  rc = degrid_dispatch(a, support, npg, (rows + chunk - 1) / chunk, as_stream(stream));
  if (rc) return rc;
  // a shared plan's exceptions (none listed in a degridder plan: the kernel
  // reads a zero count and returns)
  ExcArgs e;
  e.count = p.exc_count;
  e.rows = p.exc_rows;
  e.uv = p.uv;
  e.freq = p.freq;
  e.chan_map = p.chan_map;
  e.dpar = p.dpar;
  e.g = g;
  e.g.scale0 = e.g.scale1 = e.g.offset0 = e.g.offset1 = 0.0;
  e.d = d;
  e.d.cf = convFunc;
  e.accumulate = a.accumulate;
  k_degrid_exceptions<<<(unsigned)sms, 128, 0, as_stream(stream)>>>(e);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

int av_degrid_fault_read(int *out, int clear, void *stream) {
  clear_error();
  AV_CHECK_ARG(out, "av_degrid_fault_read: null pointer");
  cudaStream_t st = as_stream(stream);
  uint32_t v = 0u;
  AV_CUDA(cudaMemcpyFromSymbolAsync(&v, g_degrid_fault, sizeof(v), 0, cudaMemcpyDeviceToHost, st));
  AV_CUDA(cudaStreamSynchronize(st));
  *out = (int)v;
  if (clear && v) {
    const uint32_t z = 0u;
    AV_CUDA(cudaMemcpyToSymbolAsync(g_degrid_fault, &z, sizeof(z), 0, cudaMemcpyHostToDevice, st));
    AV_CUDA(cudaStreamSynchronize(st));
  }
  return AV_OK;
}

int av_degrid_tiled(const double *uvw, const double *dphase, void *values, int values_dtype,
                    int accumulate, const uint8_t *flag, double scale_x, double scale_y, double offset_x, double offset_y,
                    const void *grid, int grid_dtype, int64_t g_nchan, int64_t g_npol,
                    int64_t g_n2, int64_t g_n3, const double *freq, double c, int support,
                    int sampling, const double *convFunc, const int32_t *chanmap,
                    const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                    int64_t nvpol, void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(c == C_LIGHT, "av_degrid_tiled: c must be 299792458.0 (use av_degrid_plain)");
  int rc = av_degrid_tiled_plan(uvw, freq, chanmap, scale_x, scale_y, offset_x, offset_y, g_nchan,
                                g_n2, g_n3, support, sampling, nt, nb, nvchan, workspace,
                                workspace_bytes, stream);
  if (rc) return rc;
  return av_degrid_tiled_execute(dphase, values, values_dtype, accumulate, flag, grid, grid_dtype,
                                 g_nchan,
                                 g_npol, g_n2, g_n3, freq, support, sampling, convFunc, polmap, nt,
                                 nb, nvchan, nvpol, workspace, workspace_bytes, stream);
}

}  // extern "C"
