// Convolutional gridding (standard_grid_jit, standard_grid.py:246-432).
//
// av_grid_plain: one thread per (time, baseline, channel) sample, FP64, the
//   reference's per-sample arithmetic and tap order, FP64 atomics.
// av_grid_tiled: tiled gridder over a cell-sorted plan (plan.cuh) for FP32
//   visibilities and weights, accumulating in FP64.  Persistent CTAs (one
//   per SM) take chunks of records; per tile segment a CTA keeps a
//   (T+S-1)^2 x npg FP64 complex sub-grid in shared memory.  Each warp
//   streams a slice of the segment and keeps its accumulators in registers
//   while the samples stay in one cell, flushing to the sub-grid only on a
//   cell change: for supports up to 8 as FP64 tensor-core tiles
//   (mma.sync.m16n8k4.f64, four samples per step), otherwise with each
//   lane owning a footprint row x polarisation x column range (DFMA).  The
//   sub-grid goes to the global grid once per segment.
#include <type_traits>

#include "plan.cuh"

namespace av {

// ---------------------------------------------------------------------------
// plain kernel
// ---------------------------------------------------------------------------
struct GridArgs {
  void *grid;
  int grid_dtype;
  double *sumw;
  int do_psf, do_iw;
  const void *vis;
  int vis_dtype;
  const void *wt;
  int wt_dtype;
  const double *uvw, *freq;
  const int32_t *chan_map, *pol_map;
  const double *cgk;
  int64_t n_u, n_v;
  double dl0, dl1;
  int support, os;
  int64_t nt, nb, nchan, npol, n_img_chan, n_img_pol;
};

__device__ __forceinline__ double load_real(const void *p, int dt, int64_t i) {
  return dt == AV_F32 ? (double)((const float *)p)[i] : ((const double *)p)[i];
}
__device__ __forceinline__ double2 load_cplx(const void *p, int dt, int64_t i) {
  if (dt == AV_C64) {
    float2 v = ((const float2 *)p)[i];
    return make_double2(v.x, v.y);
  }
  return ((const double2 *)p)[i];
}
__device__ __forceinline__ void grid_add(void *g, int dt, int64_t i, double re, double im) {
  switch (dt) {
    case AV_C128:
      atomicAdd(&((double2 *)g)[i].x, re);
      atomicAdd(&((double2 *)g)[i].y, im);
      break;
    case AV_C64:
      atomicAdd(&((float2 *)g)[i].x, (float)re);
      atomicAdd(&((float2 *)g)[i].y, (float)im);
      break;
    case AV_F64: atomicAdd(&((double *)g)[i], re); break;
    default: atomicAdd(&((float *)g)[i], (float)re); break;
  }
}

__global__ void __launch_bounds__(256) k_grid_plain(GridArgs a) {
  int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= a.nt * a.nb * a.nchan) return;
  int64_t tb = row / a.nchan;
  int c = (int)(row - tb * a.nchan);
  int a_chan = a.chan_map[c];
  if (a_chan < 0 || a_chan >= a.n_img_chan) return;  // outside the image: dropped
  double f = a.freq[c];
  double us0 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, a.dl0), (double)a.n_u), C_LIGHT);
  double us1 = __ddiv_rn(-__dmul_rn(__dmul_rn(f, a.dl1), (double)a.n_v), C_LIGHT);
  double u = __dmul_rn(a.uvw[3 * tb + 0], us0), v = __dmul_rn(a.uvw[3 * tb + 1], us1);
  if (isnan(u) || isnan(v)) return;
  double u_pos = __dadd_rn(u, (double)(a.n_u / 2)), v_pos = __dadd_rn(v, (double)(a.n_v / 2));
  double u_pos_c = __dadd_rn(-u, (double)(a.n_u / 2)), v_pos_c = __dadd_rn(-v, (double)(a.n_v / 2));
  long long ui = trunc_ll(__dadd_rn(u_pos, 0.5)), vi = trunc_ll(__dadd_rn(v_pos, 0.5));
  long long uic = trunc_ll(__dadd_rn(u_pos_c, 0.5)), vic = trunc_ll(__dadd_rn(v_pos_c, 0.5));
  const long long sc = a.support / 2;
  if (!((ui + sc < a.n_u) && (vi + sc < a.n_v) && (ui - sc >= 0) && (vi - sc >= 0))) return;
  long long uoi = (long long)floor(__dadd_rn(__dmul_rn(__dsub_rn((double)ui, u_pos), (double)a.os), 0.5));
  long long voi = (long long)floor(__dadd_rn(__dmul_rn(__dsub_rn((double)vi, v_pos), (double)a.os), 0.5));
  const long long s0 = -sc, s1 = a.support - sc;
  const bool is_cplx = (a.grid_dtype == AV_C64 || a.grid_dtype == AV_C128);
  for (int64_t ip = 0; ip < a.npol; ++ip) {
    int64_t idx = row * a.npol + ip;
    double sel_w, wr, wi;
    if (a.do_psf) {
      if (a.npol >= 2 && a.do_iw) {
        wr = __ddiv_rn(__dadd_rn(load_real(a.wt, a.wt_dtype, row * a.npol),
                                 load_real(a.wt, a.wt_dtype, row * a.npol + 1)), 2.0);
        wi = 0.0;
        sel_w = wr;
      } else {
        sel_w = load_real(a.wt, a.wt_dtype, idx);
        wr = sel_w;
        wi = 0.0;
      }
    } else {
      sel_w = load_real(a.wt, a.wt_dtype, idx);
      double2 vv = load_cplx(a.vis, a.vis_dtype, idx);
      wr = __dmul_rn(vv.x, sel_w);
      wi = __dmul_rn(vv.y, sel_w);
    }
    if (isnan(wr) || isnan(wi)) continue;
    if (!(wr != 0.0 || wi != 0.0)) continue;
    int a_pol = a.pol_map[ip];
    if (a_pol < 0 || a_pol >= a.n_img_pol) continue;
    int64_t plane = ((int64_t)a_chan * a.n_img_pol + a_pol) * a.n_u * a.n_v;
    double norm = 0.0;
    for (long long iv = s0; iv < s1; ++iv) {
      long long vo = (long long)a.os * iv + voi;
      double conv_v = a.cgk[vo < 0 ? -vo : vo];
      long long v_indx = vi + iv, v_indx_c = vic + iv;
      for (long long iu = s0; iu < s1; ++iu) {
        long long uo = (long long)a.os * iu + uoi;
        double conv_u = a.cgk[uo < 0 ? -uo : uo];
        double conv = __dmul_rn(conv_u, conv_v);
        long long u_indx = ui + iu;
        grid_add(a.grid, a.grid_dtype, plane + u_indx * a.n_v + v_indx, __dmul_rn(conv, wr),
                 is_cplx ? __dmul_rn(conv, wi) : 0.0);
        norm = __dadd_rn(norm, conv);
        if (a.do_iw) {
          // standard_grid.py:407-421 indexes the conjugate cell without a
          // bounds check: Numba wraps negative indices per axis and lets an
          // index of n run into the next row / plane.  The same flat cell is
          // used here while it lies inside the array; beyond the array the
          // reference writes out of bounds and the sample is skipped.
          long long uc = uic + iu, vc = v_indx_c;
          if (uc < 0) uc += a.n_u;
          if (vc < 0) vc += a.n_v;
          long long flat = plane + uc * a.n_v + vc;
          long long total = a.n_img_chan * a.n_img_pol * a.n_u * a.n_v;
          if (uc >= 0 && vc >= 0 && flat < total)
            grid_add(a.grid, a.grid_dtype, flat, __dmul_rn(conv, wr),
                     is_cplx ? __dmul_rn(conv, wi) : 0.0);
        }
      }
    }
    double add = __dmul_rn(sel_w, norm);
    atomicAdd(&a.sumw[(int64_t)a_chan * a.n_img_pol + a_pol], add);
    if (a.do_iw) atomicAdd(&a.sumw[(int64_t)a_chan * a.n_img_pol + a_pol], add);
  }
}

// ---------------------------------------------------------------------------
// tiled kernel: FP32 data, FP64 accumulation
// ---------------------------------------------------------------------------
// Grid correction divides the image by the taper grdsf(x) grdsf(y), which is
// ~4e-3 at the edges, so white errors in the uv plane are amplified ~500x in
// the image (norm-wise).  Accumulating in FP32 (even in short runs) leaves
// 3e-5 .. 2e-4 relative error in the dirty image; FP32 products summed in
// FP64 leave ~4e-6.  The kernel therefore reads FP32 visibilities and
// weights, forms tap weights from an FP64 table, and accumulates with DFMA
// into FP64 registers and an FP64 shared-memory sub-grid.
constexpr int GT_STAGE = 32;  // samples a warp stages per round (one per lane)

struct TiledGridArgs {
  const Rec *recs;
  const uint32_t *tile_start;
  const uint32_t *n_rec;  // device: total records (offs[n_keys])
  uint32_t *sched;        // device: [0] next chunk, [1] CTAs done (both 0 between launches)
  int a16;                 // vis and weight rows are 16-byte aligned (16-byte loads / copies)
  int64_t n_tiles, ntu, ntv;
  int64_t chunk;
  const float2 *vis;
  const float *wt;
  int do_psf;
  const double *cgk;
  int cgk_len, os;
  const int32_t *pol_map;  // device, npol entries
  int npol, npg;
  void *grid;
  int grid_c128;
  double *sumw;             // may be NULL (no sum of weights)
  int64_t n_u, n_v;
  // adjoint of the degridder: weight 1 / sum_k w_k per sample, flags honoured
  int inv_norm;
  const uint8_t *flag;      // may be NULL
  // deterministic mode (k_grid_mma<.., true>): fixed-point sums, scales 2^F
  // of the grid and of the sums of weights in det_scale[0..1]
  unsigned long long *det_grid;  // (plane, npg, n_u, n_v, re | im)
  unsigned long long *det_sumw;  // (plane, npg)
  const double *det_scale;
};

// Lane mappings.  Each warp streams its own contiguous slice of a tile
// segment's cell-sorted samples, a whole run of samples in one cell (median
// ~70 on the 33M workload) at a time, so a change of cell (and the flush of
// the accumulators it triggers) is the same for every lane of the warp.  The
// accumulators stay in registers for the run and go to the shared sub-grid
// only on a cell change.  Two mappings of the run's footprint sums onto the
// lanes:
//
// RowLanes (supports 3-9).  A lane owns footprint row g, polarisations
// [pg*PPL, pg*PPL+PPL) and footprint columns [cc*KC, cc*KC+KC) and keeps
// PPL x KC FP64 complex accumulators.  Per sample and lane: 2 PPL DMUL (row
// tap x value) and 2 PPL KC DFMA.  For supports up to 8 each quarter-warp is
// one (polarisation group, column chunk) block and its lanes are the rows
// (lane = block * 8 + g): every quarter then reads one address for the
// staged value and for the column taps, which shared memory serves at its
// broadcast rate.  Support 7 with 4 polarisations: 4 quarters x 7 rows, 7
// accumulators per lane.
//
// MmaLanes (supports 3-8).  A run's footprint sums are a matrix product,
//   acc[p](ri, r, c) += sum over samples k of (ri(v_k[p]) cu_k[r]) cv_k[c],
// with ri the real or imaginary part, cu / cv the row / column taps.  Per
// group of four samples of a run and per polarisation, one FP64
// mma.sync.m16n8k4: A (16 x 4) holds the real parts' row taps in rows 0-7
// and the imaginary parts' in rows 8-15, B (4 x 8) the column taps, D
// (16 x 8) the 8 x 8 footprint of both planes (taps past the support are
// zero in the table).  With lane = 4 g + t the fragments are a0 = A[g][t],
// a1 = A[g + 8][t], b0 = B[t][g], d = D[g][2t, 2t + 1], D[g + 8][2t, 2t + 1]:
// lane (g, t) reads sample t of the group, row tap g and column tap g, and
// owns cells (g, 2t) and (g, 2t + 1).  Each product is an FP64 multiply-add,
// as a DFMA is; a group's four are summed in the tensor core's order.  Per
// group and lane: 2 tap loads, NPOL staged values, 2 NPOL DMUL and NPOL mma
// (about a quarter of RowLanes' instructions and shared-memory wavefronts
// per sample, for 512 instead of 392 multiply-adds at the FP64 rate).
//
// The warp's lanes first stage 32 samples (one each: FP64 weighted values,
// cell key, tap-table row offsets) into the warp's shared staging area.
// k_grid_tiled (RowLanes) keeps the next round's values and the record of
// the round after in registers while a round is computed; k_grid_mma
// (MmaLanes) copies the next round's raw values into a per-warp ring in
// shared memory with cp.async while a round is computed.
template <int S, int NPOL>
struct GCfg {
  // one CTA per SM; as many warps as the registers allow without spilling
  static constexpr int THREADS = (S >= 9 && NPOL == 4) ? 384 : 512;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int W = TILE + S - 1;                          // sub-grid edge
  static constexpr bool QUARTERS = S <= 8;                         // lane = block * 8 + g
  static constexpr int PPL = QUARTERS ? (NPOL <= 4 ? 1 : 2)
                                      : (S * NPOL <= 32 ? 1 : (S * NPOL <= 64 ? 2 : 4));
  static constexpr int NPGL = NPOL / PPL;                          // polarisation groups
  static constexpr int NCC_FIT = QUARTERS ? 4 / NPGL : 32 / (S * NPGL);
  static constexpr int NCC_CAP = NCC_FIT < 1 ? 1 : (NCC_FIT > S ? S : NCC_FIT);
  static constexpr int KC = (S + NCC_CAP - 1) / NCC_CAP;          // columns per lane
  static constexpr int NCC = (S + KC - 1) / KC;                    // column chunks
  static constexpr int BLOCKS = NPGL * NCC;                        // (pol group, chunk)
  static constexpr int LANES = QUARTERS ? 32 : S * BLOCKS;         // lanes with a role
  static constexpr bool PAIRS = (KC % 2 == 0) || NCC == 1;         // 16-byte tap loads
  static constexpr int KCE = PAIRS ? ((KC + 1) & ~1) : KC;         // taps addressed
  static constexpr int RT0 = (NCC - 1) * KC + KCE;
  static constexpr int RT = ((RT0 > S ? RT0 : S) + 1) & ~1;        // taps per table row
  static constexpr int RWP = (RT % 4 == 0) ? RT + 2 : RT;          // row stride (banks)
  static constexpr size_t tab_bytes = 256 * RWP * sizeof(double);
  static constexpr size_t rs_bytes = 256 * sizeof(double);
  // staged values: [pol][sample] with a 33-entry stride, so the 32 lanes'
  // stores are contiguous and the quarters' loads fall on different banks
  static constexpr int SDS = GT_STAGE + 1;
  static constexpr size_t std_bytes = (size_t)WARPS * NPOL * SDS * sizeof(double2);
  // sub-grid: separate real and imaginary planes of npg x W rows of RS
  // doubles; RS odd and PS = 1 mod 16 spread a flush's 8-byte atomics over
  // the banks (rows and polarisations land on different bank pairs)
  static constexpr int RS = W | 1;
  static constexpr int PS = ((W * RS + 15) / 16) * 16 + 1;
  static constexpr size_t stm_bytes = (size_t)WARPS * GT_STAGE * sizeof(int);
  static constexpr size_t off_rs = tab_bytes;
  static constexpr size_t off_std = off_rs + rs_bytes;
  static constexpr size_t off_stm = off_std + std_bytes;
  static constexpr size_t off_sub = off_stm + stm_bytes;
  static size_t sub_bytes(int npg) { return (size_t)2 * npg * PS * sizeof(double); }
  static size_t total(int npg) { return off_sub + sub_bytes(npg); }
  static_assert(QUARTERS ? BLOCKS <= 4 : S * BLOCKS <= 32, "lane mapping");
  static_assert(NPGL * PPL == NPOL, "polarisation split");
};

// k_grid_mma's shared memory: tap table (rows of 8 taps, zero past the
// support, stride 10), rs, the warps' rings, the warps' tap-row offsets and
// the sub-grid.  A ring slot holds one round: NPOL planes of SDS double2
// entries ([pol][sample]); the raw FP32 values of sample s arrive in its own
// entries (vis pols 0-1 in plane 0, 2-3 in plane 1, weights in plane 2 for
// NPOL 4; vis in plane 0, weights in plane 1 for NPOL 2; vis then weight in
// entry 0 for NPOL 1) and are replaced by the FP64 weighted values.  Entry
// GT_STAGE of each plane (and of the offsets) is a zero sample that empty
// group slots read.
template <int S, int NPOL>
struct MCfg {
  static constexpr int THREADS = 512;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int SLOTS = 2;                                  // rounds per ring
  static constexpr int W = TILE + S - 1;
  static constexpr int RWP = 10;
  static constexpr int SDS = GT_STAGE + 1;
  static constexpr int SLOT = NPOL * SDS;                          // double2 per slot
  static constexpr int RS = W | 1;
  static constexpr int PS = ((W * RS + 15) / 16) * 16 + 1;
  static constexpr size_t tab_bytes = 256 * RWP * sizeof(double);
  static constexpr size_t rs_bytes = 256 * sizeof(double);
  static constexpr size_t ring_bytes = (size_t)WARPS * SLOTS * SLOT * sizeof(double2);
  static constexpr size_t stm_bytes = (size_t)WARPS * SDS * sizeof(int);
  static constexpr size_t off_rs = tab_bytes;
  static constexpr size_t off_ring = off_rs + rs_bytes;
  static constexpr size_t off_stm = off_ring + ring_bytes;
  static constexpr size_t off_sub = off_stm + stm_bytes;
  static size_t sub_bytes(int npg) { return (size_t)2 * npg * PS * sizeof(double); }
  static size_t total(int npg) { return off_sub + sub_bytes(npg); }
  static_assert(S <= 8, "one 8 x 8 footprint per polarisation");
  static_assert(off_ring % 16 == 0, "ring alignment");
};

// Per-offset tap tables: tab[(o + 128) * RWP + i] = cgk[|os * (i - S/2) + o|]
// for i < S (zero beyond) and rs[o + 128] = sum_i of the same, so the sum of
// a sample's footprint weights is rs[ou] * rs[ov].
template <int S, int RWP>
__device__ void build_tap_tables64(double *tab, double *rs, const double *cgk, int cgk_len,
                                   int os) {
  for (int o = threadIdx.x; o < 256; o += blockDim.x) {
    int off = o - 128;
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < RWP; ++i) {
      double v = 0.0;
      if (i < S) {
        int k = os * (i - S / 2) + off;
        k = k < 0 ? -k : k;
        v = (k < cgk_len) ? cgk[k] : 0.0;
        s += v;
      }
      tab[o * RWP + i] = v;
    }
    rs[o] = s;
  }
}

// One staged sample in registers (loads in flight until used).
template <int NPOL>
struct Pref {
  Rec rc;
  float w[NPOL];
  float2 v[NPOL];
  bool ok;
};

// Loads of one sample's weights and visibilities, issued from a record that
// is already in a register (records are loaded one round earlier still, so
// these addresses never wait on a load).
template <int NPOL>
__device__ __forceinline__ void prefetch(Pref<NPOL> &f, const TiledGridArgs &a, const Rec &rc,
                                         bool valid) {
  f.ok = valid;
  if (!valid) return;
  f.rc = rc;
  const int64_t vb = (int64_t)rc.row * a.npol;
  if (a.wt == nullptr) {  // unit weights (degridder adjoint)
#pragma unroll
    for (int p = 0; p < NPOL; ++p) {
      f.w[p] = p < a.npol ? ((a.flag && a.flag[vb + p]) ? 0.f : 1.f) : 0.f;
      f.v[p] = p < a.npol ? __ldg(a.vis + vb + p) : make_float2(0.f, 0.f);
    }
    return;
  }
  if (NPOL == 4 && a.npol == 4 && a.a16) {  // 16-byte loads need 16-byte aligned rows
    const float4 w4 = __ldg((const float4 *)(a.wt + vb));
    f.w[0] = w4.x; f.w[1 % NPOL] = w4.y; f.w[2 % NPOL] = w4.z; f.w[3 % NPOL] = w4.w;
    if (!a.do_psf) {
      const float4 v01 = __ldg((const float4 *)(a.vis + vb));
      const float4 v23 = __ldg((const float4 *)(a.vis + vb + 2));
      f.v[0] = make_float2(v01.x, v01.y);
      f.v[1 % NPOL] = make_float2(v01.z, v01.w);
      f.v[2 % NPOL] = make_float2(v23.x, v23.y);
      f.v[3 % NPOL] = make_float2(v23.z, v23.w);
    }
  } else {
#pragma unroll
    for (int p = 0; p < NPOL; ++p) {
      f.w[p] = p < a.npol ? __ldg(a.wt + vb + p) : 0.f;
      if (!a.do_psf) f.v[p] = p < a.npol ? __ldg(a.vis + vb + p) : make_float2(0.f, 0.f);
    }
  }
}

template <int S, int NPOL>
struct RowLanes {
  using C = GCfg<S, NPOL>;
  static constexpr int PPL = C::PPL, KC = C::KC, KCE = C::KCE;
  double2 acc[PPL][KC];
  int g, pg, c0;
  bool owner;
  int ipm[PPL];  // this lane's image polarisations (-1: none)

  // lanes without a role repeat a valid one (no divergent compute) but
  // never flush
  __device__ __forceinline__ void setup(int lane, const int (&pm)[NPOL]) {
    int blk;
    if (C::QUARTERS) {
      g = lane & 7;
      blk = lane >> 3;
      owner = g < S && blk < C::BLOCKS;
      g = g < S ? g : S - 1;
      blk = blk < C::BLOCKS ? blk : 0;
    } else {
      owner = lane < C::LANES;
      const int li = lane % C::LANES;
      g = li % S;
      blk = li / S;
    }
    pg = blk / C::NCC;
    c0 = (blk % C::NCC) * KC;
#pragma unroll
    for (int pp = 0; pp < PPL; ++pp) {
      ipm[pp] = -1;
#pragma unroll
      for (int p = 0; p < NPOL; ++p)
        if (p == pg * PPL + pp) ipm[pp] = pm[p];
    }
    clear();
  }

  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int pp = 0; pp < PPL; ++pp)
#pragma unroll
      for (int k = 0; k < KC; ++k) acc[pp][k] = make_double2(0.0, 0.0);
  }

  // Adds the run's accumulators (cell key: du | dv << 8) to the shared
  // sub-grid (real plane sre, imaginary plane sim) and clears them.
  // Columns past the support are padding.
  __device__ __forceinline__ void flush(double *sre, double *sim, int key) {
    const int du = key & 255, dv = (key >> 8) & 255;
    const int base = (du + g) * C::RS + dv + c0;
#pragma unroll
    for (int pp = 0; pp < PPL; ++pp) {
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const double2 v = acc[pp][k];
        if (owner && ipm[pp] >= 0 && c0 + k < S && (v.x != 0.0 || v.y != 0.0)) {
          const int e = ipm[pp] * C::PS + base + k;
          atomicAdd(sre + e, v.x);
          atomicAdd(sim + e, v.y);
        }
        acc[pp][k] = make_double2(0.0, 0.0);
      }
    }
  }

  // Staged samples [j, j1) of the current round, all in the current cell.
  __device__ __forceinline__ void run(int j, int j1, const double2 *wd, const int *wm,
                                      const double *tab) {
    for (; j < j1; ++j) {
      const int ro = wm[j];
      const double cu = tab[(ro & 0xffff) + g];
      const double *cvp = tab + (ro >> 16) + c0;
      double cv[KCE];
      if (C::PAIRS) {
#pragma unroll
        for (int k = 0; k + 1 < KC; k += 2) {
          const double2 c2 = *(const double2 *)(cvp + k);
          cv[k] = c2.x;
          cv[k + 1] = c2.y;
        }
        if (KC % 2) cv[KC - 1] = cvp[KC - 1];
      } else {
#pragma unroll
        for (int k = 0; k < KC; ++k) cv[k] = cvp[k];
      }
#pragma unroll
      for (int pp = 0; pp < PPL; ++pp) {
        const double2 d = wd[(pg * PPL + pp) * C::SDS + j];
        const double tr = cu * d.x, ti = cu * d.y;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          acc[pp][k].x = fma(cv[k], tr, acc[pp][k].x);
          acc[pp][k].y = fma(cv[k], ti, acc[pp][k].y);
        }
      }
    }
  }
};

// D += A B for one m16n8k4 FP64 tile (fragment layout above).
__device__ __forceinline__ void mma_f64_m16n8k4(double (&d)[4], double a0, double a1,
                                                double b0) {
  asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

template <int S, int NPOL>
struct MmaLanes {
  using C = MCfg<S, NPOL>;
  double acc[NPOL][4];  // per polarisation: re (g, 2t), re (g, 2t+1), im (g, 2t), im (g, 2t+1)
  int g, t;
  int ipm[NPOL];

  __device__ __forceinline__ void setup(int lane, const int (&pm)[NPOL]) {
    g = lane >> 2;
    t = lane & 3;
#pragma unroll
    for (int p = 0; p < NPOL; ++p) ipm[p] = pm[p];
    clear();
  }

  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int p = 0; p < NPOL; ++p) acc[p][0] = acc[p][1] = acc[p][2] = acc[p][3] = 0.0;
  }

  // Rows and columns past the support hold zeros (zero taps) and are skipped.
  // DET: the sub-grid holds fixed-point integers (value x scale, rounded to
  // nearest), whose sums do not depend on the order of the additions.
  template <bool DET = false>
  __device__ __forceinline__ void flush(double *sre, double *sim, int key, double scale = 0.0) {
    const int du = key & 255, dv = (key >> 8) & 255;
    const int base = (du + g) * C::RS + dv + 2 * t;
#pragma unroll
    for (int p = 0; p < NPOL; ++p) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double re = acc[p][q], im = acc[p][2 + q];
        if (ipm[p] >= 0 && g < S && 2 * t + q < S && (re != 0.0 || im != 0.0)) {
          const int e = ipm[p] * C::PS + base + q;
          if (DET) {
            atomicAdd((unsigned long long *)(sre + e),
                      (unsigned long long)__double2ll_rn(re * scale));
            atomicAdd((unsigned long long *)(sim + e),
                      (unsigned long long)__double2ll_rn(im * scale));
          } else {
            atomicAdd(sre + e, re);
            atomicAdd(sim + e, im);
          }
        }
      }
    }
    clear();
  }

  // Staged samples [j, j1) of the current round (values wd[p * SDS + s]),
  // all in the current cell, in groups of four; a short group's empty slots
  // read the zero sample (entry GT_STAGE: zero values, offset row 0), so
  // their A columns are zero.
  __device__ __forceinline__ void run(int j, int j1, const double2 *wd, const int *wm,
                                      const double *tab) {
    for (; j < j1; j += 4) {
      const int s = j + t < j1 ? j + t : GT_STAGE;
      const int ro = wm[s];
      const double cu = tab[(ro & 0xffff) + g];
      const double cv = tab[(ro >> 16) + g];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        const double2 d = wd[p * C::SDS + s];
        mma_f64_m16n8k4(acc[p], cu * d.x, cu * d.y, cv);
      }
    }
  }

  // A whole round of one cell (32 samples, eight full groups), unrolled so
  // the next groups' operand loads overlap the current group's MMAs.
  __device__ __forceinline__ void run_full(const double2 *wd, const int *wm,
                                           const double *tab) {
#pragma unroll
    for (int j = 0; j < GT_STAGE; j += 4) {
      const int s = j + t;
      const int ro = wm[s];
      const double cu = tab[(ro & 0xffff) + g];
      const double cv = tab[(ro >> 16) + g];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        const double2 d = wd[p * C::SDS + s];
        mma_f64_m16n8k4(acc[p], cu * d.x, cu * d.y, cv);
      }
    }
  }
};

// Sum of weights of a warp's slice: one atomic per warp and polarisation.
template <int NPOL>
__device__ __forceinline__ void add_sum_weight(const TiledGridArgs &a, double (&sw)[NPOL],
                                               const int (&pm)[NPOL], int64_t plane, int lane) {
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    double v = sw[p];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && a.sumw && pm[p] >= 0 && v != 0.0)
      atomicAdd(&a.sumw[plane * a.npg + pm[p]], v);
  }
}

// Adds a tile's shared sub-grid to the global grid and clears it (the whole
// block; one trip count for every thread).
template <int W, int RS, int PS, int THREADS>
__device__ __forceinline__ void flush_subgrid(const TiledGridArgs &a, double *sre, double *sim,
                                              int64_t plane, int tu, int tv) {
  const int sub_n = a.npg * W * W;
  for (int i0 = 0; i0 < sub_n; i0 += THREADS) {
    const int i = i0 + threadIdx.x;
    if (i >= sub_n) continue;
    const int gp = i / (W * W);
    const int cell = i - gp * W * W;
    const int iu = cell / W, iv = cell - iu * W;
    const int e = gp * PS + iu * RS + iv;
    const double2 v = make_double2(sre[e], sim[e]);
    if (v.x != 0.0 || v.y != 0.0) {
      int64_t gu = (int64_t)tu * TILE + iu, gv = (int64_t)tv * TILE + iv;
      int64_t gi = ((plane * a.npg + gp) * a.n_u + gu) * a.n_v + gv;
      if (a.grid_c128) {
        double2 *gd = (double2 *)a.grid + gi;
        atomicAdd(&gd->x, v.x);
        atomicAdd(&gd->y, v.y);
      } else {
        atomicAdd((float2 *)a.grid + gi, make_float2((float)v.x, (float)v.y));
      }
      sre[e] = 0.0;
      sim[e] = 0.0;
    }
  }
}

// Deterministic mode: a warp's sums of weights (summed over its lanes in a
// fixed order) as fixed-point integers.
template <int NPOL>
__device__ __forceinline__ void add_sum_weight_det(const TiledGridArgs &a, double (&sw)[NPOL],
                                                   const int (&pm)[NPOL], int64_t plane,
                                                   int lane, double scale) {
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    double v = sw[p];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && pm[p] >= 0 && v != 0.0)
      atomicAdd(&a.det_sumw[plane * a.npg + pm[p]],
                (unsigned long long)__double2ll_rn(v * scale));
  }
}

// Deterministic mode: the fixed-point sub-grid added to the fixed-point grid
// (integer additions: exact, in any order) and cleared.
template <int W, int RS, int PS, int THREADS>
__device__ __forceinline__ void flush_subgrid_det(const TiledGridArgs &a, double *sre,
                                                  double *sim, int64_t plane, int tu, int tv) {
  unsigned long long *qre = (unsigned long long *)sre, *qim = (unsigned long long *)sim;
  const int sub_n = a.npg * W * W;
  for (int i0 = 0; i0 < sub_n; i0 += THREADS) {
    const int i = i0 + threadIdx.x;
    if (i >= sub_n) continue;
    const int gp = i / (W * W);
    const int cell = i - gp * W * W;
    const int iu = cell / W, iv = cell - iu * W;
    const int e = gp * PS + iu * RS + iv;
    const unsigned long long x = qre[e], y = qim[e];
    if (x != 0ull || y != 0ull) {
      const int64_t gu = (int64_t)tu * TILE + iu, gv = (int64_t)tv * TILE + iv;
      const int64_t gi = ((plane * a.npg + gp) * a.n_u + gu) * a.n_v + gv;
      if (x) atomicAdd(a.det_grid + 2 * gi, x);
      if (y) atomicAdd(a.det_grid + 2 * gi + 1, y);
      qre[e] = 0ull;
      qim[e] = 0ull;
    }
  }
}

// Every CTA has taken its last chunk: the last one to get here re-arms the
// plan's counters for the next launch.
__device__ __forceinline__ void rearm_schedule(const TiledGridArgs &a) {
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&a.sched[1], 1u) == gridDim.x - 1) {
      a.sched[0] = 0u;
      a.sched[1] = 0u;
      __threadfence();
    }
  }
}

// Persistent: one CTA per SM takes chunks of records from a.sched[0] until
// none are left; the last CTA to finish sets both counters back to zero for
// the next launch on the same plan.
template <int S, int NPOL>
__global__ void __launch_bounds__(GCfg<S, NPOL>::THREADS, 1) k_grid_tiled(TiledGridArgs a) {
  using C = GCfg<S, NPOL>;
  constexpr int W = C::W, RWP = C::RWP;
  extern __shared__ __align__(16) unsigned char smem[];
  double *tab = (double *)smem;
  double *rs = (double *)(smem + C::off_rs);
  double2 *st_d = (double2 *)(smem + C::off_std);
  int *st_m = (int *)(smem + C::off_stm);
  double *sre = (double *)(smem + C::off_sub);
  double *sim = sre + (size_t)a.npg * C::PS;
  __shared__ int s_chunk;

  const uint32_t n_rec = *a.n_rec;
  const int64_t n_chunks = ((int64_t)n_rec + a.chunk - 1) / a.chunk;
  const int npg = a.npg;

  build_tap_tables64<S, RWP>(tab, rs, a.cgk, a.cgk_len, a.os);
  // strided loops that precede a block barrier keep one trip count for the
  // whole block (bounds test inside), so every warp reaches the barrier
  // converged
  for (int i0 = 0; i0 < 2 * npg * C::PS; i0 += C::THREADS) {
    const int i = i0 + threadIdx.x;
    if (i < 2 * npg * C::PS) sre[i] = 0.0;
  }

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // image polarisation of each visibility polarisation (-1 drops it)
  int pm[NPOL];
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    int v = p < a.npol ? a.pol_map[p] : -1;
    pm[p] = (v >= 0 && v < npg) ? v : -1;
  }
  RowLanes<S, NPOL> lanes;
  lanes.setup(lane, pm);
  double2 *wd = st_d + warp * NPOL * C::SDS;
  int *wm = st_m + warp * GT_STAGE;

  for (;;) {
    __syncthreads();  // tables and sub-grid ready; previous s_chunk consumed
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(&a.sched[0], 1u);
    __syncthreads();
    const int64_t ch = s_chunk;
    if (ch >= n_chunks) break;
    const uint32_t r0 = (uint32_t)(ch * a.chunk);
    const uint32_t r1 = (uint32_t)min((int64_t)n_rec, (int64_t)r0 + a.chunk);
    int t = find_tile_warp(a.tile_start, a.n_tiles, r0);
    uint32_t seg_lo = r0;
    while (seg_lo < r1) {
      const uint32_t t_end = a.tile_start[t + 1];
      const uint32_t seg_hi = min(r1, t_end);
      if (seg_hi <= seg_lo) {  // empty tile (uniform across the CTA)
        ++t;
        continue;
      }
      const int64_t plane = t / (a.ntu * a.ntv);
      const int64_t trem = t - plane * a.ntu * a.ntv;
      const int tu = (int)(trem / a.ntv), tv = (int)(trem - (int64_t)tu * a.ntv);
      const uint32_t seg_n = seg_hi - seg_lo;
      const uint32_t w_lo = seg_lo + (uint32_t)(((uint64_t)seg_n * warp) / C::WARPS);
      const uint32_t w_hi = seg_lo + (uint32_t)(((uint64_t)seg_n * (warp + 1)) / C::WARPS);
      const int n_rounds = (int)((w_hi - w_lo + GT_STAGE - 1) / GT_STAGE);

      int cur = -1;  // the warp's current cell
      double sw[NPOL];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) sw[p] = 0.0;

      // software pipeline: values of round rd + 1 and the record of round
      // rd + 2 are in flight while round rd is computed
      Pref<NPOL> pf;
      Rec rnext;
      {
        const uint32_t r = w_lo + lane;
        Rec r0;
        if (r < w_hi) r0 = a.recs[r];
        prefetch<NPOL>(pf, a, r0, r < w_hi);
      }
      bool rnext_ok = w_lo + GT_STAGE + lane < w_hi;
      if (rnext_ok) rnext = a.recs[w_lo + GT_STAGE + lane];
      for (int rd = 0; rd < n_rounds; ++rd) {
        // ---- stage this round's samples, one per lane: FP64 weighted
        // values, the cell key and the offsets of the two tap-table rows
        int my_key = -1;
        if (pf.ok) {
          const Rec rc = pf.rc;
          const double nrm = rs[rc.ou] * rs[rc.ov];
          double scl = 1.0;
          if (a.inv_norm) scl = nrm != 0.0 ? 1.0 / nrm : 0.0;
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            double2 d;
            if (a.do_psf) d = make_double2((double)pf.w[p], 0.0);
            else d = make_double2((double)pf.v[p].x * (double)pf.w[p] * scl,
                                  (double)pf.v[p].y * (double)pf.w[p] * scl);
            // the reference skips NaN and exact-zero weighted data
            // (standard_grid.py:378)
            const bool ok = p < a.npol && !isnan(d.x) && !isnan(d.y) &&
                            (d.x != 0.0 || d.y != 0.0);
            wd[p * C::SDS + lane] = ok ? d : make_double2(0.0, 0.0);
            if (ok) sw[p] += (double)pf.w[p] * nrm;
          }
          my_key = (int)rc.du | ((int)rc.dv << 8);
          wm[lane] = (int)rc.ou * RWP | (((int)rc.ov * RWP) << 16);
        }
        // samples that open a new cell (the first compares with the last
        // cell of the previous round)
        int prev = __shfl_up_sync(0xffffffffu, my_key, 1);
        if (lane == 0) prev = cur;
        const unsigned starts = __ballot_sync(0xffffffffu, my_key >= 0 && my_key != prev);
        __syncwarp();
        // ---- next round's values go out before this round is computed
        if (rd + 1 < n_rounds) {
          prefetch<NPOL>(pf, a, rnext, rnext_ok);
          const uint32_t r = w_lo + (uint32_t)(rd + 2) * GT_STAGE + lane;
          rnext_ok = r < w_hi;
          if (rnext_ok) rnext = a.recs[r];
        }
        // ---- compute the round's samples in runs of one cell
        const int jn = (int)min((uint32_t)GT_STAGE, w_hi - (w_lo + (uint32_t)rd * GT_STAGE));
        int j = 0;
        while (j < jn) {
          if ((starts >> j) & 1u) {
            if (cur >= 0) lanes.flush(sre, sim, cur);
            cur = __shfl_sync(0xffffffffu, my_key, j);
          }
          const unsigned later = j < 31 ? (starts & (0xfffffffeu << j)) : 0u;
          const int j1 = later ? min(jn, __ffs(later) - 1) : jn;
          lanes.run(j, j1, wd, wm, tab);
          j = j1;
        }
        __syncwarp();
      }
      if (cur >= 0) lanes.flush(sre, sim, cur);
      add_sum_weight<NPOL>(a, sw, pm, plane, lane);
      __syncthreads();
      flush_subgrid<W, C::RS, C::PS, C::THREADS>(a, sre, sim, plane, tu, tv);
      __syncthreads();
      seg_lo = seg_hi;
      if (seg_hi == t_end) ++t;
    }
  }
  rearm_schedule(a);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src));
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src));
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Raw values of one sample (this lane's record) into its entries of a ring
// slot (layout at MCfg): 16-byte copies when a.a16 says the rows allow them,
// else one copy per polarisation.
template <int NPOL>
__device__ __forceinline__ void issue_raw(const TiledGridArgs &a, double2 *slot, int s,
                                          uint32_t row) {
  constexpr int SDS = GT_STAGE + 1;
  const int64_t vb = (int64_t)row * a.npol;
  unsigned char *e0 = (unsigned char *)(slot + s);
  unsigned char *e1 = (unsigned char *)(slot + (NPOL > 1 ? SDS : 0) + s);
  unsigned char *e2 = (unsigned char *)(slot + (NPOL > 2 ? 2 * SDS : 0) + s);
  if (NPOL == 4) {  // vis 0-1 -> plane 0, vis 2-3 -> plane 1, weights -> plane 2
    if (a.a16) {
      if (!a.do_psf) {
        cp_async16(e0, a.vis + vb);
        cp_async16(e1, a.vis + vb + 2);
      }
      cp_async16(e2, a.wt + vb);
    } else {
      for (int p = 0; p < a.npol; ++p) {
        if (!a.do_psf) cp_async8((p < 2 ? e0 : e1) + 8 * (p & 1), a.vis + vb + p);
        cp_async4(e2 + 4 * p, a.wt + vb + p);
      }
    }
  } else if (NPOL == 2) {  // vis -> plane 0, weights -> plane 1
    if (a.a16 && a.npol == 2) {
      if (!a.do_psf) cp_async16(e0, a.vis + vb);
      cp_async8(e1, a.wt + vb);
    } else {
      for (int p = 0; p < a.npol; ++p) {
        if (!a.do_psf) cp_async8(e0 + 8 * p, a.vis + vb + p);
        cp_async4(e1 + 4 * p, a.wt + vb + p);
      }
    }
  } else {  // vis then weight in entry 0
    if (!a.do_psf) cp_async8(e0, a.vis + vb);
    cp_async4(e0 + 8, a.wt + vb);
  }
}

// Reads sample s's raw values back from its ring entries (after the copies
// are complete).
template <int NPOL>
__device__ __forceinline__ void read_raw(const TiledGridArgs &a, const double2 *slot, int s,
                                         float2 (&v)[NPOL], float (&w)[NPOL]) {
  constexpr int SDS = GT_STAGE + 1;
  if (NPOL == 4) {
    const float4 v01 = *(const float4 *)(slot + s);
    const float4 v23 = *(const float4 *)(slot + SDS + s);
    const float4 w4 = *(const float4 *)(slot + 2 * SDS + s);
    v[0] = make_float2(v01.x, v01.y);
    v[1 % NPOL] = make_float2(v01.z, v01.w);
    v[2 % NPOL] = make_float2(v23.x, v23.y);
    v[3 % NPOL] = make_float2(v23.z, v23.w);
    w[0] = w4.x; w[1 % NPOL] = w4.y; w[2 % NPOL] = w4.z; w[3 % NPOL] = w4.w;
  } else if (NPOL == 2) {
    const float4 v01 = *(const float4 *)(slot + s);
    const float2 w2 = *(const float2 *)(slot + (NPOL > 1 ? SDS : 0) + s);
    v[0] = make_float2(v01.x, v01.y);
    v[1 % NPOL] = make_float2(v01.z, v01.w);
    w[0] = w2.x;
    w[1 % NPOL] = w2.y;
  } else {
    const float4 e = *(const float4 *)(slot + s);
    v[0] = make_float2(e.x, e.y);
    w[0] = e.z;
  }
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    if (p >= a.npol) {  // polarisations past npol were not copied
      v[p] = make_float2(0.f, 0.f);
      w[p] = 0.f;
    } else if (a.do_psf) {
      v[p] = make_float2(0.f, 0.f);
    }
  }
}

// k_grid_tiled's schedule and segments with MmaLanes and a cp.async ring of
// two slots: the raw values of round rd + 1 are copied while round rd is
// computed (a round of 32 samples takes several microseconds, well beyond
// the copies' latency; a third slot, two rounds ahead, measured 3 % slower),
// and records are loaded one round before their copies are issued.  Only
// for weighted gridding (a.wt != NULL, no 1 / norm scaling).
template <int S, int NPOL, bool DET = false>
__global__ void __launch_bounds__(MCfg<S, NPOL>::THREADS, 1) k_grid_mma(TiledGridArgs a) {
  using C = MCfg<S, NPOL>;
  const double dscale = DET ? a.det_scale[0] : 0.0;
  const double wscale = DET ? a.det_scale[1] : 0.0;
  constexpr int W = C::W, RWP = C::RWP;
  extern __shared__ __align__(16) unsigned char smem[];
  double *tab = (double *)smem;
  double *rs = (double *)(smem + C::off_rs);
  double2 *ring = (double2 *)(smem + C::off_ring);
  int *st_m = (int *)(smem + C::off_stm);
  double *sre = (double *)(smem + C::off_sub);
  double *sim = sre + (size_t)a.npg * C::PS;
  __shared__ int s_chunk;

  const uint32_t n_rec = *a.n_rec;
  const int64_t n_chunks = ((int64_t)n_rec + a.chunk - 1) / a.chunk;
  const int npg = a.npg;

  build_tap_tables64<S, RWP>(tab, rs, a.cgk, a.cgk_len, a.os);
  for (int i0 = 0; i0 < 2 * npg * C::PS; i0 += C::THREADS) {
    const int i = i0 + threadIdx.x;
    if (i < 2 * npg * C::PS) sre[i] = 0.0;
  }

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int pm[NPOL];
#pragma unroll
  for (int p = 0; p < NPOL; ++p) {
    int v = p < a.npol ? a.pol_map[p] : -1;
    pm[p] = (v >= 0 && v < npg) ? v : -1;
  }
  MmaLanes<S, NPOL> lanes;
  lanes.setup(lane, pm);
  double2 *wring = ring + (size_t)warp * C::SLOTS * C::SLOT;
  int *wm = st_m + warp * C::SDS;
  if (lane == 0) {  // the zero samples (nothing else writes entry GT_STAGE)
    for (int k = 0; k < C::SLOTS; ++k)
#pragma unroll
      for (int p = 0; p < NPOL; ++p)
        wring[k * C::SLOT + p * C::SDS + GT_STAGE] = make_double2(0.0, 0.0);
    wm[GT_STAGE] = 0;
  }

  for (;;) {
    __syncthreads();  // tables and sub-grid ready; previous s_chunk consumed
    if (threadIdx.x == 0) s_chunk = (int)atomicAdd(&a.sched[0], 1u);
    __syncthreads();
    const int64_t ch = s_chunk;
    if (ch >= n_chunks) break;
    const uint32_t r0 = (uint32_t)(ch * a.chunk);
    const uint32_t r1 = (uint32_t)min((int64_t)n_rec, (int64_t)r0 + a.chunk);
    int t = find_tile_warp(a.tile_start, a.n_tiles, r0);
    uint32_t seg_lo = r0;
    while (seg_lo < r1) {
      const uint32_t t_end = a.tile_start[t + 1];
      const uint32_t seg_hi = min(r1, t_end);
      if (seg_hi <= seg_lo) {
        ++t;
        continue;
      }
      const int64_t plane = t / (a.ntu * a.ntv);
      const int64_t trem = t - plane * a.ntu * a.ntv;
      const int tu = (int)(trem / a.ntv), tv = (int)(trem - (int64_t)tu * a.ntv);
      const uint32_t seg_n = seg_hi - seg_lo;
      const uint32_t w_lo = seg_lo + (uint32_t)(((uint64_t)seg_n * warp) / C::WARPS);
      const uint32_t w_hi = seg_lo + (uint32_t)(((uint64_t)seg_n * (warp + 1)) / C::WARPS);
      const int n_rounds = (int)((w_hi - w_lo + GT_STAGE - 1) / GT_STAGE);

      int cur = -1;
      double sw[NPOL];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) sw[p] = 0.0;

      // records of rounds rd and rd + 1 (row 0xffffffff: none)
      Rec rc0, rc1;
      auto load_rec = [&](int rd) {
        const uint32_t r = w_lo + (uint32_t)rd * GT_STAGE + lane;
        Rec x;
        if (rd < n_rounds && r < w_hi) x = a.recs[r];
        else x.row = 0xffffffffu;
        return x;
      };
      rc0 = load_rec(0);
      rc1 = load_rec(1);
      if (rc0.row != 0xffffffffu) issue_raw<NPOL>(a, wring, lane, rc0.row);
      cp_async_commit();
      for (int rd = 0; rd < n_rounds; ++rd) {
        double2 *slot = wring + (rd % C::SLOTS) * C::SLOT;
        cp_async_wait<0>();  // this lane's copies of round rd are complete
        // ---- stage: FP64 weighted values in place of the raw ones, the
        // cell key and the offsets of the two tap-table rows
        int my_key = -1;
        if (rc0.row != 0xffffffffu) {
          float2 v[NPOL];
          float w[NPOL];
          read_raw<NPOL>(a, slot, lane, v, w);
          const double nrm = rs[rc0.ou] * rs[rc0.ov];
#pragma unroll
          for (int p = 0; p < NPOL; ++p) {
            double2 d;
            // the reference skips NaN and exact-zero weighted data
            // (standard_grid.py:378); tested on the FP32 factors: their FP64
            // product is exact, NaN exactly when their FP32 product is, and
            // zero exactly when a factor is (the FP32 pipe, not the FP64 one
            // the MMAs use)
            bool ok;
            if (a.do_psf) {
              d = make_double2((double)w[p], 0.0);
              ok = !isnan(w[p]) && w[p] != 0.f;
            } else {
              d = make_double2((double)v[p].x * (double)w[p], (double)v[p].y * (double)w[p]);
              ok = !isnan(__fmul_rn(v[p].x, w[p])) && !isnan(__fmul_rn(v[p].y, w[p])) &&
                   w[p] != 0.f && (v[p].x != 0.f || v[p].y != 0.f);
            }
            ok = ok && p < a.npol;
            slot[p * C::SDS + lane] = ok ? d : make_double2(0.0, 0.0);
            if (ok) sw[p] += (double)w[p] * nrm;
          }
          my_key = (int)rc0.du | ((int)rc0.dv << 8);
          wm[lane] = (int)rc0.ou * RWP | (((int)rc0.ov * RWP) << 16);
        }
        int prev = __shfl_up_sync(0xffffffffu, my_key, 1);
        if (lane == 0) prev = cur;
        const unsigned starts = __ballot_sync(0xffffffffu, my_key >= 0 && my_key != prev);
        // ---- copies of round rd + 1 (into the slot round rd - 1 used) and
        // the record of round rd + 2
        if (rc1.row != 0xffffffffu)
          issue_raw<NPOL>(a, wring + ((rd + 1) % C::SLOTS) * C::SLOT, lane, rc1.row);
        cp_async_commit();
        const Rec rc2 = load_rec(rd + 2);
        __syncwarp();
        // ---- compute the round's samples in runs of one cell
        const int jn = (int)min((uint32_t)GT_STAGE, w_hi - (w_lo + (uint32_t)rd * GT_STAGE));
        int j = 0;
        if (starts <= 1u && jn == GT_STAGE) {  // one run over the whole round
          if (starts) {
            if (cur >= 0) lanes.template flush<DET>(sre, sim, cur, dscale);
            cur = __shfl_sync(0xffffffffu, my_key, 0);
          }
          lanes.run_full(slot, wm, tab);
          j = jn;
        }
        while (j < jn) {
          if ((starts >> j) & 1u) {
            if (cur >= 0) lanes.template flush<DET>(sre, sim, cur, dscale);
            cur = __shfl_sync(0xffffffffu, my_key, j);
          }
          const unsigned later = j < 31 ? (starts & (0xfffffffeu << j)) : 0u;
          const int j1 = later ? min(jn, __ffs(later) - 1) : jn;
          lanes.run(j, j1, slot, wm, tab);
          j = j1;
        }
        __syncwarp();
        rc0 = rc1;
        rc1 = rc2;
      }
      cp_async_wait<0>();
      if (cur >= 0) lanes.template flush<DET>(sre, sim, cur, dscale);
      if (DET) add_sum_weight_det<NPOL>(a, sw, pm, plane, lane, wscale);
      else add_sum_weight<NPOL>(a, sw, pm, plane, lane);
      __syncthreads();
      if (DET) flush_subgrid_det<W, C::RS, C::PS, C::THREADS>(a, sre, sim, plane, tu, tv);
      else flush_subgrid<W, C::RS, C::PS, C::THREADS>(a, sre, sim, plane, tu, tv);
      __syncthreads();
      seg_lo = seg_hi;
      if (seg_hi == t_end) ++t;
    }
  }
  rearm_schedule(a);
}

template <int S, int NPOL>
static int launch_grid_rows(const TiledGridArgs &a, int64_t nblocks, cudaStream_t st) {
  using C = GCfg<S, NPOL>;
  size_t smem = C::total(a.npg);
  static bool configured[64] = {false};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    AV_CUDA(cudaFuncSetAttribute(k_grid_tiled<S, NPOL>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::total(4)));
    configured[dev] = true;
  }
  k_grid_tiled<S, NPOL><<<(unsigned)nblocks, C::THREADS, smem, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

template <int S, int NPOL, bool DET = false>
static int launch_grid_mma(const TiledGridArgs &a, int64_t nblocks, cudaStream_t st) {
  using C = MCfg<S, NPOL>;
  size_t smem = C::total(a.npg);
  static bool configured[64] = {false};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    AV_CUDA(cudaFuncSetAttribute(k_grid_mma<S, NPOL, DET>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::total(4)));
    configured[dev] = true;
  }
  k_grid_mma<S, NPOL, DET><<<(unsigned)nblocks, C::THREADS, smem, st>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// k_grid_mma for weighted gridding as the AV_TUNE_GRID_LANES knob says
// (automatically for supports 5-8: with smaller footprints most of the 8 x 8
// tile is padding and the row lanes are faster); k_grid_tiled otherwise
// (support 9, the degridder's adjoint).
template <int S, int NPOL>
static int launch_grid_tiled(const TiledGridArgs &a, int64_t nblocks, cudaStream_t st) {
  if constexpr (S <= 8) {
    const int64_t lanes = tune_value(AV_TUNE_GRID_LANES);
    const bool mma = lanes == AV_GRID_LANES_MMA || (lanes == AV_GRID_LANES_AUTO && S >= 5);
    if (a.wt != nullptr && !a.inv_norm && mma) return launch_grid_mma<S, NPOL>(a, nblocks, st);
  }
  return launch_grid_rows<S, NPOL>(a, nblocks, st);
}

template <int S>
static int dispatch_npol(const TiledGridArgs &a, int npol, int64_t nb, cudaStream_t st) {
  if (npol == 1) return launch_grid_tiled<S, 1>(a, nb, st);
  if (npol == 2) return launch_grid_tiled<S, 2>(a, nb, st);
  return launch_grid_tiled<S, 4>(a, nb, st);
}

// Chunks of records the persistent CTAs take one at a time: about
// AV_TUNE_GRID_CHUNKS_PER_SM (16) per SM, so the last chunks even out the
// CTAs' finishing times, and at least 2048 records, so a chunk's tile
// flushes stay small against its samples.
static int64_t grid_chunking(int64_t rows, int64_t &nblocks) {
  const int sms = sm_count();
  const int64_t per_sm = tune_value(AV_TUNE_GRID_CHUNKS_PER_SM);
  int64_t chunk = (rows + (int64_t)sms * per_sm - 1) / ((int64_t)sms * per_sm);
  if (chunk < 2048) chunk = 2048;
  const int64_t n_chunks = (rows + chunk - 1) / chunk;
  nblocks = n_chunks < sms ? n_chunks : sms;
  if (nblocks < 1) nblocks = 1;
  return chunk;
}

static int dispatch_support(const TiledGridArgs &a, int support, int npol, int64_t nb,
                            cudaStream_t st) {
  switch (support) {
    case 3: return dispatch_npol<3>(a, npol, nb, st);
    case 4: return dispatch_npol<4>(a, npol, nb, st);
    case 5: return dispatch_npol<5>(a, npol, nb, st);
    case 6: return dispatch_npol<6>(a, npol, nb, st);
    case 7: return dispatch_npol<7>(a, npol, nb, st);
    case 8: return dispatch_npol<8>(a, npol, nb, st);
    case 9: return dispatch_npol<9>(a, npol, nb, st);
  }
  set_error("av_grid_tiled: support %d not in [3, 9]", support);
  return AV_ERR_UNSUPPORTED;
}

// ---------------------------------------------------- deterministic mode ----
// av_grid_tiled_execute_det: k_grid_mma over a row-ordered plan with the
// run, sub-grid and grid sums in 64-bit fixed point.  A run's FP64 sum is
// fixed by the order of its records (rows) and by where the chunk and warp
// slices cut it (fixed by the plan and the launch settings); every sum after
// that is an integer addition, exact in any order.  The scale 2^F is chosen
// from a bound of any cell's sum of magnitudes, n_rec * max|value| *
// max|tap|^2, so that F leaves that bound below 2^61 (no overflow; the
// rounding of each run sum is at most 2^-F-1).  The sums of weights use
// their own bound, n_rec * max|weight| * (S max|tap|)^2.
template <int NPOL>
static int dispatch_det_npol(const TiledGridArgs &a, int support, int64_t nb, cudaStream_t st) {
  switch (support) {
    case 3: return launch_grid_mma<3, NPOL, true>(a, nb, st);
    case 4: return launch_grid_mma<4, NPOL, true>(a, nb, st);
    case 5: return launch_grid_mma<5, NPOL, true>(a, nb, st);
    case 6: return launch_grid_mma<6, NPOL, true>(a, nb, st);
    case 7: return launch_grid_mma<7, NPOL, true>(a, nb, st);
    case 8: return launch_grid_mma<8, NPOL, true>(a, nb, st);
  }
  set_error("av_grid_tiled_execute_det: support %d not in [3, 8]", support);
  return AV_ERR_UNSUPPORTED;
}

// Largest |re|, |im| of the weighted values and |weight| of the planned
// samples that the gridder adds (NaN skipped), as bit patterns of
// non-negative doubles (whose integer order is their numeric order).
__global__ void __launch_bounds__(256) k_det_bound(TiledGridArgs a, unsigned long long *mx) {
  const uint32_t n_rec = *a.n_rec;
  double md = 0.0, mw = 0.0;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rec;
       r += gridDim.x * blockDim.x) {
    const int64_t vb = (int64_t)a.recs[r].row * a.npol;
    for (int p = 0; p < a.npol; ++p) {
      const double w = (double)a.wt[vb + p];
      double dx = w, dy = 0.0;
      if (!a.do_psf) {
        const float2 v = a.vis[vb + p];
        dx = (double)v.x * w;
        dy = (double)v.y * w;
      }
      if (isnan(dx) || isnan(dy) || (dx == 0.0 && dy == 0.0)) continue;
      md = fmax(md, fmax(fabs(dx), fabs(dy)));
      mw = fmax(mw, fabs(w));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
    mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(mx, (unsigned long long)__double_as_longlong(md));
    atomicMax(mx + 1, (unsigned long long)__double_as_longlong(mw));
  }
}

// 2^F with bound * 2^F < 2^61 (2^0 for a zero bound); err = 1 for a bound
// that is not finite (an infinite value has no fixed-point sum).
__device__ __forceinline__ double det_scale_of(double bound, int *err) {
  if (!(bound <= 1.7e308)) {
    *err = 1;
    return 0.0;
  }
  if (bound == 0.0) return 1.0;
  int e = 0;
  frexp(bound, &e);  // bound < 2^e
  int f = 61 - e;
  if (f > 1000) f = 1000;
  return ldexp(1.0, f);
}

__global__ void k_det_scale(const uint32_t *n_rec, const unsigned long long *mx,
                            const double *cgk, int cgk_len, int support, double *scale,
                            int *err) {
  double mt = 0.0;
  for (int i = 0; i < cgk_len; ++i) mt = fmax(mt, fabs(cgk[i]));
  const double n = (double)*n_rec;
  const double md = __longlong_as_double((long long)mx[0]);
  const double mw = __longlong_as_double((long long)mx[1]);
  *err = 0;
  scale[0] = det_scale_of(n * md * mt * mt, err);
  scale[1] = det_scale_of(n * mw * (support * mt) * (support * mt), err);
}

// grid += fixed-point sums / 2^F (one FP64 or FP32 addition per value);
// sum_weight likewise.
__global__ void __launch_bounds__(256) k_det_finish(void *grid, int grid_c128,
                                                    const unsigned long long *q, int64_t n,
                                                    double *sumw, const unsigned long long *qw,
                                                    int64_t nw, const double *scale) {
  const double inv = 1.0 / scale[0], invw = 1.0 / scale[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const long long x = (long long)q[2 * i], y = (long long)q[2 * i + 1];
    if (x == 0 && y == 0) continue;
    const double re = (double)x * inv, im = (double)y * inv;
    if (grid_c128) {
      double2 *g = (double2 *)grid + i;
      g->x += re;
      g->y += im;
    } else {
      float2 *g = (float2 *)grid + i;
      g->x = (float)((double)g->x + re);
      g->y = (float)((double)g->y + im);
    }
  }
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < nw) sumw[t] += (double)(long long)qw[t] * invw;
}

}  // namespace av

using namespace av;

extern "C" {

int av_grid_plain(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                  int do_imaging_weight, const void *vis, int vis_dtype, const void *weight,
                  int weight_dtype, const double *uvw, const double *freq,
                  const int32_t *chan_map, const int32_t *pol_map, const double *cgk,
                  int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                  int oversampling, int64_t nt, int64_t nb, int64_t nchan, int64_t npol,
                  int64_t n_img_chan, int64_t n_img_pol, void *stream) {
  clear_error();
  AV_CHECK_ARG(grid && sum_weight && weight && uvw && freq && chan_map && pol_map && cgk,
               "av_grid_plain: null pointer");
  AV_CHECK_ARG(do_psf || vis, "av_grid_plain: vis is required unless do_psf");
  AV_CHECK_ARG(grid_dtype >= AV_F32 && grid_dtype <= AV_C128, "av_grid_plain: grid dtype");
  AV_CHECK_ARG(do_psf || grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_grid_plain: a real grid needs do_psf");
  AV_CHECK_ARG(vis_dtype == AV_C64 || vis_dtype == AV_C128 || do_psf, "av_grid_plain: vis dtype");
  AV_CHECK_ARG(weight_dtype == AV_F32 || weight_dtype == AV_F64, "av_grid_plain: weight dtype");
  AV_CHECK_ARG(n_u > 0 && n_v > 0 && support >= 1 && oversampling >= 1,
               "av_grid_plain: bad grid/kernel sizes");
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nchan >= 0 && npol >= 0, "av_grid_plain: bad shape");
  int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  GridArgs a;
  a.grid = grid; a.grid_dtype = grid_dtype; a.sumw = sum_weight;
  a.do_psf = do_psf; a.do_iw = do_imaging_weight;
  a.vis = vis; a.vis_dtype = vis_dtype; a.wt = weight; a.wt_dtype = weight_dtype;
  a.uvw = uvw; a.freq = freq; a.chan_map = chan_map; a.pol_map = pol_map; a.cgk = cgk;
  a.n_u = n_u; a.n_v = n_v; a.dl0 = delta_l; a.dl1 = delta_m;
  a.support = support; a.os = oversampling;
  a.nt = nt; a.nb = nb; a.nchan = nchan; a.npol = npol;
  a.n_img_chan = n_img_chan; a.n_img_pol = n_img_pol;
  k_grid_plain<<<(unsigned)((rows + 255) / 256), 256, 0, as_stream(stream)>>>(a);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_grid_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u,
                                    int64_t n_v, int64_t n_img_chan, int support) {
  PlanGeom g;
  plan_geometry(g, nt, nb, nchan, n_img_chan, n_u, n_v, support, 100);
  return plan_workspace_bytes(g);
}

static int grid_geom_checked(PlanGeom &g, int64_t n_u, int64_t n_v, int support,
                             int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                             int64_t n_img_chan, void *workspace, size_t workspace_bytes,
                             Plan &p, const char *who) {
  AV_CHECK_ARG(support >= 3 && support <= 9, "%s: support must be in [3, 9]", who);
  AV_CHECK_ARG(oversampling >= 1 && oversampling <= 254, "%s: oversampling must be in [1, 254]",
               who);
  AV_CHECK_ARG(n_u >= support && n_v >= support && n_u < 131072 && n_v < 131072,
               "%s: grid size out of range", who);
  AV_CHECK_ARG(nt >= 0 && nb >= 0 && nchan >= 0 && n_img_chan >= 1, "%s: bad shape", who);
  AV_CHECK_ARG(workspace && (((uintptr_t)workspace) & 255) == 0,
               "%s: workspace must be 256-byte aligned", who);
  plan_geometry(g, nt, nb, nchan, n_img_chan, n_u, n_v, support, oversampling);
  g.convention = 0;
  g.chk_x = g.chk_y = 0;
  g.scale0 = g.scale1 = g.offset0 = g.offset1 = 0.0;
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

int av_grid_tiled_plan(const double *uvw, const double *freq, const int32_t *chan_map,
                       int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                       int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                       int64_t n_img_chan, void *workspace, size_t workspace_bytes,
                       void *stream) {
  clear_error();
  AV_CHECK_ARG(uvw && freq && chan_map, "av_grid_tiled_plan: null pointer");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, oversampling, nt, nb, nchan, n_img_chan,
                             workspace, workspace_bytes, p, "av_grid_tiled_plan");
  if (rc) return rc;
  return plan_build(g, p, uvw, freq, chan_map, delta_l, delta_m, as_stream(stream));
}

int av_grid_tiled_plan_weighted(const double *uvw, const double *freq, const int32_t *chan_map,
                                const float *weight, int64_t npol, int64_t n_u, int64_t n_v,
                                double delta_l, double delta_m, int support, int oversampling,
                                int64_t nt, int64_t nb, int64_t nchan, int64_t n_img_chan,
                                void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(uvw && freq && chan_map && weight, "av_grid_tiled_plan_weighted: null pointer");
  AV_CHECK_ARG(npol >= 1 && npol <= 4, "av_grid_tiled_plan_weighted: npol must be in [1, 4]");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, oversampling, nt, nb, nchan, n_img_chan,
                             workspace, workspace_bytes, p, "av_grid_tiled_plan_weighted");
  if (rc) return rc;
  return plan_build(g, p, uvw, freq, chan_map, delta_l, delta_m, as_stream(stream), weight,
                    (int)npol);
}

int av_grid_tiled_clear(void *grid, int grid_dtype, int64_t n_img_pol, int64_t n_u, int64_t n_v,
                        int support, int64_t nt, int64_t nb, int64_t nchan, int64_t n_img_chan,
                        const void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(grid, "av_grid_tiled_clear: null pointer");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_grid_tiled_clear: grid must be complex64 or complex128");
  AV_CHECK_ARG(n_img_pol >= 1, "av_grid_tiled_clear: bad shape");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, 100, nt, nb, nchan, n_img_chan,
                             (void *)workspace, workspace_bytes, p, "av_grid_tiled_clear");
  if (rc) return rc;
  return plan_clear_tiles(g, p, grid, grid_dtype == AV_C128, n_img_pol, as_stream(stream));
}

int av_tiled_plan_shared(const double *uvw, const double *freq, const int32_t *chan_map,
                         int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                         int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                         int64_t n_img_chan, void *workspace, size_t workspace_bytes,
                         void *stream) {
  clear_error();
  AV_CHECK_ARG(uvw && freq && chan_map, "av_tiled_plan_shared: null pointer");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, oversampling, nt, nb, nchan, n_img_chan,
                             workspace, workspace_bytes, p, "av_tiled_plan_shared");
  if (rc) return rc;
  // the degridder's conventions for a grid of (n_img_chan, pols, n_u, n_v)
  // and cell (delta_l, delta_m), as degrid_spheroid_ms4 passes them
  // (standard_degrid.py:568-584): scale -cell * n, offset n / 2, bounds
  // against shape[3] and shape[2]
  g.convention = 2;
  g.chk_x = n_v;
  g.chk_y = n_u;
  g.scale0 = -delta_l * (double)n_u;
  g.scale1 = -delta_m * (double)n_v;
  g.offset0 = (double)n_u / 2.0;
  g.offset1 = (double)n_v / 2.0;
  return plan_build(g, p, uvw, freq, chan_map, delta_l, delta_m, as_stream(stream));
}

int av_tiled_plan_counts(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u, int64_t n_v,
                         int64_t n_img_chan, int support, const void *workspace,
                         size_t workspace_bytes, uint32_t *out, void *stream) {
  clear_error();
  AV_CHECK_ARG(out, "av_tiled_plan_counts: null pointer");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, 100, nt, nb, nchan, n_img_chan,
                             (void *)workspace, workspace_bytes, p, "av_tiled_plan_counts");
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  AV_CUDA(cudaMemcpyAsync(&out[0], p.offs + g.n_keys(), sizeof(uint32_t), cudaMemcpyDeviceToHost,
                          st));
  AV_CUDA(cudaMemcpyAsync(&out[1], p.exc_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  AV_CUDA(cudaStreamSynchronize(st));
  return AV_OK;
}

int av_grid_tiled_execute(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                          const void *vis, int vis_dtype, const void *weight, int weight_dtype,
                          const int32_t *pol_map, const double *cgk, int64_t n_u, int64_t n_v,
                          int support, int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                          int64_t npol, int64_t n_img_chan, int64_t n_img_pol, void *workspace,
                          size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(grid && sum_weight && weight && pol_map && cgk,
               "av_grid_tiled_execute: null pointer");
  AV_CHECK_ARG(do_psf || vis, "av_grid_tiled_execute: vis is required unless do_psf");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_grid_tiled_execute: grid must be complex64 or complex128");
  AV_CHECK_ARG(do_psf || vis_dtype == AV_C64, "av_grid_tiled_execute: vis must be complex64");
  AV_CHECK_ARG(weight_dtype == AV_F32, "av_grid_tiled_execute: weight must be float32");
  AV_CHECK_ARG(npol >= 0 && npol <= 4 && n_img_pol >= 1 && n_img_pol <= 4,
               "av_grid_tiled_execute: npol and n_img_pol must be in [1, 4]");
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, oversampling, nt, nb, nchan, n_img_chan,
                             workspace, workspace_bytes, p, "av_grid_tiled_execute");
  if (rc) return rc;
  int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  int npol_t = npol <= 1 ? 1 : (npol <= 2 ? 2 : 4);
  TiledGridArgs a;
  a.recs = p.recs;
  a.tile_start = p.tile_start;
  a.n_rec = p.offs + g.n_keys();
  a.n_tiles = g.n_tiles();
  a.ntu = g.ntu;
  a.ntv = g.ntv;
  int64_t nblocks = 0;
  a.chunk = grid_chunking(rows, nblocks);
  a.sched = p.counters;
  a.vis = (const float2 *)vis;
  a.wt = (const float *)weight;
  a.do_psf = do_psf;
  a.cgk = cgk;
  a.cgk_len = oversampling * (support / 2 + 1);
  a.os = oversampling;
  a.pol_map = pol_map;
  a.npol = (int)npol;
  a.npg = (int)n_img_pol;
  a.grid = grid;
  a.grid_c128 = grid_dtype == AV_C128;
  a.sumw = sum_weight;
  a.n_u = n_u;
  a.n_v = n_v;
  a.inv_norm = 0;
  a.flag = nullptr;
  {
    const uintptr_t vp = (uintptr_t)vis, wp = (uintptr_t)weight;
    const bool v16 = do_psf || vp % 16 == 0;
    a.a16 = v16 && ((npol == 4 && wp % 16 == 0) || (npol == 2 && wp % 8 == 0));
  }
  return dispatch_support(a, support, npol_t, nblocks, as_stream(stream));
}

int av_tiled_plan_order_rows(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u, int64_t n_v,
                             int64_t n_img_chan, int support, void *workspace,
                             size_t workspace_bytes, void *stream) {
  clear_error();
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, 100, nt, nb, nchan, n_img_chan, workspace,
                             workspace_bytes, p, "av_tiled_plan_order_rows");
  if (rc) return rc;
  return plan_order_rows(g, p, as_stream(stream));
}

size_t av_grid_tiled_det_workspace_size(int64_t n_img_chan, int64_t n_img_pol, int64_t n_u,
                                        int64_t n_v) {
  const size_t cells = (size_t)(n_img_chan > 0 ? n_img_chan : 1) *
                       (size_t)(n_img_pol > 0 ? n_img_pol : 1) * (size_t)(n_u > 0 ? n_u : 1) *
                       (size_t)(n_v > 0 ? n_v : 1);
  const size_t planes = (size_t)(n_img_chan > 0 ? n_img_chan : 1) *
                        (size_t)(n_img_pol > 0 ? n_img_pol : 1);
  return Workspace::need(sizeof(unsigned long long) * 2 * cells) +
         Workspace::need(sizeof(unsigned long long) * planes) +
         Workspace::need(sizeof(unsigned long long) * 2) + Workspace::need(sizeof(double) * 2) +
         Workspace::need(sizeof(int) * 4);
}

int av_grid_tiled_execute_det(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                              const void *vis, int vis_dtype, const void *weight,
                              int weight_dtype, const int32_t *pol_map, const double *cgk,
                              int64_t n_u, int64_t n_v, int support, int oversampling, int64_t nt,
                              int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                              int64_t n_img_pol, void *workspace, size_t workspace_bytes,
                              void *det_workspace, size_t det_workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(grid && sum_weight && weight && pol_map && cgk && det_workspace,
               "av_grid_tiled_execute_det: null pointer");
  AV_CHECK_ARG(do_psf || vis, "av_grid_tiled_execute_det: vis is required unless do_psf");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_grid_tiled_execute_det: grid must be complex64 or complex128");
  AV_CHECK_ARG(do_psf || vis_dtype == AV_C64, "av_grid_tiled_execute_det: vis must be complex64");
  AV_CHECK_ARG(weight_dtype == AV_F32, "av_grid_tiled_execute_det: weight must be float32");
  AV_CHECK_ARG(npol >= 0 && npol <= 4 && n_img_pol >= 1 && n_img_pol <= 4,
               "av_grid_tiled_execute_det: npol and n_img_pol must be in [1, 4]");
  AV_CHECK_ARG(support >= 3 && support <= 8,
               "av_grid_tiled_execute_det: deterministic gridding covers supports 3-8");
  AV_CHECK_ARG((((uintptr_t)det_workspace) & 255) == 0,
               "av_grid_tiled_execute_det: det_workspace must be 256-byte aligned");
  const size_t need = av_grid_tiled_det_workspace_size(n_img_chan, n_img_pol, n_u, n_v);
  if (det_workspace_bytes < need) {
    set_error("av_grid_tiled_execute_det: det_workspace %zu bytes < %zu needed",
              det_workspace_bytes, need);
    return AV_ERR_WORKSPACE;
  }
  PlanGeom g;
  Plan p;
  int rc = grid_geom_checked(g, n_u, n_v, support, oversampling, nt, nb, nchan, n_img_chan,
                             workspace, workspace_bytes, p, "av_grid_tiled_execute_det");
  if (rc) return rc;
  int64_t rows = nt * nb * nchan;
  if (rows == 0 || npol == 0) return AV_OK;
  const int64_t cells = n_img_chan * n_img_pol * n_u * n_v, planes = n_img_chan * n_img_pol;
  Workspace dw(det_workspace, det_workspace_bytes);
  unsigned long long *qg = dw.take<unsigned long long>(2 * cells);
  unsigned long long *qw = dw.take<unsigned long long>(planes);
  unsigned long long *mx = dw.take<unsigned long long>(2);
  double *scale = dw.take<double>(2);
  int *err = dw.take<int>(4);
  cudaStream_t st = as_stream(stream);
  int npol_t = npol <= 1 ? 1 : (npol <= 2 ? 2 : 4);
  TiledGridArgs a;
  a.recs = p.recs;
  a.tile_start = p.tile_start;
  a.n_rec = p.offs + g.n_keys();
  a.n_tiles = g.n_tiles();
  a.ntu = g.ntu;
  a.ntv = g.ntv;
  int64_t nblocks = 0;
  a.chunk = grid_chunking(rows, nblocks);
  a.sched = p.counters;
  a.vis = (const float2 *)vis;
  a.wt = (const float *)weight;
  a.do_psf = do_psf;
  a.cgk = cgk;
  a.cgk_len = oversampling * (support / 2 + 1);
  a.os = oversampling;
  a.pol_map = pol_map;
  a.npol = (int)npol;
  a.npg = (int)n_img_pol;
  a.grid = grid;
  a.grid_c128 = grid_dtype == AV_C128;
  a.sumw = sum_weight;
  a.n_u = n_u;
  a.n_v = n_v;
  a.inv_norm = 0;
  a.flag = nullptr;
  a.det_grid = qg;
  a.det_sumw = qw;
  a.det_scale = scale;
  {
    const uintptr_t vp = (uintptr_t)vis, wp = (uintptr_t)weight;
    const bool v16 = do_psf || vp % 16 == 0;
    a.a16 = v16 && ((npol == 4 && wp % 16 == 0) || (npol == 2 && wp % 8 == 0));
  }
  AV_CUDA(cudaMemsetAsync(qg, 0, sizeof(unsigned long long) * (size_t)(2 * cells), st));
  AV_CUDA(cudaMemsetAsync(qw, 0, sizeof(unsigned long long) * (size_t)planes, st));
  AV_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long) * 2, st));
  const int sms = sm_count();
  k_det_bound<<<(unsigned)(sms * 4), 256, 0, st>>>(a, mx);
  AV_LAUNCH_CHECK();
  k_det_scale<<<1, 1, 0, st>>>(a.n_rec, mx, cgk, a.cgk_len, support, scale, err);
  AV_LAUNCH_CHECK();
  int host[2] = {0, 0};
  uint32_t ordered = 0;
  AV_CUDA(cudaMemcpyAsync(&host[0], err, sizeof(int), cudaMemcpyDeviceToHost, st));
  AV_CUDA(cudaMemcpyAsync(&ordered, p.counters + PLAN_ROWS_ORDERED, sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, st));
  AV_CUDA(cudaStreamSynchronize(st));
  if (ordered != 1u) {
    set_error("av_grid_tiled_execute_det: the plan's records are not ordered by row "
              "(av_tiled_plan_order_rows)");
    return AV_ERR_ARG;
  }
  if (host[0]) {
    set_error("av_grid_tiled_execute_det: an infinite weighted value or weight has no "
              "fixed-point sum");
    return AV_ERR_ARG;
  }
  if (npol_t == 1) rc = dispatch_det_npol<1>(a, support, nblocks, st);
  else if (npol_t == 2) rc = dispatch_det_npol<2>(a, support, nblocks, st);
  else rc = dispatch_det_npol<4>(a, support, nblocks, st);
  if (rc) return rc;
  int64_t fb = (cells + 255) / 256;
  if (fb > (int64_t)sms * 8) fb = (int64_t)sms * 8;
  if (fb < 1) fb = 1;
  k_det_finish<<<(unsigned)fb, 256, 0, st>>>(grid, a.grid_c128, qg, cells, sum_weight, qw, planes,
                                            scale);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// Adjoint of the tiled degridder on a degrid plan (av_degrid_tiled_plan):
// grid[c, p] += sum over unflagged samples of w_k / (sum_k w_k) * values,
// with the degridder's cells, offsets, channel and polarisation maps.
int av_degrid_tiled_adjoint(void *grid, int grid_dtype, const void *values, int values_dtype,
                            const uint8_t *flag, int64_t g_nchan, int64_t g_npol, int64_t g_n2,
                            int64_t g_n3, int support, int sampling, const double *convFunc,
                            const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                            int64_t nvpol, void *workspace, size_t workspace_bytes,
                            void *stream) {
  clear_error();
  AV_CHECK_ARG(grid && values && convFunc && polmap, "av_degrid_tiled_adjoint: null pointer");
  AV_CHECK_ARG(grid_dtype == AV_C64 || grid_dtype == AV_C128,
               "av_degrid_tiled_adjoint: grid dtype");
  AV_CHECK_ARG(values_dtype == AV_C64, "av_degrid_tiled_adjoint: values must be complex64");
  AV_CHECK_ARG(nvpol >= 1 && nvpol <= 4 && g_npol >= 1 && g_npol <= 4,
               "av_degrid_tiled_adjoint: polarisations must be in [1, 4]");
  AV_CHECK_ARG(support >= 3 && support <= 9 && sampling >= 1 && sampling <= 254,
               "av_degrid_tiled_adjoint: support / sampling out of range");
  AV_CHECK_ARG(workspace && (((uintptr_t)workspace) & 255) == 0,
               "av_degrid_tiled_adjoint: workspace must be 256-byte aligned");
  PlanGeom g;
  plan_geometry(g, nt, nb, nvchan, g_nchan > 0 ? g_nchan : 1, g_n2, g_n3, support, sampling);
  if (workspace_bytes < plan_workspace_bytes(g)) {
    set_error("av_degrid_tiled_adjoint: workspace too small");
    return AV_ERR_WORKSPACE;
  }
  Workspace ws(workspace, workspace_bytes);
  Plan p;
  if (!plan_carve(g, ws, p)) {
    set_error("av_degrid_tiled_adjoint: workspace carve failed");
    return AV_ERR_WORKSPACE;
  }
  int64_t rows = nt * nb * nvchan;
  if (rows == 0 || g_nchan == 0) return AV_OK;
  TiledGridArgs a;
  a.recs = p.recs;
  a.tile_start = p.tile_start;
  a.n_rec = p.offs + g.n_keys();
  a.n_tiles = g.n_tiles();
  a.ntu = g.ntu;
  a.ntv = g.ntv;
  int64_t nblocks = 0;
  a.chunk = grid_chunking(rows, nblocks);
  a.sched = p.counters;
  a.vis = (const float2 *)values;
  a.wt = nullptr;
  a.do_psf = 0;
  a.cgk = convFunc;
  a.cgk_len = sampling * (support / 2 + 1);
  a.os = sampling;
  a.pol_map = polmap;
  a.npol = (int)nvpol;
  a.npg = (int)g_npol;
  a.grid = grid;
  a.grid_c128 = grid_dtype == AV_C128;
  a.sumw = nullptr;
  a.n_u = g_n2;
  a.n_v = g_n3;
  a.inv_norm = 1;
  a.flag = flag;
  a.a16 = 0;
  int npol_t = nvpol <= 1 ? 1 : (nvpol <= 2 ? 2 : 4);
  return dispatch_support(a, support, npol_t, nblocks, as_stream(stream));
}

int av_grid_tiled(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                  const void *vis, int vis_dtype, const void *weight, int weight_dtype,
                  const double *uvw, const double *freq, const int32_t *chan_map,
                  const int32_t *pol_map, const double *cgk, int64_t n_u, int64_t n_v,
                  double delta_l, double delta_m, int support, int oversampling, int64_t nt,
                  int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                  int64_t n_img_pol, void *workspace, size_t workspace_bytes, void *stream) {
  int rc = av_grid_tiled_plan(uvw, freq, chan_map, n_u, n_v, delta_l, delta_m, support,
                              oversampling, nt, nb, nchan, n_img_chan, workspace,
                              workspace_bytes, stream);
  if (rc) return rc;
  return av_grid_tiled_execute(grid, grid_dtype, sum_weight, do_psf, vis, vis_dtype, weight,
                               weight_dtype, pol_map, cgk, n_u, n_v, support, oversampling, nt,
                               nb, nchan, npol, n_img_chan, n_img_pol, workspace,
                               workspace_bytes, stream);
}

}  // extern "C"
