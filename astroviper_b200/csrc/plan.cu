// Counting-sort plan of samples by uv cell (see plan.cuh).
#include "plan.cuh"

namespace av {

// Per-channel uv scale of the gridder: -(f * dl * n) / c (standard_grid.py:297-299).
__global__ void k_chan_scale(const double *freq, int64_t nchan, double dl0, double dl1,
                             int64_t n_u, int64_t n_v, double *scale) {
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nchan) return;
  double f = freq[c];
  scale[2 * c + 0] = __ddiv_rn(-__dmul_rn(__dmul_rn(f, dl0), (double)n_u), C_LIGHT);
  scale[2 * c + 1] = __ddiv_rn(-__dmul_rn(__dmul_rn(f, dl1), (double)n_v), C_LIGHT);
}

// Work units of the two passes: unit u = (baseline b, block of 32 time
// steps), lane = time step inside the block.  A warp takes units u, u +
// n_warps, ... and walks the unit's channels one after the other, so the
// uvw row is read once per unit and the 32 lanes of one channel hold
// consecutive time steps of one (baseline, channel) series: those fall in
// one or a few cells, so the per-key atomics aggregate.  Walk order (the
// index of the stored keys and records) is (b * nchan + c) * nt + t.  All
// indices fit 32 bits (plan_build checks n_keys and n_rows).
struct Unit {
  uint32_t b, t;  // baseline, this lane's time step
  bool in;        // t < nt
};

__device__ __forceinline__ Unit unit_of(uint32_t u, uint32_t ntb, uint32_t nt, int lane) {
  Unit w;
  w.b = u / ntb;
  w.t = (u - w.b * ntb) * 32u + (uint32_t)lane;
  w.in = w.t < nt;
  return w;
}

// Key and record (row | du | dv << 8 | (ou + 128) << 16 | (ov + 128) << 24
// in the second word, the byte layout of Rec) of one sample with uvw row
// (um, vm), channel c on image plane `plane`; skipped samples get key n_keys
// and a zero second word.
__device__ __forceinline__ uint32_t sample_key(const PlanGeom &g, double um, double vm,
                                               double us0, double us1, double f, int plane,
                                               uint32_t row, uint2 &rec) {
  rec = make_uint2(row, 0u);
  const uint32_t skip = (uint32_t)g.n_keys();
  if (plane < 0 || plane >= g.n_planes) return skip;
  int fu, fv, ou, ov;
  const bool ok = g.convention == 0
                      ? sample_pos_grid(um, vm, us0, us1, g.n_u, g.n_v, g.support, g.os,
                                        g.margin, fu, fv, ou, ov)
                      : sample_pos_degrid(um, vm, f, g, fu, fv, ou, ov);
  if (!ok) return skip;
  // fu, fv >= 0 here
  const uint32_t tu = (uint32_t)fu / TILE, tv = (uint32_t)fv / TILE;
  const uint32_t du = (uint32_t)fu - tu * TILE, dv = (uint32_t)fv - tv * TILE;
  const uint32_t tile = ((uint32_t)plane * (uint32_t)g.ntu + tu) * (uint32_t)g.ntv + tv;
  const int side_shift = 5 - g.res_shift;  // log2(TILE >> res_shift)
  const uint32_t cell = ((du >> g.res_shift) << side_shift) + (dv >> g.res_shift);
  rec.y = du | (dv << 8) | ((uint32_t)(ou + 128) << 16) | ((uint32_t)(ov + 128) << 24);
  return tile * (uint32_t)g.kpt + cell;
}

// Shared plan: the gridder's key and record of one sample, marked for the
// degridder.  When the gridder keeps the sample and all its rounded
// quantities lie clear of a rounding boundary (sample_pos_grid's `safe`),
// the degridder's half-even rounding of its own FP64 position (which differs
// from the gridder's by less than 1e-10 cells) gives the same cell and
// offsets, so only its bounds tests (against the reference's swapped
// extents, standard_degrid.py:457-462) are evaluated, in integers.
// Otherwise the degridder's position is computed exactly.  A record the
// degridder cannot use as it stands gets REC_DEGRID_EXC in its walk-order
// row (k_plan_scatter moves it to exc_mark); `exc` says the degridder keeps
// the sample, so it goes to the exception list.
__device__ __forceinline__ uint32_t sample_key_shared(const PlanGeom &g, double um, double vm,
                                                      double us0, double us1, double f,
                                                      int plane, uint32_t row, uint2 &rec,
                                                      bool &exc) {
  rec = make_uint2(row, 0u);
  exc = false;
  const uint32_t skip = (uint32_t)g.n_keys();
  if (plane < 0 || plane >= g.n_planes) return skip;  // neither convention maps the channel
  int fu, fv, ou, ov;
  bool safe = false;
  const bool ok = sample_pos_grid(um, vm, us0, us1, g.n_u, g.n_v, g.support, g.os, g.margin, fu,
                                  fv, ou, ov, &safe);
  bool dok, same;
  if (ok && safe) {
    const long long sc = g.support / 2, beg = -sc, end = beg + g.support;
    const long long X0 = (long long)fu + sc, Y0 = (long long)fv + sc;
    dok = (X0 + beg >= 0) && (X0 + end - 1 < g.chk_x) && (Y0 + beg >= 0) &&
          (Y0 + end - 1 < g.chk_y) && (X0 + end - 1 < g.n_u) && (Y0 + end - 1 < g.n_v);
    same = true;
  } else {
    int dfu, dfv, dou, dov;
    dok = sample_pos_degrid(um, vm, f, g, dfu, dfv, dou, dov);
    same = ok && dok && dfu == fu && dfv == fv && dou == ou && dov == ov;
  }
  if (!ok) {
    exc = dok;  // the gridder skips it, the degridder keeps it
    return skip;
  }
  const uint32_t tu = (uint32_t)fu / TILE, tv = (uint32_t)fv / TILE;
  const uint32_t du = (uint32_t)fu - tu * TILE, dv = (uint32_t)fv - tv * TILE;
  const uint32_t tile = ((uint32_t)plane * (uint32_t)g.ntu + tu) * (uint32_t)g.ntv + tv;
  const int side_shift = 5 - g.res_shift;
  const uint32_t cell = ((du >> g.res_shift) << side_shift) + (dv >> g.res_shift);
  rec.y = du | (dv << 8) | ((uint32_t)(ou + 128) << 16) | ((uint32_t)(ov + 128) << 24);
  if (!(same && dok)) {
    rec.x |= REC_DEGRID_EXC;
    exc = dok;
  }
  return tile * (uint32_t)g.kpt + cell;
}

// Warp aggregation of per-key atomics over runs of equal keys in lane order
// (a warp holds consecutive time steps of one series, so equal keys are
// adjacent).  Returns whether this lane leads a run and, for a leader, the
// run's length.  Lanes without a sample (in = false) form no run and end
// the previous one; they are always at the top of the warp.
__device__ __forceinline__ bool run_leader(uint32_t key, bool in, int lane, uint32_t &len) {
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool lead = in && (lane == 0 || prev != key);
  const unsigned leaders = __ballot_sync(0xffffffffu, lead);
  const unsigned valid = __ballot_sync(0xffffffffu, in);
  // next leader above this lane, else the end of the valid lanes
  const unsigned above = leaders & ~(0xffffffffu >> (31 - lane));
  const int end = above ? __ffs(above) - 1 : 32 - __clz(valid);
  len = (uint32_t)(end - lane);
  return lead;
}

// Pass 1: key and record of every sample, stored in walk order, and the
// count per key (warp-aggregated).  Loop trip counts are uniform per warp.
__global__ void __launch_bounds__(256) k_plan_count(PlanGeom g, const double *__restrict__ uvw,
                                                    const double *__restrict__ freq,
                                                    const double *__restrict__ scale,
                                                    const int32_t *__restrict__ chan_map,
                                                    uint32_t *hist, uint32_t *walk_key,
                                                    uint2 *walk_rec, uint32_t *exc_count,
                                                    uint32_t *exc_rows,
                                                    const float *__restrict__ drop_wt,
                                                    int drop_npol) {
  const int lane = threadIdx.x & 31;
  const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nt = (uint32_t)g.nt, nb = (uint32_t)g.nb, nchan = (uint32_t)g.nchan;
  const uint32_t ntb = (nt + 31u) >> 5;
  const uint32_t n_units = nb * ntb;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n_units; u += n_warps) {
    const Unit w = unit_of(u, ntb, nt, lane);
    const uint32_t tb = w.t * nb + w.b;  // uvw row (meaningful when in)
    double um = 0.0, vm = 0.0;
    if (w.in) {
      um = uvw[3 * (size_t)tb + 0];
      vm = uvw[3 * (size_t)tb + 1];
    }
    uint32_t widx = w.b * nchan * nt + w.t;
    // unrolled so the position arithmetic of several channels overlaps
#pragma unroll 4
    for (uint32_t c = 0; c < nchan; ++c, widx += nt) {
      const int plane = __ldg(chan_map + c);
      const double us0 = __ldg(scale + 2 * c), us1 = __ldg(scale + 2 * c + 1);
      const double f = __ldg(freq + c);
      uint32_t key = 0xffffffffu;
      if (w.in) {
        uint2 rec;
        if (g.convention == 2) {
          bool exc;
          key = sample_key_shared(g, um, vm, us0, us1, f, plane, tb * nchan + c, rec, exc);
          if (exc) exc_rows[atomicAdd(exc_count, 1u)] = tb * nchan + c;  // rare
        } else {
          key = sample_key(g, um, vm, us0, us1, f, plane, tb * nchan + c, rec);
          if (drop_wt != nullptr && key != (uint32_t)g.n_keys()) {
            // a sample whose every weight is zero or NaN adds nothing: the
            // reference skips zero and NaN weighted data (standard_grid.py:378)
            const float *wr = drop_wt + (size_t)(tb * nchan + c) * drop_npol;
            bool any = false;
            for (int p = 0; p < drop_npol; ++p) {
              const float x = wr[p];
              any |= (x == x) && x != 0.f;
            }
            if (!any) {
              key = (uint32_t)g.n_keys();
              rec = make_uint2(tb * nchan + c, 0u);
            }
          }
        }
        walk_key[widx] = key;
        walk_rec[widx] = rec;
      }
      uint32_t len;
      const uint32_t skip = (uint32_t)g.n_keys();
      const bool lead = run_leader(key, w.in, lane, len);
      if (lead && key != skip) atomicAdd(&hist[key], len);
      // skipped samples (any order will do): one count per warp, and none in
      // a gridder plan, which keeps no list of them - a weighted plan skips
      // every fully flagged sample, and counting those per run would put
      // millions of atomics on the one skip key
      const unsigned sm = __ballot_sync(0xffffffffu, w.in && key == skip);
      if (g.convention != 0 && sm != 0u && lane == __ffs(sm) - 1)
        atomicAdd(&hist[skip], (uint32_t)__popc(sm));
    }
  }
}

// Pass 2: scatter the stored records to their key ranges (the same walk and
// warp aggregation; no position arithmetic).  SC channels at a time, so that
// many cursor atomics are in flight per warp before their records are stored.
constexpr int SC = 4;

__global__ void __launch_bounds__(256) k_plan_scatter(PlanGeom g,
                                                      const uint32_t *__restrict__ walk_key,
                                                      const uint2 *__restrict__ walk_rec,
                                                      uint32_t *cursor, uint2 *recs,
                                                      uint32_t *exc_mark) {
  const int lane = threadIdx.x & 31;
  const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t nt = (uint32_t)g.nt, nb = (uint32_t)g.nb, nchan = (uint32_t)g.nchan;
  const uint32_t ntb = (nt + 31u) >> 5;
  const uint32_t n_units = nb * ntb;
  const unsigned below = 0xffffffffu >> (31 - lane);  // lanes 0..lane
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n_units; u += n_warps) {
    const Unit w = unit_of(u, ntb, nt, lane);
    const uint32_t wbase = w.b * nchan * nt + w.t;
    for (uint32_t c0 = 0; c0 < nchan; c0 += SC) {
      uint32_t key[SC], pos[SC];
      uint2 rec[SC];
      bool in[SC], lead[SC];
#pragma unroll
      for (int k = 0; k < SC; ++k) {
        in[k] = w.in && c0 + k < nchan;
        key[k] = 0xffffffffu;
        if (in[k]) {
          const uint32_t widx = wbase + (c0 + k) * nt;
          key[k] = walk_key[widx];
          rec[k] = walk_rec[widx];
        }
      }
      const uint32_t skip = (uint32_t)g.n_keys();
      unsigned smask[SC];
#pragma unroll
      for (int k = 0; k < SC; ++k) {
        uint32_t len;
        lead[k] = run_leader(key[k], in[k], lane, len);
        pos[k] = 0;
        if (lead[k] && key[k] != skip) pos[k] = atomicAdd(&cursor[key[k]], len);
        // skipped samples: one cursor atomic per warp (degridder and shared
        // plans; a gridder plan lists none)
        smask[k] = __ballot_sync(0xffffffffu, in[k] && key[k] == skip);
        if (g.convention != 0 && smask[k] != 0u && lane == __ffs(smask[k]) - 1)
          pos[k] = atomicAdd(&cursor[skip], (uint32_t)__popc(smask[k]));
      }
#pragma unroll
      for (int k = 0; k < SC; ++k) {
        // each lane's run leader: the highest leader at or below it; a
        // skipped sample's place follows the warp's first skipped lane
        const unsigned leaders = __ballot_sync(0xffffffffu, lead[k] && key[k] != skip);
        const int ll = 31 - __clz(leaders & below);
        const int sl = smask[k] != 0u ? __ffs(smask[k]) - 1 : 0;
        const uint32_t pr = __shfl_sync(0xffffffffu, pos[k], ll & 31) + (uint32_t)(lane - ll);
        const uint32_t ps = __shfl_sync(0xffffffffu, pos[k], sl) +
                            (uint32_t)__popc(smask[k] & (below >> 1));
        const bool is_skip = key[k] == skip;
        const uint32_t p = is_skip ? ps : pr;
        if (in[k] && (!is_skip || g.convention != 0)) {
          uint2 r = rec[k];
          if (g.convention == 2 && (r.x & REC_DEGRID_EXC)) {  // rare
            r.x &= ~REC_DEGRID_EXC;
            atomicOr(exc_mark + (p >> 5), 1u << (p & 31u));
          }
          recs[p] = r;
        }
      }
    }
  }
}

// --------------------------------------------------------------- scan ------
// Exclusive scan of n uint32 values in place into out (n + 1 entries; out[n]
// = total), three phases with 4096 items per block.
constexpr int SCAN_BLK = 1024, SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLK * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *sh,
                                                         uint32_t &total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  uint32_t warp_base = wid ? sh[wid - 1] : 0;
  uint32_t r = warp_base + x - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_BLK) k_scan_reduce(const uint32_t *in, int64_t n,
                                                          uint32_t *partial) {
  __shared__ uint32_t sh[32];
  int64_t base = blockIdx.x * (int64_t)SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k)
    if (base + k < n) s += in[base + k];
  uint32_t total;
  block_exclusive_scan(s, sh, total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_BLK) k_scan_partials(uint32_t *partial, int64_t np) {
  __shared__ uint32_t sh[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < np; base += SCAN_BLK) {
    int64_t i = base + threadIdx.x;
    uint32_t v = i < np ? partial[i] : 0;
    uint32_t total;
    uint32_t ex = block_exclusive_scan(v, sh, total);
    if (i < np) partial[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SCAN_BLK) k_scan_final(const uint32_t *in, int64_t n,
                                                         const uint32_t *partial,
                                                         uint32_t *out, uint32_t *out2) {
  __shared__ uint32_t sh[32];
  int64_t base = blockIdx.x * (int64_t)SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, sh, total) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) {
      out[base + k] = ex;
      out2[base + k] = ex;
    }
    ex += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) {
    out[n] = ex;
    out2[n] = ex;
  }
}

// Scan of counts held in `cursor` into offs (and a copy back into cursor to
// serve as the scatter cursors).
static int scan_counts(uint32_t *counts_then_cursor, uint32_t *offs, int64_t n,
                       uint32_t *tmp, cudaStream_t st) {
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb < 1) nb = 1;
  if (nb > SCAN_MAX_BLOCKS) {
    set_error("plan: key count %lld exceeds the scan capacity", (long long)n);
    return AV_ERR_UNSUPPORTED;
  }
  k_scan_reduce<<<(unsigned)nb, SCAN_BLK, 0, st>>>(counts_then_cursor, n, tmp);
  AV_LAUNCH_CHECK();
  k_scan_partials<<<1, SCAN_BLK, 0, st>>>(tmp, nb);
  AV_LAUNCH_CHECK();
  k_scan_final<<<(unsigned)nb, SCAN_BLK, 0, st>>>(counts_then_cursor, n, tmp, offs,
                                                   counts_then_cursor);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// ------------------------------------------------------------- row order ---
// For deterministic gridding (av_grid_tiled_execute_det): each key's records
// ordered by row, so the order in which a cell's samples are summed is a
// property of the data, not of the scatter pass's atomics.  Keys of up to
// ORD_WCAP records are sorted by one warp in shared memory, keys of up to
// ROW_BCAP (224 KiB of records) by one CTA in shared memory
// (k_plan_order_rows_big, from a list), longer ones by one CTA in place in
// global memory.  The sort is the bitonic
// network with every comparator ascending (each size-k merge first compares
// mirrored pairs), which sorts any n: a pair reaching past n would compare
// with a virtual +inf and is left alone.  A shared plan's degridder marks
// (exc_mark) follow their records: during the sort they ride in the top bit
// of du (a footprint start inside a tile, below TILE).
constexpr int ROW_WARPS = 8, ROW_BCAP = 28672, ROW_BTHREADS = 1024;
constexpr size_t ROW_SMEM = (size_t)ROW_WARPS * ORD_WCAP * sizeof(Rec);
constexpr size_t ROW_BSMEM = (size_t)ROW_BCAP * sizeof(Rec);
constexpr uint8_t ROW_MARK = 0x80;

__device__ __forceinline__ void row_cmpswap(Rec *x, uint32_t lo, uint32_t hi) {
  const Rec a = x[lo], b = x[hi];
  if (b.row < a.row) {
    x[lo] = b;
    x[hi] = a;
  }
}

// Sorts x[0, n) by row; threads tid = 0 .. nthr - 1 of a warp or CTA, `sync`
// between the network's stages.
template <typename Sync>
__device__ void bitonic_rows(Rec *x, uint32_t n, uint32_t tid, uint32_t nthr, Sync sync) {
  int lg = 0;  // N = 2^lg >= n
  while ((1u << lg) < n) ++lg;
  const uint32_t half = (1u << lg) >> 1;
  for (int lk = 1; lk <= lg; ++lk) {  // blocks of k = 2^lk
    const int lh = lk - 1;
    const uint32_t hm = (1u << lh) - 1u, k = 1u << lk;
    for (uint32_t i = tid; i < half; i += nthr) {  // mirrored pairs within blocks of k
      const uint32_t b = (i >> lh) << lk, o = i & hm;
      if (b + k - 1 - o < n) row_cmpswap(x, b + o, b + k - 1 - o);
    }
    sync();
    for (int lj = lk - 2; lj >= 0; --lj) {  // pairs at distance j = 2^lj
      const uint32_t jm = (1u << lj) - 1u, j = 1u << lj;
      for (uint32_t i = tid; i < half; i += nthr) {
        const uint32_t lo = ((i >> lj) << (lj + 1)) | (i & jm);
        if (lo + j < n) row_cmpswap(x, lo, lo + j);
      }
      sync();
    }
  }
}

// Record base + i with its degridder mark moved into du (the bitmap bit
// cleared), and back.
__device__ __forceinline__ Rec take_rec(const Rec *recs, uint32_t *exc_mark, uint32_t pos) {
  Rec r = recs[pos];
  const uint32_t bit = 1u << (pos & 31u);
  if (exc_mark[pos >> 5] & bit) {
    atomicAnd(exc_mark + (pos >> 5), ~bit);
    r.du |= ROW_MARK;
  }
  return r;
}

__device__ __forceinline__ void put_rec(Rec *recs, uint32_t *exc_mark, uint32_t pos, Rec r) {
  if (r.du & ROW_MARK) {
    r.du &= (uint8_t)~ROW_MARK;
    atomicOr(exc_mark + (pos >> 5), 1u << (pos & 31u));
  }
  recs[pos] = r;
}

__global__ void __launch_bounds__(ROW_WARPS * 32) k_plan_order_rows(const uint32_t *offs,
                                                                    int64_t n_keys, Rec *recs,
                                                                    uint32_t *exc_mark,
                                                                    uint32_t *big,
                                                                    uint32_t *n_big) {
  extern __shared__ __align__(16) unsigned char rsm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  Rec *buf = (Rec *)rsm + (size_t)wid * ORD_WCAP;
  const int64_t stride = (int64_t)gridDim.x * ROW_WARPS * 32;
  for (int64_t k0 = ((int64_t)blockIdx.x * ROW_WARPS + wid) * 32; k0 < n_keys; k0 += stride) {
    const int64_t k = k0 + lane;
    uint32_t lo = 0, n = 0;
    if (k < n_keys) {
      lo = offs[k];
      n = offs[k + 1] - lo;
    }
    if (n > (uint32_t)ORD_WCAP) big[atomicAdd(n_big, 1u)] = (uint32_t)k;
    unsigned todo = __ballot_sync(0xffffffffu, n >= 2 && n <= (uint32_t)ORD_WCAP);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t klo = __shfl_sync(0xffffffffu, lo, src);
      const uint32_t kn = __shfl_sync(0xffffffffu, n, src);
      for (uint32_t i = lane; i < kn; i += 32) buf[i] = take_rec(recs, exc_mark, klo + i);
      __syncwarp();
      bitonic_rows(buf, kn, (uint32_t)lane, 32u, []() { __syncwarp(); });
      for (uint32_t i = lane; i < kn; i += 32) put_rec(recs, exc_mark, klo + i, buf[i]);
      __syncwarp();
    }
  }
}

__global__ void __launch_bounds__(ROW_BTHREADS) k_plan_order_rows_big(const uint32_t *offs,
                                                                      Rec *recs,
                                                                      uint32_t *exc_mark,
                                                                      const uint32_t *big,
                                                                      const uint32_t *n_big,
                                                                      uint32_t *plan_counters) {
  extern __shared__ __align__(16) unsigned char rsm[];
  Rec *buf = (Rec *)rsm;
  const uint32_t nb = *n_big;
  // the plan's counters[PLAN_ROWS_ORDERED] records that its records are
  // ordered by row (the plan build zeroes it); read once this launch is done
  if (blockIdx.x == 0 && threadIdx.x == 0) plan_counters[PLAN_ROWS_ORDERED] = 1u;
  for (uint32_t it = blockIdx.x; it < nb; it += gridDim.x) {
    const uint32_t k = big[it];
    const uint32_t lo = offs[k], n = offs[k + 1] - lo;
    const bool in_smem = n <= (uint32_t)ROW_BCAP;  // uniform over the CTA
    if (in_smem) {
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        buf[i] = take_rec(recs, exc_mark, lo + i);
      __syncthreads();
      bitonic_rows(buf, n, threadIdx.x, blockDim.x, []() { __syncthreads(); });
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        put_rec(recs, exc_mark, lo + i, buf[i]);
    } else {
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        recs[lo + i] = take_rec(recs, exc_mark, lo + i);
      __syncthreads();
      bitonic_rows(recs + lo, n, threadIdx.x, blockDim.x, []() {
        __threadfence_block();
        __syncthreads();
      });
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        put_rec(recs, exc_mark, lo + i, recs[lo + i]);
    }
    __syncthreads();
  }
}

int plan_order_rows(const PlanGeom &g, const Plan &p, cudaStream_t st) {
  static bool configured[64] = {false};
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    AV_CUDA(cudaFuncSetAttribute(k_plan_order_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ROW_SMEM));
    AV_CUDA(cudaFuncSetAttribute(k_plan_order_rows_big,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROW_BSMEM));
    configured[dev] = true;
  }
  const int64_t nk = g.n_keys();
  const int sms = sm_count();
  AV_CUDA(cudaMemsetAsync(p.n_big, 0, sizeof(uint32_t), st));
  int64_t blocks = (nk + ROW_WARPS * 32 - 1) / (ROW_WARPS * 32);
  if (blocks > (int64_t)sms * 3) blocks = (int64_t)sms * 3;
  k_plan_order_rows<<<(unsigned)blocks, ROW_WARPS * 32, ROW_SMEM, st>>>(p.offs, nk, p.recs,
                                                                       p.exc_mark, p.big,
                                                                       p.n_big);
  AV_LAUNCH_CHECK();
  k_plan_order_rows_big<<<(unsigned)sms, ROW_BTHREADS, ROW_BSMEM, st>>>(p.offs, p.recs,
                                                                        p.exc_mark, p.big,
                                                                        p.n_big, p.counters);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

// Tile starts, and the plan's scheduling counters set to zero (the tiled
// kernels take chunks from them and leave them at zero when they finish).
__global__ void k_tile_starts(const uint32_t *offs, int64_t n_tiles, int64_t kpt,
                              uint32_t *tile_start, uint32_t *counters) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < 16) counters[t] = 0u;
  if (t > n_tiles) return;
  tile_start[t] = offs[t * kpt];
}

// Zeroes the cells a plan's records can touch: the (TILE + support - 1)^2
// footprint region of every tile that holds records, all grid polarisations
// (one CTA per tile; empty tiles return at once).  Neighbouring regions
// overlap; they all write zero.
__global__ void __launch_bounds__(256) k_clear_tiles(const uint32_t *tile_start, PlanGeom g,
                                                     void *grid, int grid_c128, int64_t npg) {
  const int64_t t = blockIdx.x;
  if (t >= g.n_tiles() || tile_start[t + 1] == tile_start[t]) return;
  const int64_t plane = t / (g.ntu * g.ntv);
  const int64_t trem = t - plane * g.ntu * g.ntv;
  const int64_t tu = trem / g.ntv, tv = trem - tu * g.ntv;
  const int W = TILE + g.support - 1;
  const int64_t n = (int64_t)W * W * npg;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int64_t gp = i / ((int64_t)W * W), cell = i - gp * W * W;
    const int64_t gu = tu * TILE + cell / W, gv = tv * TILE + cell % W;
    if (gu >= g.n_u || gv >= g.n_v) continue;
    const int64_t gi = ((plane * npg + gp) * g.n_u + gu) * g.n_v + gv;
    if (grid_c128) ((double2 *)grid)[gi] = make_double2(0.0, 0.0);
    else ((float2 *)grid)[gi] = make_float2(0.f, 0.f);
  }
}

int plan_clear_tiles(const PlanGeom &g, const Plan &p, void *grid, int grid_c128, int64_t npg,
                     cudaStream_t st) {
  if (g.n_tiles() == 0) return AV_OK;
  k_clear_tiles<<<(unsigned)g.n_tiles(), 256, 0, st>>>(p.tile_start, g, grid, grid_c128, npg);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

bool plan_carve(const PlanGeom &g, Workspace &ws, Plan &p) {
  p.offs = ws.take<uint32_t>(g.n_keys() + 2);
  p.cursor = ws.take<uint32_t>(g.n_keys() + 2);
  p.tile_start = ws.take<uint32_t>(g.n_tiles() + 1);
  p.recs = ws.take<Rec>(g.n_rows > 0 ? g.n_rows : 1);
  p.scale = ws.take<double>(2 * (g.nchan > 0 ? g.nchan : 1));
  p.scan_tmp = ws.take<uint32_t>(SCAN_MAX_BLOCKS);
  p.counters = ws.take<uint32_t>(16);
  p.walk_key = ws.take<uint32_t>(g.n_rows > 0 ? g.n_rows : 1);
  p.walk_rec = ws.take<Rec>(g.n_rows > 0 ? g.n_rows : 1);
  p.exc_count = ws.take<uint32_t>(4);
  p.exc_rows = ws.take<uint32_t>(g.n_rows > 0 ? g.n_rows : 1);
  p.exc_mark = ws.take<uint32_t>((g.n_rows > 0 ? g.n_rows : 1) / 32 + 2);
  p.n_big = ws.take<uint32_t>(4);
  p.big = ws.take<uint32_t>((g.n_rows > 0 ? g.n_rows : 1) / (ORD_WCAP + 1) + 2);
  p.uv = ws.take<double2>(g.nt * g.nb > 0 ? g.nt * g.nb : 1);
  p.freq = ws.take<double>(g.nchan > 0 ? g.nchan : 1);
  p.chan_map = ws.take<int32_t>(g.nchan > 0 ? g.nchan : 1);
  p.dpar = ws.take<double>(4);
  return p.offs && p.cursor && p.tile_start && p.recs && p.scale && p.scan_tmp &&
         p.counters && p.walk_key && p.walk_rec && p.exc_count && p.exc_rows && p.exc_mark &&
         p.n_big && p.big && p.uv &&
         p.freq && p.chan_map && p.dpar;
}

// What the exception kernel of a shared plan reads: u, v of every (time,
// baseline), the frequencies, the channel map and the degridder's scale /
// offset (so the plan stands on its own after the caller's arrays change).
__global__ void k_shared_copy(const double *uvw, int64_t ntb, const double *freq,
                              const int32_t *chan_map, int64_t nchan, double s0, double s1,
                              double o0, double o1, double2 *uv, double *fcopy, int32_t *ccopy,
                              double *dpar) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < ntb) uv[i] = make_double2(uvw[3 * i], uvw[3 * i + 1]);
  if (i < nchan) {
    fcopy[i] = freq[i];
    ccopy[i] = chan_map[i];
  }
  if (i == 0) {
    dpar[0] = s0;
    dpar[1] = s1;
    dpar[2] = o0;
    dpar[3] = o1;
  }
}

int plan_build(const PlanGeom &g, Plan &p, const double *uvw, const double *freq,
               const int32_t *chan_map, double delta_l, double delta_m, cudaStream_t st,
               const float *drop_wt, int drop_npol) {
  int64_t nk = g.n_keys();
  if (nk >= (int64_t)0xffffffffu || g.n_rows >= (int64_t)0xffffffffu) {
    set_error("plan: %lld keys / %lld samples exceed 32-bit indexing", (long long)nk,
              (long long)g.n_rows);
    return AV_ERR_UNSUPPORTED;
  }
  if (g.convention == 2 && g.n_rows >= (int64_t)REC_DEGRID_EXC) {
    set_error("plan: %lld samples exceed a shared plan's 31-bit rows", (long long)g.n_rows);
    return AV_ERR_UNSUPPORTED;
  }
  AV_CUDA(cudaMemsetAsync(p.cursor, 0, sizeof(uint32_t) * (nk + 2), st));
  AV_CUDA(cudaMemsetAsync(p.exc_count, 0, sizeof(uint32_t) * 4, st));
  AV_CUDA(cudaMemsetAsync(p.exc_mark, 0,
                          sizeof(uint32_t) * ((g.n_rows > 0 ? g.n_rows : 1) / 32 + 2), st));
  if (g.convention == 2) {
    const int64_t n = std::max<int64_t>(g.nt * g.nb, g.nchan);
    if (n > 0) {
      k_shared_copy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
          uvw, g.nt * g.nb, freq, chan_map, g.nchan, g.scale0, g.scale1, g.offset0, g.offset1,
          p.uv, p.freq, p.chan_map, p.dpar);
      AV_LAUNCH_CHECK();
    }
  }
  if (g.nchan > 0) {
    k_chan_scale<<<(unsigned)((g.nchan + 127) / 128), 128, 0, st>>>(
        freq, g.nchan, delta_l, delta_m, g.n_u, g.n_v, p.scale);
    AV_LAUNCH_CHECK();
  }
  int sms = sm_count();
  // one warp per (baseline, 32 time steps) unit, 8 warps per block
  int64_t blocks = (g.nb * ((g.nt + 31) / 32) + 7) / 8;
  if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
  if (blocks < 1) blocks = 1;
  if (g.n_rows > 0) {
    k_plan_count<<<(unsigned)blocks, 256, 0, st>>>(g, uvw, freq, p.scale, chan_map, p.cursor,
                                                  p.walk_key, (uint2 *)p.walk_rec,
                                                  p.exc_count, p.exc_rows, drop_wt, drop_npol);
    AV_LAUNCH_CHECK();
  }
  int rc = scan_counts(p.cursor, p.offs, nk + 1, p.scan_tmp, st);
  if (rc) return rc;
  if (g.n_rows > 0) {
    k_plan_scatter<<<(unsigned)blocks, 256, 0, st>>>(g, p.walk_key, (const uint2 *)p.walk_rec,
                                                    p.cursor, (uint2 *)p.recs, p.exc_mark);
    AV_LAUNCH_CHECK();
  }
  int64_t nt = g.n_tiles() + 1;
  k_tile_starts<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(p.offs, g.n_tiles(), g.kpt,
                                                              p.tile_start, p.counters);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // namespace av
