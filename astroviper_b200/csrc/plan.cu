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

// Key and record of sample (t, b, c).  The passes walk (baseline, channel)
// series with a warp each, 32 consecutive time steps at a time: those fall in
// one or a few cells, so the per-key atomics aggregate.
__device__ __forceinline__ bool sample_key(const PlanGeom &g, const double *uvw,
                                           const double *freq, const double *scale,
                                           const int32_t *chan_map, int64_t t, int64_t b,
                                           int c, uint32_t &key, Rec &rec) {
  const int64_t nb = g.nb;
  const int64_t tb = t * nb + b;
  const int64_t row = tb * g.nchan + c;
  rec.row = (uint32_t)row;
  rec.du = rec.dv = rec.ou = rec.ov = 0;
  key = (uint32_t)g.n_keys();  // skipped samples
  int plane = chan_map[c];
  if (plane < 0 || plane >= g.n_planes) return false;
  double um = uvw[3 * tb + 0], vm = uvw[3 * tb + 1];
  int fu, fv, ou, ov;
  bool ok;
  if (g.convention == 0)
    ok = sample_pos_grid(um, vm, scale[2 * c], scale[2 * c + 1], g.n_u, g.n_v, g.support, g.os,
                         fu, fv, ou, ov);
  else
    ok = sample_pos_degrid(um, vm, freq[c], g, fu, fv, ou, ov);
  if (!ok) return false;
  int tu = fu / TILE, tv = fv / TILE;
  int du = fu - tu * TILE, dv = fv - tv * TILE;
  int64_t tile = ((int64_t)plane * g.ntu + tu) * g.ntv + tv;
  int side_shift = 5 - g.res_shift;  // log2(TILE >> res_shift)
  int64_t cell = ((int64_t)(du >> g.res_shift) << side_shift) + (dv >> g.res_shift);
  key = (uint32_t)(tile * g.kpt + cell);
  rec.du = (uint8_t)du;
  rec.dv = (uint8_t)dv;
  rec.ou = (uint8_t)(ou + 128);
  rec.ov = (uint8_t)(ov + 128);
  return true;
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

// Pass 1: key and record of every sample, stored in walk order (sample
// index series * nt + t), and the count per key (warp-aggregated).  Warp w
// takes series w, w + n_warps, ... (series = b * nchan + c); the loops' trip
// counts are the same on every lane of a warp.
__global__ void __launch_bounds__(256) k_plan_count(PlanGeom g, const double *uvw,
                                                    const double *freq, const double *scale,
                                                    const int32_t *chan_map, uint32_t *hist,
                                                    uint32_t *walk_key, Rec *walk_rec) {
  const int lane = threadIdx.x & 31;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t n_series = g.nb * g.nchan;
  for (int64_t sr = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; sr < n_series;
       sr += n_warps) {
    const int64_t b = sr / g.nchan;
    const int c = (int)(sr - b * g.nchan);
    for (int64_t t0 = 0; t0 < g.nt; t0 += 32) {
      const int64_t t = t0 + lane;
      uint32_t key = 0xffffffffu;
      Rec rec;
      const bool in = t < g.nt;
      if (in) {
        sample_key(g, uvw, freq, scale, chan_map, t, b, c, key, rec);
        walk_key[sr * g.nt + t] = key;
        walk_rec[sr * g.nt + t] = rec;
      }
      uint32_t len;
      const bool lead = run_leader(key, in, lane, len);
      if (lead) atomicAdd(&hist[key], len);
    }
  }
}

// Pass 2: scatter the stored records to their key ranges (the same walk, so
// the same warp aggregation; no position arithmetic).
__global__ void __launch_bounds__(256) k_plan_scatter(PlanGeom g, const uint32_t *walk_key,
                                                      const Rec *walk_rec, uint32_t *cursor,
                                                      Rec *recs) {
  const int lane = threadIdx.x & 31;
  const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t n_series = g.nb * g.nchan;
  for (int64_t sr = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; sr < n_series;
       sr += n_warps) {
    for (int64_t t0 = 0; t0 < g.nt; t0 += 32) {
      const int64_t t = t0 + lane;
      const bool in = t < g.nt;
      uint32_t key = 0xffffffffu;
      Rec rec;
      if (in) {
        key = walk_key[sr * g.nt + t];
        rec = walk_rec[sr * g.nt + t];
      }
      uint32_t len;
      const bool lead = run_leader(key, in, lane, len);
      uint32_t pos = 0;
      if (lead) pos = atomicAdd(&cursor[key], len);
      // each lane's run leader: the highest leader at or below it
      const unsigned leaders = __ballot_sync(0xffffffffu, lead);
      const int ll = 31 - __clz(leaders & (0xffffffffu >> (31 - lane)));
      pos = __shfl_sync(0xffffffffu, pos, ll) + (uint32_t)(lane - ll);
      if (in) recs[pos] = rec;
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

// Tile starts, and the plan's scheduling counters set to zero (the tiled
// kernels take chunks from them and leave them at zero when they finish).
__global__ void k_tile_starts(const uint32_t *offs, int64_t n_tiles, int64_t kpt,
                              uint32_t *tile_start, uint32_t *counters) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < 16) counters[t] = 0u;
  if (t > n_tiles) return;
  tile_start[t] = offs[t * kpt];
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
  return p.offs && p.cursor && p.tile_start && p.recs && p.scale && p.scan_tmp &&
         p.counters && p.walk_key && p.walk_rec;
}

int plan_build(const PlanGeom &g, Plan &p, const double *uvw, const double *freq,
               const int32_t *chan_map, double delta_l, double delta_m, cudaStream_t st) {
  int64_t nk = g.n_keys();
  if (nk >= (int64_t)0xffffffffu || g.n_rows >= (int64_t)0xffffffffu) {
    set_error("plan: %lld keys / %lld samples exceed 32-bit indexing", (long long)nk,
              (long long)g.n_rows);
    return AV_ERR_UNSUPPORTED;
  }
  AV_CUDA(cudaMemsetAsync(p.cursor, 0, sizeof(uint32_t) * (nk + 2), st));
  if (g.nchan > 0) {
    k_chan_scale<<<(unsigned)((g.nchan + 127) / 128), 128, 0, st>>>(
        freq, g.nchan, delta_l, delta_m, g.n_u, g.n_v, p.scale);
    AV_LAUNCH_CHECK();
  }
  int sms = sm_count();
  // one warp per (baseline, channel) series, 8 warps per block
  int64_t blocks = (g.nb * g.nchan + 7) / 8;
  if (blocks > (int64_t)sms * 16) blocks = (int64_t)sms * 16;
  if (blocks < 1) blocks = 1;
  if (g.n_rows > 0) {
    k_plan_count<<<(unsigned)blocks, 256, 0, st>>>(g, uvw, freq, p.scale, chan_map, p.cursor,
                                                  p.walk_key, p.walk_rec);
    AV_LAUNCH_CHECK();
  }
  int rc = scan_counts(p.cursor, p.offs, nk + 1, p.scan_tmp, st);
  if (rc) return rc;
  if (g.n_rows > 0) {
    k_plan_scatter<<<(unsigned)blocks, 256, 0, st>>>(g, p.walk_key, p.walk_rec, p.cursor,
                                                    p.recs);
    AV_LAUNCH_CHECK();
  }
  int64_t nt = g.n_tiles() + 1;
  k_tile_starts<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(p.offs, g.n_tiles(), g.kpt,
                                                              p.tile_start, p.counters);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // namespace av
