// Binning plan shared by the tiled gridder and degridder.
//
// Every (time, baseline, channel) sample whose kernel footprint lies inside
// the grid becomes one 8-byte record, sorted by key
//   key = ((plane * ntu + tu) * ntv + tv) * KPT + cell-in-tile / R^2
// where (tu, tv) is the T x T tile holding the footprint's first cell
// (fu, fv), plane the image channel, and R the in-tile resolution of the key
// (1 = one key per cell; coarser only when planes x cells would exceed the
// key budget).  Sorting by cell makes samples that share a cell contiguous,
// which is what lets the gridder keep runs in registers and the degridder
// read its sub-grid by broadcast.
//
// The sort is a counting sort: count keys (warp-aggregated atomics), scan,
// scatter (warp-aggregated atomic cursors).  Order inside a key is the
// arrival order of the atomics.  Samples that are skipped (off the grid, NaN
// uvw, channel outside the image) go to one extra key, n_keys, after all
// tiles: offs[n_keys] counts the usable records and the rest of recs[] lists
// the skipped rows (a store-mode degrid writes zeros there).
//
// A shared plan (convention 2) serves the gridder and the degridder at once:
// records are sorted by the gridder's key (int(x + 0.5) rounding,
// standard_grid.py:337-352), and the samples whose cell, kernel offsets or
// bounds verdict differ under the degridder's half-even rounding
// (standard_degrid.py:435-462) are marked for it in a bitmap of record
// positions, exc_mark (the degridder writes zero there or skips them; the
// gridder never reads it), and those the degridder keeps are listed in
// exc_rows, which a small FP64 kernel degrids after the tiled one.  The degridder's position is computed exactly only for samples near a
// rounding boundary (see sample_key_shared in plan.cu); elsewhere the two
// conventions provably agree.
#pragma once
#include "common.cuh"

namespace av {

constexpr int TILE = 32;                       // tile edge in cells
constexpr int PLAN_ROWS_ORDERED = 8;           // Plan::counters entry set by plan_order_rows
constexpr int ORD_WCAP = 1024;                 // records a warp orders by row (plan_order_rows)
constexpr int SCAN_MAX_BLOCKS = 65536;                    // scan partials
constexpr int64_t KEY_BUDGET = (int64_t(1) << 28) - 65536;  // scan capacity: 65536 x 4096 keys

// While a shared plan is built, the top bit of a walk-order record's row
// marks a sample whose degridder convention differs; the scatter pass moves
// the mark into exc_mark, so sorted records carry plain rows.
constexpr uint32_t REC_DEGRID_EXC = 0x80000000u;

// Whether sorted record r is marked for the degridder (exc_mark bit r).
__device__ __forceinline__ bool degrid_marked(const uint32_t *exc_mark, uint32_t r) {
  return (__ldg(exc_mark + (r >> 5)) >> (r & 31u)) & 1u;
}

struct __align__(8) Rec {
  uint32_t row;     // (t * nb + b) * nchan + c
  uint8_t du, dv;   // footprint start inside the tile (cells)
  uint8_t ou, ov;   // kernel offsets + 128
};

// Tile of record r: the largest t in [0, n_tiles) with ts[t] <= r (ts[0] =
// 0 <= r < ts[n_tiles]), searched by the calling warp 32 ways at a time: each
// step probes 32 positions at once, so a plan of 4096 tiles takes 3
// dependent loads instead of 12.  Every lane of the warp calls it, converged,
// with the same r, and every lane gets the result.
__device__ __forceinline__ int find_tile_warp(const uint32_t *ts, int64_t n_tiles, uint32_t r) {
  const int lane = threadIdx.x & 31;
  int64_t lo = 0, hi = n_tiles;  // ts[lo] <= r < ts[hi]
  while (hi - lo > 1) {
    const int64_t step = (hi - lo + 31) / 32;
    const int64_t p = lo + (int64_t)(lane + 1) * step;
    const bool le = p < hi && ts[p] <= r;
    // ts does not decrease, so the probes at or below r are a prefix of lanes
    const int cnt = __popc(__ballot_sync(0xffffffffu, le));
    lo += (int64_t)cnt * step;
    hi = min(hi, lo + step);
  }
  return (int)lo;
}

struct PlanGeom {
  int64_t n_rows;            // nt * nb * nchan
  int64_t nb_nchan;          // nb * nchan (rows per time step)
  int64_t nt, nb;
  int64_t nchan;
  int64_t n_planes;          // image channels
  int64_t n_u, n_v;          // grid extent of axes 2 and 3
  int64_t ntu, ntv;          // tiles per axis
  int64_t kpt;               // keys per tile
  int res_shift;             // log2(R)
  int support, os;
  // gridder convention: a sample is kept when its centre cell is at least
  // `margin` cells from both grid edges (support / 2 for standard_grid_jit;
  // np.max(weight_support) for mosaic_grid_jit, mosaic_grid.py:398-403)
  int margin;
  int convention;            // 0 = gridder (standard_grid.py), 1 = degridder,
                             // 2 = shared (gridder order, degridder exceptions)
  // degridder only: the reference's own bounds extents and the scale/offset
  int64_t chk_x, chk_y;      // nx = shape[3], ny = shape[2] (standard_degrid.py:407)
  double scale0, scale1, offset0, offset1;
  __host__ __device__ int64_t n_tiles() const { return n_planes * ntu * ntv; }
  __host__ __device__ int64_t n_keys() const { return n_tiles() * kpt; }
};

// Fill the tile / key geometry for a grid of (n_planes, n_u, n_v).
inline void plan_geometry(PlanGeom &g, int64_t nt, int64_t nb, int64_t nchan,
                          int64_t n_planes, int64_t n_u, int64_t n_v, int support, int os) {
  g.n_rows = nt * nb * nchan;
  g.nb_nchan = nb * nchan;
  g.nt = nt;
  g.nb = nb;
  g.nchan = nchan;
  g.n_planes = n_planes;
  g.n_u = n_u;
  g.n_v = n_v;
  int64_t span_u = n_u - support + 1, span_v = n_v - support + 1;
  if (span_u < 1) span_u = 1;
  if (span_v < 1) span_v = 1;
  g.ntu = (span_u + TILE - 1) / TILE;
  g.ntv = (span_v + TILE - 1) / TILE;
  g.support = support;
  g.os = os;
  g.margin = support / 2;
  g.res_shift = 0;
  while (g.res_shift < 5 &&
         g.n_planes * g.ntu * g.ntv * ((int64_t)(TILE >> g.res_shift) * (TILE >> g.res_shift)) >
             KEY_BUDGET)
    g.res_shift++;
  int64_t side = TILE >> g.res_shift;
  g.kpt = side * side;
}

inline size_t plan_workspace_bytes(const PlanGeom &g) {
  size_t b = 0;
  b += Workspace::need(sizeof(uint32_t) * (g.n_keys() + 2));  // offsets
  b += Workspace::need(sizeof(uint32_t) * (g.n_keys() + 2));  // cursors
  b += Workspace::need(sizeof(uint32_t) * (g.n_tiles() + 1)); // tile starts
  b += Workspace::need(sizeof(Rec) * (g.n_rows > 0 ? g.n_rows : 1));
  b += Workspace::need(sizeof(double) * 2 * (g.nchan > 0 ? g.nchan : 1));
  b += Workspace::need(sizeof(uint32_t) * SCAN_MAX_BLOCKS);    // scan partials
  b += Workspace::need(sizeof(uint32_t) * 16);                 // counters
  const size_t nr = g.n_rows > 0 ? (size_t)g.n_rows : 1;
  b += Workspace::need(sizeof(uint32_t) * nr);                 // keys in walk order
  b += Workspace::need(sizeof(Rec) * nr);                      // records in walk order
  // degridder exceptions of a shared plan (count, rows) and what their
  // kernel needs: u, v per (time, baseline), frequencies, channel map and
  // the degridder's scale / offset
  const size_t ntb = g.nt * g.nb > 0 ? (size_t)(g.nt * g.nb) : 1;
  const size_t nc = g.nchan > 0 ? (size_t)g.nchan : 1;
  b += Workspace::need(sizeof(uint32_t) * 4);
  b += Workspace::need(sizeof(uint32_t) * nr);
  b += Workspace::need(sizeof(uint32_t) * (nr / 32 + 2));     // exc_mark
  b += Workspace::need(sizeof(uint32_t) * 4);                 // keys too long for a warp
  b += Workspace::need(sizeof(uint32_t) * (nr / (ORD_WCAP + 1) + 2));  // their list
  b += Workspace::need(sizeof(double2) * ntb);
  b += Workspace::need(sizeof(double) * nc);
  b += Workspace::need(sizeof(int32_t) * nc);
  b += Workspace::need(sizeof(double) * 4);
  return b;
}

struct Plan {
  uint32_t *offs;      // n_keys + 2: start of each key (exclusive scan); the
                       // last key (n_keys) holds the skipped samples
  uint32_t *cursor;    // n_keys + 2
  uint32_t *tile_start;// n_tiles + 1
  Rec *recs;           // n_rows (only the first n_rec are used)
  double *scale;       // 2 * nchan: per-channel uv scale (gridder convention)
  uint32_t *scan_tmp;
  uint32_t *counters;  // 16, zero after a build: [0..1] the gridders' chunk schedule,
                       // [2..3] the degridder's, [PLAN_ROWS_ORDERED] plan_order_rows ran
  uint32_t *walk_key;  // n_rows: key of each sample in walk order (pass 1)
  Rec *walk_rec;       // n_rows: record of each sample in walk order (pass 1)
  uint32_t *exc_count; // [0]: degridder exceptions listed (0 unless shared)
  uint32_t *exc_rows;  // n_rows: their rows
  uint32_t *exc_mark;  // bit per sorted record: the degridder must not use it
  uint32_t *n_big;     // [0]: keys listed in big (row-order pass)
  uint32_t *big;       // keys too long for one warp to order by row
  double2 *uv;         // nt * nb: u, v of each (time, baseline) (shared only)
  double *freq;        // nchan (shared only)
  int32_t *chan_map;   // nchan (shared only)
  double *dpar;        // scale0, scale1, offset0, offset1 (shared only)
};

// Margins that make the gridder's and the degridder's roundings agree (see
// sample_key_shared in plan.cu): the two FP64 positions of a sample differ
// by less than 1e-10 cells, its kernel-offset arguments by less than 3e-8.
constexpr double CELL_SLACK = 1e-7, OFFSET_SLACK = 1e-5;

// Whether x - k (x in [k, k + 1)) lies more than `slack` from both k and k + 1.
__device__ __forceinline__ bool clear_of_integers(double frac, double slack) {
  return frac > slack && frac < 1.0 - slack;
}

// Position of one sample in the gridder's convention (standard_grid.py:
// 297-352): returns false when it is skipped.  fu/fv = first footprint cell.
// ui = int(u_pos + 0.5) truncates; a kept sample has margin <= ui < n_u -
// margin, which for margin >= 1 is margin <= u_pos + 0.5 < n_u - margin (for
// margin 0 the lower bound is -1 < u_pos + 0.5), so the range is tested in
// FP64 (NaN fails it) and only kept values are converted, to 32 bits.  The
// offsets floor((ui - u_pos) * os + 0.5) convert once, rounding down.  With
// `safe`, also whether all four rounded quantities (the cells' and the
// offsets' arguments) lie more than CELL_SLACK / OFFSET_SLACK from a rounding
// boundary, read from the fractional parts at hand.
__device__ __forceinline__ bool sample_pos_grid(double um, double vm, double us0, double us1,
                                                int64_t n_u, int64_t n_v, int support, int os,
                                                int margin, int &fu, int &fv, int &offu,
                                                int &offv, bool *safe = nullptr) {
  const double u = __dmul_rn(um, us0), v = __dmul_rn(vm, us1);
  const double u_pos = __dadd_rn(u, (double)(n_u / 2));
  const double v_pos = __dadd_rn(v, (double)(n_v / 2));
  const double au = __dadd_rn(u_pos, 0.5), av = __dadd_rn(v_pos, 0.5);
  const double lo = margin > 0 ? (double)margin : -1.0;
  const bool in_u = (margin > 0 ? au >= lo : au > lo) && au < (double)(n_u - margin);
  const bool in_v = (margin > 0 ? av >= lo : av > lo) && av < (double)(n_v - margin);
  if (!(in_u && in_v)) return false;
  const int ui = __double2int_rz(au), vi = __double2int_rz(av);
  const double dui = (double)ui, dvi = (double)vi;
  const double uo = __dsub_rn(dui, u_pos), vo = __dsub_rn(dvi, v_pos);
  const double bu = __dadd_rn(__dmul_rn(uo, (double)os), 0.5);
  const double bv = __dadd_rn(__dmul_rn(vo, (double)os), 0.5);
  offu = __double2int_rd(bu);
  offv = __double2int_rd(bv);
  const int sc = support / 2;
  fu = ui - sc;
  fv = vi - sc;
  if (safe)
    *safe = clear_of_integers(__dsub_rn(au, dui), CELL_SLACK) &&
            clear_of_integers(__dsub_rn(av, dvi), CELL_SLACK) &&
            clear_of_integers(__dsub_rn(bu, (double)offu), OFFSET_SLACK) &&
            clear_of_integers(__dsub_rn(bv, (double)offv), OFFSET_SLACK);
  return true;
}

// Position in the degridder's convention (standard_degrid.py:435-462):
// np.round (half to even), loc/off stored as int32, bounds against the
// reference's nx = shape[3], ny = shape[2] and the true extents.
__device__ __forceinline__ bool sample_pos_degrid(double um, double vm, double freq,
                                                  const PlanGeom &g, int &fu, int &fv,
                                                  int &offu, int &offv) {
  const double c = C_LIGHT;
  double p0 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(g.scale0, um), freq), c), g.offset0);
  double p1 = __dadd_rn(__ddiv_rn(__dmul_rn(__dmul_rn(g.scale1, vm), freq), c), g.offset1);
  int x0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p0));
  int y0 = (int)(unsigned)(unsigned long long)trunc_ll(rint(p1));
  int o0 = (int)(unsigned)(unsigned long long)trunc_ll(
      rint(__dmul_rn(__dsub_rn((double)x0, p0), (double)g.os)));
  int o1 = (int)(unsigned)(unsigned long long)trunc_ll(
      rint(__dmul_rn(__dsub_rn((double)y0, p1), (double)g.os)));
  long long beg = -(g.support / 2), end = beg + g.support;
  long long X0 = x0, Y0 = y0;
  if (!((X0 + beg >= 0) && (X0 + end - 1 < g.chk_x) && (Y0 + beg >= 0) &&
        (Y0 + end - 1 < g.chk_y)))
    return false;
  if (!(X0 + end - 1 < g.n_u && Y0 + end - 1 < g.n_v)) return false;
  fu = (int)(X0 + beg);
  fv = (int)(Y0 + beg);
  offu = o0;
  offv = o1;
  return true;
}

// Host: enqueue the plan build for uvw / freq / chan_map (plane per channel;
// entries outside [0, n_planes) drop the channel).  Nothing is synchronised:
// the record count stays on the device in offs[n_keys] (and a shared plan's
// exception count in exc_count[0]).  A shared plan (g.convention == 2) needs
// the degridder's scale / offset / bounds extents in g as well as the
// gridder's cell size (delta_l, delta_m).
// With drop_wt (float32 weights, drop_npol per sample), samples whose every
// weight is zero or NaN are left out of the records (gridder convention).
int plan_build(const PlanGeom &g, Plan &p, const double *uvw, const double *freq,
               const int32_t *chan_map, double delta_l, double delta_m, cudaStream_t st,
               const float *drop_wt = nullptr, int drop_npol = 0);

// Orders each key's records by row (deterministic gridding); the degridder
// marks of a shared plan move with their records.
int plan_order_rows(const PlanGeom &g, const Plan &p, cudaStream_t st);

// Zeroes the grid cells the plan's records can touch (every non-empty tile's
// footprint region, all npg grid polarisations).
int plan_clear_tiles(const PlanGeom &g, const Plan &p, void *grid, int grid_c128, int64_t npg,
                     cudaStream_t st);

// Carve a Plan out of the workspace.
bool plan_carve(const PlanGeom &g, Workspace &ws, Plan &p);

}  // namespace av
