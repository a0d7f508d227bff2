// Hogbom CLEAN minor cycle (hclean::clean, hclean.cpp:106-210) and maximg
// (hclean.cpp:51-81) on one GPU.
//
// One cooperative persistent launch runs many iterations.  Every CTA owns a
// contiguous band of residual rows; when the band fits, it stays in shared
// memory for the whole launch.  Each iteration a CTA subtracts the scaled PSF
// from its band (where the PSF window covers it) and, in the same pass, finds
// the band's largest |r| inside the clean box (first maximum in row-major
// order wins, as the reference's strict '>').  CTAs publish one candidate
// each, meet at a grid barrier with a bounded wait, and every CTA reduces the
// candidates identically, so all of them agree on the next peak and on when
// to stop.  Arithmetic matches the reference bit for bit: products and
// differences are rounded separately (no FMA), the model is accumulated in
// iteration order by one thread.
#include <algorithm>
#include <cstddef>
#include <type_traits>

#include "common.cuh"

namespace av {

struct __align__(16) HogState {
  int iter;      // next iteration
  int px, py;    // current peak
  int stopped;   // 1: threshold reached
  int err;       // device error (1 = barrier timeout)
  unsigned gen;  // barrier generation
  unsigned count;
  int pad;
  double peak;   // r[py, px] for iteration `iter`
  double absval; // |peak| found (0 when no pixel exceeded 0)
  // FP32: the iteration's winner as one 64-bit maximum over the CTAs, bits of
  // |r| above the complement of 2 * index + sign (0: no pixel above 0), two
  // of them used in turn; kpar: the one the next launch starts with
  double pad1[10];  // the keys on the second cache line, away from gen / count
  unsigned long long key[2];
  int kpar;
  int pad3;
  double pad2[13];
};
static_assert(sizeof(HogState) == 256, "state size");
static_assert(offsetof(HogState, key) == 128, "keys on their own cache line");

template <typename T>
struct __align__(16) HogCand {
  T absval;
  T val;
  T at_prev;      // r at the previous peak (owner CTA only)
  int idx;        // linear index of the band maximum (-1 none)
  int has_prev;
};

template <typename T>
struct HogArgs {
  T *model, *resid;
  const T *psf, *mask;
  int nx, ny, pnx, pny;
  int xbeg, xend, ybeg, yend;
  int niter, siter, iter_begin, iter_end;
  T gain, thres, speedup;
  HogState *state;
  HogCand<T> *cand;  // 2 x gridDim.x
  int init;
  int resident;
  unsigned long long timeout_ns;  // bounded wait at the grid barrier
};

__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float t_pow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double t_pow(double a, double b) { return pow(a, b); }

// (a_abs, a_idx) beats (b_abs, b_idx): larger |r|, then lower index.
template <typename T>
__device__ __forceinline__ bool beats(T aa, int ai, T ba, int bi) {
  if (ai < 0) return false;
  if (bi < 0) return true;
  return aa > ba || (aa == ba && ai < bi);
}

// Grid barrier with a bounded wait (timeout_ns of wall time, 2 s unless the
// AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US knob says otherwise); returns false on
// timeout and records it in the state.  Every CTA adds itself to the count
// exactly once per barrier, timed out or not, so the last one to arrive still
// releases the barrier and no CTA waits beyond its own bound.
// The last CTA to arrive clears *reset (if given) before releasing the others.
__device__ bool grid_barrier(HogState *st, int *s_flag, unsigned long long timeout_ns,
                             unsigned long long *reset = nullptr) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *vgen = &st->gen;
    unsigned g0 = *vgen;
    __threadfence();
    unsigned arrived = atomicAdd(&st->count, 1u);
    int ok = 1;
    if (arrived == gridDim.x - 1) {
      if (reset) atomicExch(reset, 0ull);
      atomicExch(&st->count, 0u);
      __threadfence();
      atomicAdd(&st->gen, 1u);
    } else {
      unsigned long long t0;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
      while (*vgen == g0) {
        __nanosleep(32);
        unsigned long long t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
        if (t1 - t0 > timeout_ns) {
          ok = 0;
          atomicExch(&st->err, 1);
          break;
        }
      }
    }
    __threadfence();
    *s_flag = ok && (((volatile int *)&st->err)[0] == 0);
  }
  __syncthreads();
  return *s_flag != 0;
}

constexpr int HOG_THREADS = 1024;
// band pass for images up to HOG_NPR * HOG_THREADS columns: a thread's
// columns are fixed, so whether the PSF window and the clean box cover them
// is decided once per iteration and per row, not per pixel
constexpr int HOG_NPR = 2;
constexpr int HOG_RB = 7;  // rows whose PSF values are loaded together
// candidates a lane loads at once in the reduction after the grid barrier
constexpr int HOG_CPL = 4;

template <typename T>
__global__ void __launch_bounds__(HOG_THREADS, 1) k_hogbom(HogArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ T s_abs[32], s_val[32];
  __shared__ int s_idx[32];
  __shared__ int s_flag;
  __shared__ T s_prev;
  __shared__ int s_use_key;
  constexpr bool KEYED = std::is_same<T, float>::value;
  const int G = gridDim.x, b = blockIdx.x;
  const int y_lo = (int)((long long)a.ny * b / G), y_hi = (int)((long long)a.ny * (b + 1) / G);
  const int nx = a.nx;
  T *band = a.resident ? (T *)smem : a.resid + (size_t)y_lo * nx;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  if (a.resident) {
    // one trip count per block: every warp reaches the next barrier converged
    for (int i0 = 0; i0 < (y_hi - y_lo) * nx; i0 += HOG_THREADS) {
      const int i = i0 + threadIdx.x;
      if (i < (y_hi - y_lo) * nx) band[i] = a.resid[(size_t)y_lo * nx + i];
    }
  }
  // current peak
  int px, py, it = a.iter_begin;
  T peak = (T)0, absval = (T)0;
  if (a.init) {
    px = 0;
    py = 0;
  } else {
    px = a.state->px;
    py = a.state->py;
    peak = (T)a.state->peak;
    absval = (T)a.state->absval;
  }
  __syncthreads();

  int par = a.init ? 0 : a.state->kpar;
  bool first = a.init != 0;
  bool stopped = false;
  for (;;) {
    T pv = (T)0;
    bool do_sub = false;
    if (!first) {
      if (it >= a.iter_end) break;
      T cthres = a.thres;
      if (a.speedup > (T)0) cthres = a.thres * t_pow((T)2, (T)(it - a.siter) / a.speedup);
      if (absval < cthres) {
        stopped = true;
        break;
      }
      pv = rn_mul(a.gain, peak);
      do_sub = true;
      if (b == 0 && threadIdx.x == 0) {
        size_t mi = (size_t)py * nx + px;
        a.model[mi] = rn_add(a.model[mi], pv);
      }
    }
    // PSF window (hclean.cpp:172-175 with the PSF's own half sizes)
    const int x1 = max(0, px - a.pnx / 2), y1 = max(0, py - a.pny / 2);
    const int x2 = min(nx - 1, px + a.pnx / 2 - 1), y2 = min(a.ny - 1, py + a.pny / 2 - 1);
    // subtract + band argmax
    T best_abs = (T)0;
    int best_idx = -1;
    T best_val = (T)0;
    const int npr = (nx + HOG_THREADS - 1) / HOG_THREADS;
    const int tpr4 = nx >> 2;  // FP32, 4 pixels per thread: threads per row
    if (std::is_same<T, float>::value && (nx & 3) == 0 && tpr4 > 0 && tpr4 <= HOG_THREADS &&
        HOG_THREADS % tpr4 == 0) {
      // thread t: columns c0 .. c0 + 3 of rows y_lo + t / tpr4, + rpp, ...
      const int rpp = HOG_THREADS / tpr4;
      const int c0 = (threadIdx.x % tpr4) * 4, rofs = threadIdx.x / tpr4;
      // which of the 4 columns the PSF window (with an existing PSF column)
      // and the clean box cover, once per iteration
      const int wlo = max(x1, px - a.pnx / 2), whi = min(x2, px + a.pnx / 2 - 1);
      unsigned wm = 0u, bm = 0u;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = c0 + j;
        if (do_sub && c >= wlo && c <= whi) wm |= 1u << j;
        if (c >= a.xbeg && c < a.xend) bm |= 1u << j;
      }
      const int pxo0 = a.pnx / 2 + c0 - px;  // PSF column of c0
      for (int iy = y_lo + rofs; iy < y_hi; iy += rpp) {
        const int psf_y = a.pny / 2 + iy - py;
        const bool rsub = wm != 0u && iy >= y1 && iy <= y2 && psf_y >= 0 && psf_y < a.pny;
        float *rp = (float *)band + (size_t)(iy - y_lo) * nx + c0;
        const float4 r4 = *(const float4 *)rp;
        float rr[4] = {r4.x, r4.y, r4.z, r4.w};
        if (rsub) {
          const float *pp = (const float *)a.psf + (size_t)psf_y * a.pnx + pxo0;
          float p4[4];
          if (wm == 0xfu && (((uintptr_t)pp) & 15) == 0) {
            const float4 q = __ldg((const float4 *)pp);
            p4[0] = q.x; p4[1] = q.y; p4[2] = q.z; p4[3] = q.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) p4[j] = ((wm >> j) & 1u) ? __ldg(pp + j) : 0.f;
          }
          const float fpv = (float)pv;
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if ((wm >> j) & 1u) rr[j] = __fsub_rn(rr[j], __fmul_rn(fpv, p4[j]));
          *(float4 *)rp = make_float4(rr[0], rr[1], rr[2], rr[3]);
        }
        if (bm != 0u && iy >= a.ybeg && iy < a.yend) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (!((bm >> j) & 1u)) continue;
            if (a.mask != nullptr && !(a.mask[(size_t)iy * nx + c0 + j] > (T)0.5)) continue;
            const float v = rr[j] < 0.f ? -rr[j] : rr[j];
            if ((T)v > best_abs) {
              best_abs = (T)v;
              best_idx = iy * nx + c0 + j;
              best_val = (T)rr[j];
            }
          }
        }
      }
    } else if (npr <= HOG_NPR) {
      // this thread's columns ix = threadIdx.x + k * HOG_THREADS: whether the
      // PSF window (with an existing PSF column) and the clean box cover them
      const int wlo = max(x1, px - a.pnx / 2), whi = min(x2, px + a.pnx / 2 - 1);
      bool colw[HOG_NPR], colb[HOG_NPR];
      int pxo[HOG_NPR];
#pragma unroll
      for (int k = 0; k < HOG_NPR; ++k) {
        const int ix = threadIdx.x + k * HOG_THREADS;
        const bool valid = k < npr && ix < nx;
        colw[k] = valid && do_sub && ix >= wlo && ix <= whi;
        colb[k] = valid && ix >= a.xbeg && ix < a.xend;
        pxo[k] = a.pnx / 2 + ix - px;
      }
      for (int iy0 = y_lo; iy0 < y_hi; iy0 += HOG_RB) {
        // the PSF values of HOG_RB rows through the read-only path, all
        // issued before the band is touched: one L2 round trip per batch
        T pk[HOG_RB][HOG_NPR];
#pragma unroll
        for (int q = 0; q < HOG_RB; ++q) {
          const int iy = iy0 + q;
          const int psf_y = a.pny / 2 + iy - py;
          const bool rsub = iy < y_hi && iy >= y1 && iy <= y2 && psf_y >= 0 && psf_y < a.pny;
          const T *prow = a.psf + (size_t)(rsub ? psf_y : 0) * a.pnx;
#pragma unroll
          for (int k = 0; k < HOG_NPR; ++k)
            pk[q][k] = (rsub && colw[k]) ? __ldg(prow + pxo[k]) : (T)0;
        }
#pragma unroll
        for (int q = 0; q < HOG_RB; ++q) {
          const int iy = iy0 + q;
          if (iy >= y_hi) break;  // the same for every thread of the block
          const int psf_y = a.pny / 2 + iy - py;
          const bool rsub = iy >= y1 && iy <= y2 && psf_y >= 0 && psf_y < a.pny;
          const bool rbox = iy >= a.ybeg && iy < a.yend;
          T *rrow = band + (size_t)(iy - y_lo) * nx;
#pragma unroll
          for (int k = 0; k < HOG_NPR; ++k) {
            const int ix = threadIdx.x + k * HOG_THREADS;
            if (k >= npr || ix >= nx) continue;
            T r = rrow[ix];
            if (rsub && colw[k]) {
              r = rn_sub(r, rn_mul(pv, pk[q][k]));
              rrow[ix] = r;
            }
            if (rbox && colb[k] &&
                (a.mask == nullptr || a.mask[(size_t)iy * nx + ix] > (T)0.5)) {
              const T v = r < (T)0 ? -r : r;
              if (v > best_abs) {
                best_abs = v;
                best_idx = iy * nx + ix;
                best_val = r;
              }
            }
          }
        }
      }
    } else
    for (int iy = y_lo; iy < y_hi; ++iy) {
      const bool row_sub = do_sub && iy >= y1 && iy <= y2;
      const bool row_box = iy >= a.ybeg && iy < a.yend;
      const int psf_y = a.pny / 2 + iy - py;
      const bool psf_row_ok = psf_y >= 0 && psf_y < a.pny;
      T *rrow = band + (size_t)(iy - y_lo) * nx;
      const T *prow = a.psf + (size_t)(psf_row_ok ? psf_y : 0) * a.pnx;
      for (int ix = threadIdx.x; ix < nx; ix += HOG_THREADS) {
        T r = rrow[ix];
        if (row_sub && psf_row_ok && ix >= x1 && ix <= x2) {
          int psf_x = a.pnx / 2 + ix - px;
          if (psf_x >= 0 && psf_x < a.pnx) {
            r = rn_sub(r, rn_mul(pv, prow[psf_x]));
            rrow[ix] = r;
          }
        }
        if (row_box && ix >= a.xbeg && ix < a.xend &&
            (a.mask == nullptr || a.mask[(size_t)iy * nx + ix] > (T)0.5)) {
          T v = r < (T)0 ? -r : r;
          if (v > best_abs) {
            best_abs = v;
            best_idx = iy * nx + ix;
            best_val = r;
          }
        }
      }
    }
    // block reduction (only strictly positive maxima count)
    if (best_idx >= 0 && !(best_abs > (T)0)) best_idx = -1;
    for (int o = 16; o > 0; o >>= 1) {
      T oa = __shfl_xor_sync(0xffffffffu, best_abs, o);
      int oi = __shfl_xor_sync(0xffffffffu, best_idx, o);
      T ov = __shfl_xor_sync(0xffffffffu, best_val, o);
      if (beats(oa, oi, best_abs, best_idx)) {
        best_abs = oa;
        best_idx = oi;
        best_val = ov;
      }
    }
    if (lane == 0) {
      s_abs[warp] = best_abs;
      s_idx[warp] = best_idx;
      s_val[warp] = best_val;
    }
    __syncthreads();
    if (warp == 0) {
      best_abs = s_abs[lane];
      best_idx = s_idx[lane];
      best_val = s_val[lane];
      for (int o = 16; o > 0; o >>= 1) {
        T oa = __shfl_xor_sync(0xffffffffu, best_abs, o);
        int oi = __shfl_xor_sync(0xffffffffu, best_idx, o);
        T ov = __shfl_xor_sync(0xffffffffu, best_val, o);
        if (beats(oa, oi, best_abs, best_idx)) {
          best_abs = oa;
          best_idx = oi;
          best_val = ov;
        }
      }
      if (lane == 0) {
        HogCand<T> c;
        c.absval = best_abs;
        c.val = best_val;
        c.idx = best_idx;
        // value at the current peak, published by its owner (used when no
        // pixel beats 0, where the reference keeps the previous position);
        // the block barrier above has ordered the band pass's writes
        const bool hp = py >= y_lo && py < y_hi;
        c.has_prev = hp ? 1 : 0;
        c.at_prev = hp ? band[(size_t)(py - y_lo) * nx + px] : (T)0;
        a.cand[par * G + b] = c;
        if (KEYED && best_idx >= 0) {
          const uint32_t code = 2u * (uint32_t)best_idx + (best_val < (T)0 ? 1u : 0u);
          const unsigned long long key =
              ((unsigned long long)__float_as_uint((float)best_abs) << 32) |
              (unsigned long long)(0xffffffffu - code);
          atomicMax(&a.state->key[par], key);
        }
      }
    }
    if (!grid_barrier(a.state, &s_flag, a.timeout_ns, KEYED ? &a.state->key[par ^ 1] : nullptr))
      break;
    // FP32: the winner from the 64-bit maximum (one load); otherwise, and
    // when no pixel was above 0, every CTA reduces all candidates the same way
    if (KEYED) {
      if (threadIdx.x == 0) {
        const unsigned long long kv = *(volatile unsigned long long *)&a.state->key[par];
        s_use_key = kv != 0ull;
        if (kv != 0ull) {
          const uint32_t code = 0xffffffffu - (uint32_t)kv;
          const float av = __uint_as_float((uint32_t)(kv >> 32));
          s_abs[0] = (T)av;
          s_idx[0] = (int)(code >> 1);
          s_val[0] = (code & 1u) ? (T)-av : (T)av;
        }
      }
      __syncthreads();
    }
    if (!(KEYED && s_use_key) && warp == 0) {
      T ga = (T)0, gv = (T)0, gprev = (T)0;
      int gi = -1, ghp = 0;
      for (int k0 = 0; k0 < G; k0 += 32 * HOG_CPL) {
        // L2 loads (other CTAs wrote these before the barrier), HOG_CPL
        // candidates per lane issued together, then reduced in index order
        HogCand<T> c[HOG_CPL];
#pragma unroll
        for (int q = 0; q < HOG_CPL; ++q) {
          const int k = k0 + lane + 32 * q;
          c[q].idx = -1;
          c[q].has_prev = 0;
          if (k < G) {
            const HogCand<T> *cp = a.cand + par * G + k;
            c[q].absval = __ldcg(&cp->absval);
            c[q].val = __ldcg(&cp->val);
            c[q].at_prev = __ldcg(&cp->at_prev);
            c[q].idx = __ldcg(&cp->idx);
            c[q].has_prev = __ldcg(&cp->has_prev);
          }
        }
#pragma unroll
        for (int q = 0; q < HOG_CPL; ++q) {
          if (beats(c[q].absval, c[q].idx, ga, gi)) {
            ga = c[q].absval;
            gi = c[q].idx;
            gv = c[q].val;
          }
          if (c[q].has_prev) {
            gprev = c[q].at_prev;
            ghp = 1;
          }
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        T oa = __shfl_xor_sync(0xffffffffu, ga, o);
        int oi = __shfl_xor_sync(0xffffffffu, gi, o);
        T ov = __shfl_xor_sync(0xffffffffu, gv, o);
        T op = __shfl_xor_sync(0xffffffffu, gprev, o);
        int oh = __shfl_xor_sync(0xffffffffu, ghp, o);
        if (beats(oa, oi, ga, gi)) {
          ga = oa;
          gi = oi;
          gv = ov;
        }
        if (oh) {
          gprev = op;
          ghp = 1;
        }
      }
      if (lane == 0) {
        s_abs[0] = ga;
        s_idx[0] = gi;
        s_val[0] = gv;
        s_prev = gprev;
      }
    }
    __syncthreads();
    if (s_idx[0] >= 0) {
      px = s_idx[0] % nx;
      py = s_idx[0] / nx;
      peak = s_val[0];
      absval = s_abs[0];
    } else {
      peak = s_prev;
      absval = (T)0;
    }
    __syncthreads();
    par ^= 1;
    if (first) first = false;
    else ++it;
  }
  // write the band back and publish the state
  __syncthreads();
  if (a.resident) {
    for (int i0 = 0; i0 < (y_hi - y_lo) * nx; i0 += HOG_THREADS) {
      const int i = i0 + threadIdx.x;
      if (i < (y_hi - y_lo) * nx) a.resid[(size_t)y_lo * nx + i] = band[i];
    }
  }
  if (b == 0 && threadIdx.x == 0) {
    a.state->kpar = par;
    a.state->iter = it;
    a.state->px = px;
    a.state->py = py;
    a.state->peak = (double)peak;
    a.state->absval = (double)absval;
    a.state->stopped = stopped ? 1 : 0;
  }
}

// ------------------------------------------------------------------ maximg --
template <typename T>
__global__ void __launch_bounds__(1024) k_maximg_partial(const T *img, const T *mask, int64_t n,
                                                        T *part) {
  T mn = (T)1e20, mx = (T)-1e20;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (mask == nullptr || mask[i] > (T)0.5) {
      T w = img[i];
      if (w > mx) mx = w;
      if (w < mn) mn = w;
    }
  }
  __shared__ T smn[32], smx[32];
  for (int o = 16; o > 0; o >>= 1) {
    T a = __shfl_xor_sync(0xffffffffu, mn, o), c = __shfl_xor_sync(0xffffffffu, mx, o);
    if (a < mn) mn = a;
    if (c > mx) mx = c;
  }
  if ((threadIdx.x & 31) == 0) {
    smn[threadIdx.x >> 5] = mn;
    smx[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      if (smn[w] < mn) mn = smn[w];
      if (smx[w] > mx) mx = smx[w];
    }
    part[2 * blockIdx.x] = mn;
    part[2 * blockIdx.x + 1] = mx;
  }
}

template <typename T>
__global__ void k_maximg_final(const T *part, int np, T *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  T mn = (T)1e20, mx = (T)-1e20;
  for (int i = 0; i < np; ++i) {
    if (part[2 * i] < mn) mn = part[2 * i];
    if (part[2 * i + 1] > mx) mx = part[2 * i + 1];
  }
  out[0] = mn;
  out[1] = mx;
}

// --------------------------------------------------- ordered |x| summation --
// Sum of |x| in index order with sequential addition: zeros do not change a
// running sum, so the non-zeros are compacted in order and summed by one
// thread.
constexpr int ABS_THREADS = 1024;

template <typename T>
__device__ void thread_range(int64_t n, int64_t &lo, int64_t &hi) {
  int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
  int64_t blo = blockIdx.x * per_block, bhi = min(n, blo + per_block);
  int64_t per_t = (bhi - blo + ABS_THREADS - 1) / ABS_THREADS;
  lo = min(bhi, blo + threadIdx.x * per_t);
  hi = min(bhi, lo + per_t);
}

template <typename T>
__global__ void __launch_bounds__(ABS_THREADS) k_nz_count(const T *x, int64_t n,
                                                          uint32_t *counts) {
  int64_t lo, hi;
  thread_range<T>(n, lo, hi);
  uint32_t c = 0;
  for (int64_t i = lo; i < hi; ++i) c += x[i] != (T)0;
  __shared__ uint32_t sh[32];
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < ABS_THREADS / 32; ++w) t += sh[w];
    counts[blockIdx.x] = t;
  }
}

template <typename T>
__global__ void __launch_bounds__(ABS_THREADS) k_nz_write(const T *x, int64_t n,
                                                          const uint32_t *counts, T *out) {
  __shared__ uint32_t sh[ABS_THREADS];
  __shared__ uint32_t base;
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int k = 0; k < (int)blockIdx.x; ++k) s += counts[k];
    base = s;
  }
  int64_t lo, hi;
  thread_range<T>(n, lo, hi);
  uint32_t c = 0;
  for (int64_t i = lo; i < hi; ++i) c += x[i] != (T)0;
  sh[threadIdx.x] = c;
  __syncthreads();
  // exclusive prefix over threads (simple, once per call)
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int k = 0; k < ABS_THREADS; ++k) {
      uint32_t v = sh[k];
      sh[k] = s;
      s += v;
    }
  }
  __syncthreads();
  uint32_t pos = base + sh[threadIdx.x];
  for (int64_t i = lo; i < hi; ++i) {
    T v = x[i];
    if (v != (T)0) out[pos++] = v < (T)0 ? -v : v;
  }
}

template <typename T>
__global__ void k_seq_sum(const T *v, const uint32_t *counts, int nblocks, T *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t n = 0;
  for (int k = 0; k < nblocks; ++k) n += counts[k];
  T s = (T)0;
  for (uint32_t i = 0; i < n; ++i) s = rn_add(s, v[i]);
  out[0] = s;
}

template <typename T>
static int hogbom_launch(HogArgs<T> a, int grid, size_t smem, cudaStream_t st) {
  void *args[] = {&a};
  AV_CUDA(cudaLaunchCooperativeKernel((const void *)k_hogbom<T>, grid, HOG_THREADS, args, smem,
                                      st));
  count_launch();
  return AV_OK;
}

}  // namespace av

using namespace av;

extern "C" {

size_t av_hogbom_state_size(void) { return sizeof(HogState); }

size_t av_hogbom_workspace_size(int64_t nx, int64_t ny, int dtype) {
  (void)nx;
  (void)ny;
  size_t cs = dtype == AV_F64 ? sizeof(HogCand<double>) : sizeof(HogCand<float>);
  return Workspace::need(cs * 2 * 1024);
}

int av_hogbom_run(void *model, void *residual, const void *psf, const void *mask, int dtype,
                  int64_t nx, int64_t ny, int64_t pnx, int64_t pny, int xbeg, int xend,
                  int ybeg, int yend, int niter, int siter, int iter_begin, int iter_end,
                  double gain, double threshold, double speedup, void *state, int init_state,
                  void *workspace, size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(model && residual && psf && state && workspace, "av_hogbom_run: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_hogbom_run: dtype");
  AV_CHECK_ARG(nx > 0 && ny > 0 && pnx > 0 && pny > 0 && nx * ny < (1LL << 31),
               "av_hogbom_run: bad shape");
  AV_CHECK_ARG(xbeg >= 0 && xend <= nx && xbeg < xend && ybeg >= 0 && yend <= ny && ybeg < yend,
               "av_hogbom_run: bad clean box");
  AV_CHECK_ARG(workspace_bytes >= av_hogbom_workspace_size(nx, ny, dtype),
               "av_hogbom_run: workspace too small");
  cudaStream_t st = as_stream(stream);
  int dev = 0;
  AV_CUDA(cudaGetDevice(&dev));
  const unsigned long long timeout_ns =
      (unsigned long long)tune_value(AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US) * 1000ull;
  int sms = sm_count();
  int grid = (int)std::min<int64_t>(sms, ny);
  if (grid > 1024) grid = 1024;
  size_t esz = dtype == AV_F64 ? 8 : 4;
  int64_t band_rows = (ny + grid - 1) / grid;
  size_t band_bytes = (size_t)band_rows * nx * esz;
  int max_smem = 0;
  AV_CUDA(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  int resident = band_bytes + 4096 <= (size_t)max_smem;
  size_t smem = resident ? band_bytes : 0;
  if (init_state) AV_CUDA(cudaMemsetAsync(state, 0, sizeof(HogState), st));
  if (dtype == AV_F32) {
    AV_CUDA(cudaFuncSetAttribute(k_hogbom<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int per_sm = 0;
    AV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hogbom<float>, HOG_THREADS,
                                                          smem));
    if (per_sm < 1) {
      set_error("av_hogbom_run: kernel cannot be resident (smem %zu)", smem);
      return AV_ERR_UNSUPPORTED;
    }
    HogArgs<float> a;
    a.model = (float *)model; a.resid = (float *)residual; a.psf = (const float *)psf;
    a.mask = (const float *)mask;
    a.nx = (int)nx; a.ny = (int)ny; a.pnx = (int)pnx; a.pny = (int)pny;
    a.xbeg = xbeg; a.xend = xend; a.ybeg = ybeg; a.yend = yend;
    a.niter = niter; a.siter = siter; a.iter_begin = iter_begin; a.iter_end = iter_end;
    a.gain = (float)gain; a.thres = (float)threshold; a.speedup = (float)speedup;
    a.state = (HogState *)state; a.cand = (HogCand<float> *)workspace;
    a.init = init_state; a.resident = resident; a.timeout_ns = timeout_ns;
    return hogbom_launch<float>(a, grid, smem, st);
  }
  AV_CUDA(cudaFuncSetAttribute(k_hogbom<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  int per_sm = 0;
  AV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hogbom<double>, HOG_THREADS,
                                                        smem));
  if (per_sm < 1) {
    set_error("av_hogbom_run: kernel cannot be resident (smem %zu)", smem);
    return AV_ERR_UNSUPPORTED;
  }
  HogArgs<double> a;
  a.model = (double *)model; a.resid = (double *)residual; a.psf = (const double *)psf;
  a.mask = (const double *)mask;
  a.nx = (int)nx; a.ny = (int)ny; a.pnx = (int)pnx; a.pny = (int)pny;
  a.xbeg = xbeg; a.xend = xend; a.ybeg = ybeg; a.yend = yend;
  a.niter = niter; a.siter = siter; a.iter_begin = iter_begin; a.iter_end = iter_end;
  a.gain = gain; a.thres = threshold; a.speedup = speedup;
  a.state = (HogState *)state; a.cand = (HogCand<double> *)workspace;
  a.init = init_state; a.resident = resident; a.timeout_ns = timeout_ns;
  return hogbom_launch<double>(a, grid, smem, st);
}

int av_hogbom_state_read(const void *state, int32_t *out_i, double *out_d, void *stream) {
  clear_error();
  AV_CHECK_ARG(state && out_i && out_d, "av_hogbom_state_read: null pointer");
  HogState h;
  cudaStream_t st = as_stream(stream);
  AV_CUDA(cudaMemcpyAsync(&h, state, sizeof(h), cudaMemcpyDeviceToHost, st));
  AV_CUDA(cudaStreamSynchronize(st));
  out_i[0] = h.iter;
  out_i[1] = h.px;
  out_i[2] = h.py;
  out_i[3] = h.stopped;
  out_i[4] = h.err;
  out_d[0] = h.peak;
  out_d[1] = h.absval;
  if (h.err) {
    set_error("av_hogbom_run: grid barrier timed out");
    return AV_ERR_TIMEOUT;
  }
  return AV_OK;
}

int av_maximg(const void *image, const void *mask, int dtype, int64_t nx, int64_t ny, void *out,
              void *stream) {
  clear_error();
  AV_CHECK_ARG(image && out, "av_maximg: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_maximg: dtype");
  AV_CHECK_ARG(nx >= 0 && ny >= 0, "av_maximg: bad shape");
  cudaStream_t st = as_stream(stream);
  int64_t n = nx * ny;
  // one CTA: min / max are order independent, the pass is small
  if (dtype == AV_F32)
    k_maximg_partial<float><<<1, 1024, 0, st>>>((const float *)image, (const float *)mask, n,
                                                (float *)out);
  else
    k_maximg_partial<double><<<1, 1024, 0, st>>>((const double *)image, (const double *)mask, n,
                                                 (double *)out);
  AV_LAUNCH_CHECK();
  return AV_OK;
}

size_t av_abs_sum_workspace_size(int64_t n, int dtype) {
  size_t esz = dtype == AV_F64 ? 8 : 4;
  return Workspace::need(sizeof(uint32_t) * 1024) + Workspace::need(esz * (size_t)(n > 0 ? n : 1));
}

int av_abs_sum_ordered(const void *model, int dtype, int64_t n, void *out, void *workspace,
                       size_t workspace_bytes, void *stream) {
  clear_error();
  AV_CHECK_ARG(model && out && workspace, "av_abs_sum_ordered: null pointer");
  AV_CHECK_ARG(dtype == AV_F32 || dtype == AV_F64, "av_abs_sum_ordered: dtype");
  AV_CHECK_ARG(workspace_bytes >= av_abs_sum_workspace_size(n, dtype),
               "av_abs_sum_ordered: workspace too small");
  cudaStream_t st = as_stream(stream);
  Workspace ws(workspace, workspace_bytes);
  uint32_t *counts = ws.take<uint32_t>(1024);
  int nb = (int)std::min<int64_t>(std::max<int64_t>(1, (n + 65535) / 65536), 1024);
  if (dtype == AV_F32) {
    float *buf = ws.take<float>(n > 0 ? n : 1);
    k_nz_count<float><<<nb, ABS_THREADS, 0, st>>>((const float *)model, n, counts);
    AV_LAUNCH_CHECK();
    k_nz_write<float><<<nb, ABS_THREADS, 0, st>>>((const float *)model, n, counts, buf);
    AV_LAUNCH_CHECK();
    k_seq_sum<float><<<1, 32, 0, st>>>(buf, counts, nb, (float *)out);
  } else {
    double *buf = ws.take<double>(n > 0 ? n : 1);
    k_nz_count<double><<<nb, ABS_THREADS, 0, st>>>((const double *)model, n, counts);
    AV_LAUNCH_CHECK();
    k_nz_write<double><<<nb, ABS_THREADS, 0, st>>>((const double *)model, n, counts, buf);
    AV_LAUNCH_CHECK();
    k_seq_sum<double><<<1, 32, 0, st>>>(buf, counts, nb, (double *)out);
  }
  AV_LAUNCH_CHECK();
  return AV_OK;
}

}  // extern "C"
