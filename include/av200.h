/*
 * av200.h - C ABI of libav200.so, the B200 (sm_100a) kernels of the
 * astroviper standard-gridder imaging path.
 *
 * Conventions
 *   - Every entry point returns an int status (AV_OK = 0) and never aborts;
 *     av_last_error() gives the message of the calling thread's last failure.
 *   - All array arguments are DEVICE pointers to C-contiguous arrays owned by
 *     the caller; shapes are passed explicitly.  Nothing is copied to or from
 *     the host.  `stream` is a cudaStream_t (NULL = legacy default stream).
 *   - Scratch memory is supplied by the caller as (workspace, workspace_bytes);
 *     the matching *_workspace_size() call says how many bytes are needed.
 *     Workspace pointers must be 256-byte aligned.
 *   - Array layouts follow the reference: visibilities / weights / flags are
 *     (n_time, n_baseline, n_chan, n_pol); uvw is (n_time, n_baseline, 3)
 *     float64 metres; grids are (n_chan, n_pol, n_u, n_v) with u on axis 2.
 *   - dtype codes: AV_F32, AV_F64 (real), AV_C64, AV_C128 (complex,
 *     interleaved re/im).
 *
 * Reference interfaces each entry point replaces are cited as
 * file:line inside the astroviper project (src/astroviper/...).
 */
#ifndef AV200_H
#define AV200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum av_status {
  AV_OK = 0,
  AV_ERR_ARG = 1,          /* invalid shape, size, dtype or pointer */
  AV_ERR_CUDA = 2,         /* a CUDA or cuFFT call failed */
  AV_ERR_TIMEOUT = 3,      /* a bounded device-side wait gave up */
  AV_ERR_NAN = 4,          /* NaN where the reference raises (Briggs factors) */
  AV_ERR_UNSUPPORTED = 5,  /* valid request this kernel does not cover */
  AV_ERR_WORKSPACE = 6     /* workspace missing, misaligned or too small */
};

enum av_dtype { AV_F32 = 0, AV_F64 = 1, AV_C64 = 2, AV_C128 = 3 };

/* Library version (major*10000 + minor*100 + patch). */
int av_version(void);
/* Message of this thread's last failed call ("" if none). */
const char *av_last_error(void);
/* Number of SMs of the current device (for launch sizing by the host). */
int av_device_sm_count(void);
/* No counterpart in the reference: the FP64 tensor-core rate of the current
 * device in TFLOP/s (mma.sync.m16n8k4.f64, 8 CTAs of 8 warps per SM, four
 * independent chains per warp; three timed launches after one warm-up).  It
 * is the ceiling of the gridder's FP64 footprint sums, reported beside its
 * HBM roofline.  Synchronises the stream; writes into a 32 KiB static device
 * array, allocates nothing. */
int av_probe_fp64_mma(double *tflops, void *stream);
/* Kernels launched by this library since it was loaded (all threads). */
unsigned long long av_launch_count(void);

/* Launch tuning (no counterpart in the reference, which has no GPU path):
 * process-wide knobs read when a kernel is launched, set by the autotuner
 * (astroviper_b200.autotune) or by hand.
 *   AV_TUNE_GRID_CHUNKS_PER_SM   record chunks per SM handed out by the
 *                                persistent tiled gridder (default 16)
 *   AV_TUNE_DEGRID_CHUNKS_PER_SM record chunks per SM handed out by the
 *                                persistent tiled degridder (default 16)
 *   AV_TUNE_GRID_LANES           how the tiled gridder sums a run of samples:
 *                                AV_GRID_LANES_MMA (FP64 tensor-core tiles,
 *                                supports up to 8), AV_GRID_LANES_ROWS (a
 *                                footprint row per lane, DFMA) or
 *                                AV_GRID_LANES_AUTO (default: tensor-core
 *                                tiles for supports 5-8, where they are the
 *                                faster, rows otherwise); support 9 always
 *                                uses rows
 *   AV_TUNE_DEGRID_LANES         how the tiled degridder's fast store path
 *                                (complex64 values, 4 polarisations, no flags
 *                                or phase) runs: AV_DEGRID_LANES_TF32 (TF32
 *                                tensor-core tiles with split operands,
 *                                supports up to 8), AV_DEGRID_LANES_FP32 (FP32
 *                                FMA), AV_DEGRID_LANES_TC05 (TF32 with
 *                                split operands on the fifth-generation
 *                                tensor cores, accumulators in tensor memory,
 *                                supports up to 8) or AV_DEGRID_LANES_AUTO
 *                                (default: TF32 for supports up to 8, FP32
 *                                for 9)
 *   AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US  how long (microseconds of wall time,
 *                                default 2000000) a CTA of av_hogbom_run
 *                                waits at the per-iteration grid barrier
 *                                before it gives up; on giving up the launch
 *                                ends, av_hogbom_state_read returns
 *                                AV_ERR_TIMEOUT ("grid barrier timed out")
 *                                and the run must be started again
 *                                (init_state = 1).  0 makes every CTA but
 *                                the last to arrive give up at its first
 *                                barrier, which is how the timeout path is
 *                                tested.  Range [0, 600000000].
 * av_tune_set returns AV_ERR_ARG for an unknown knob or a value outside
 * [1, 1024] ([1, 3] for AV_TUNE_GRID_LANES, [1, 4] for AV_TUNE_DEGRID_LANES,
 * [0, 600000000] for the barrier timeout); av_tune_get returns -1 for an
 * unknown knob. */
enum av_tune {
  AV_TUNE_GRID_CHUNKS_PER_SM = 0,
  AV_TUNE_DEGRID_CHUNKS_PER_SM = 1,
  AV_TUNE_GRID_LANES = 2,
  AV_TUNE_DEGRID_LANES = 3,
  AV_TUNE_HOGBOM_BARRIER_TIMEOUT_US = 4
};
enum av_grid_lanes { AV_GRID_LANES_MMA = 1, AV_GRID_LANES_ROWS = 2, AV_GRID_LANES_AUTO = 3 };
enum av_degrid_lanes {
  AV_DEGRID_LANES_TF32 = 1,
  AV_DEGRID_LANES_FP32 = 2,
  AV_DEGRID_LANES_AUTO = 3,
  AV_DEGRID_LANES_TC05 = 4
};
int av_tune_set(int knob, int64_t value);
int64_t av_tune_get(int knob);

/* ---------------------------------------------------------------- PSWF -- */
/* prolate_spheroidal_function, gcf_prolate_spheroidal.py:102-158:
 * grdsf[i], kern[i] = (grdsf(u), (1-u^2) grdsf(u)) for u = u_in[i] (FP64).
 * Either output may be NULL. */
int av_pswf(const double *u_in, int64_t n, double *grdsf, double *kern, void *stream);

/* create_prolate_spheroidal_kernel_1D, gcf_prolate_spheroidal.py:87-99:
 * out has oversampling*(support/2+1) doubles. */
int av_pswf_table(double *out, int oversampling, int support, void *stream);

/* Grid-correction image of create_prolate_spheroidal_kernel,
 * gcf_prolate_spheroidal.py:73-79: out (nx, ny) doubles. */
int av_corr_term(double *out, int64_t nx, int64_t ny, void *stream);

/* The 4-D oversampled kernel of create_prolate_spheroidal_kernel,
 * gcf_prolate_spheroidal.py:28-67: out (n_os, n_os, support, support) doubles
 * with n_os = oversampling + 1 for even oversampling, else oversampling. */
int av_pswf_kernel4d(double *out, int oversampling, int support, void *stream);

/* ------------------------------------------------------------- gridding -- */
/* Common gridding arguments (standard_grid_jit, standard_grid.py:246-432):
 *   vis        (nt, nb, nchan, npol) of vis_dtype (AV_C64 or AV_C128); may be
 *              NULL when do_psf != 0
 *   weight     (nt, nb, nchan, npol) of weight_dtype (AV_F32 or AV_F64)
 *   uvw        (nt, nb, 3) float64; freq (nchan) float64
 *   chan_map   (nchan) int32 -> image channel; pol_map (npol) int32 -> image pol
 *   cgk        the 1-D half kernel (oversampling*(support/2+1) doubles)
 *   grid       (n_img_chan, n_img_pol, n_u, n_v) of grid_dtype, accumulated
 *              (+=); AV_C64 / AV_C128, or AV_F32 / AV_F64 with do_psf
 *   sum_weight (n_img_chan, n_img_pol) float64, accumulated (+=)
 *   delta_lm   cell size (2) in radians, as passed to the reference.
 */

/* Plain FP64 gridder: one thread per (time, baseline, channel) sample, the
 * reference's arithmetic and order per sample, FP64 atomic accumulation.
 * Covers every option of standard_grid_jit including do_imaging_weight.
 * Replaces standard_grid_jit (standard_grid.py:246). */
int av_grid_plain(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                  int do_imaging_weight, const void *vis, int vis_dtype, const void *weight,
                  int weight_dtype, const double *uvw, const double *freq,
                  const int32_t *chan_map, const int32_t *pol_map, const double *cgk,
                  int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                  int oversampling, int64_t nt, int64_t nb, int64_t nchan, int64_t npol,
                  int64_t n_img_chan, int64_t n_img_pol, void *stream);

/* Scratch bytes for av_grid_tiled with these sizes. */
size_t av_grid_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u,
                                    int64_t n_v, int64_t n_img_chan, int support);

/* Tiled gridder (same semantics as av_grid_plain without
 * do_imaging_weight): samples are binned by uv cell in a plan held in the
 * workspace, each CTA accumulates a tile's sub-grid in shared memory with
 * register-resident runs, and flushes it once.  Reads complex64 visibilities
 * and float32 weights; index math, tap weights and all accumulation in FP64
 * (FP32 accumulation leaves 1e-4-level errors in grid-corrected images).
 * The grid may be complex128 (full accuracy) or complex64.  Requires
 * npol <= 4, n_img_pol <= 4, 3 <= support <= 9, oversampling <= 254.
 * Replaces standard_grid_jit (standard_grid.py:246) for do_imaging_weight=0. */
/* The two halves of av_grid_tiled: _plan bins the samples (depends only on
 * uvw, freq, chan_map and the geometry) into the workspace; _execute grids
 * vis / weights with that plan.  A plan is reusable for any number of
 * executes with the same geometry (e.g. every major cycle), as long as the
 * workspace is left untouched in between.  The execute's persistent kernel
 * takes its work chunks from counters in the workspace, so executes on one
 * plan must not run concurrently (stream order is enough); neither call
 * synchronises, allocates or touches the host, so both can be captured in a
 * CUDA graph once the first execute on the device has run outside capture. */
int av_grid_tiled_plan(const double *uvw, const double *freq, const int32_t *chan_map,
                       int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                       int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                       int64_t n_img_chan, void *workspace, size_t workspace_bytes,
                       void *stream);
int av_grid_tiled_execute(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                          const void *vis, int vis_dtype, const void *weight, int weight_dtype,
                          const int32_t *pol_map, const double *cgk, int64_t n_u, int64_t n_v,
                          int support, int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                          int64_t npol, int64_t n_img_chan, int64_t n_img_pol, void *workspace,
                          size_t workspace_bytes, void *stream);
int av_grid_tiled(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                  const void *vis, int vis_dtype, const void *weight, int weight_dtype,
                  const double *uvw, const double *freq, const int32_t *chan_map,
                  const int32_t *pol_map, const double *cgk, int64_t n_u, int64_t n_v,
                  double delta_l, double delta_m, int support, int oversampling, int64_t nt,
                  int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                  int64_t n_img_pol, void *workspace, size_t workspace_bytes, void *stream);

/* No counterpart in the reference: av_grid_tiled_plan that also leaves out
 * the samples whose every weight is zero or NaN (flagged data), which
 * standard_grid_jit skips (standard_grid.py:378), so that grids with many
 * flagged samples take less work.  weight (nt, nb, nchan, npol) float32, as
 * the execute will read it: the plan then holds for those weights only (a
 * fresh set of flags needs a fresh plan).  Same workspace as
 * av_grid_tiled_plan; for av_grid_tiled_execute only. */
int av_grid_tiled_plan_weighted(const double *uvw, const double *freq, const int32_t *chan_map,
                                const float *weight, int64_t npol, int64_t n_u, int64_t n_v,
                                double delta_l, double delta_m, int support, int oversampling,
                                int64_t nt, int64_t nb, int64_t nchan, int64_t n_img_chan,
                                void *workspace, size_t workspace_bytes, void *stream);
/* No counterpart in the reference: zeroes the grid cells a plan's records
 * can touch (the footprint region of every tile holding records, all n_img_pol
 * polarisations), in place of clearing the whole grid before an execute that
 * accumulates.  The grid's other cells are left as they are: use it on a grid
 * whose other cells are zero, such as one that held a result of a plan with
 * the same or a larger footprint.  Any tiled plan (gridder, degridder,
 * shared, weighted) with these sizes. */
int av_grid_tiled_clear(void *grid, int grid_dtype, int64_t n_img_pol, int64_t n_u, int64_t n_v,
                        int support, int64_t nt, int64_t nb, int64_t nchan, int64_t n_img_chan,
                        const void *workspace, size_t workspace_bytes, void *stream);
/* No counterpart in the reference: one plan for both av_grid_tiled_execute
 * and av_degrid_tiled_execute (the gridder's and the degridder's binning
 * differ only in their rounding, standard_grid.py:337-352 against
 * standard_degrid.py:442-450).  Same arguments as av_grid_tiled_plan and the
 * same workspace size (av_grid_tiled_workspace_size, or
 * av_degrid_tiled_workspace_size with the same sizes).  Records are sorted
 * by the gridder's cells; samples whose cell, offsets or bounds verdict differ
 * under the degridder's half-even rounding are marked, and those it keeps are
 * degridded separately in FP64 by av_degrid_tiled_execute, so both
 * executes give what a plan of their own would (the degridder's values of
 * those samples in FP64 instead of FP32).  Valid for a degrid of a grid of
 * n_img_chan channels and (n_u, n_v) cells whose channel map
 * int(i / nchan * n_img_chan) equals chan_map (continuum: all 0; cube: the
 * identity), with the degridder's scale (-delta_l * n_u, -delta_m * n_v) and
 * offset (n_u / 2, n_v / 2), as degrid_spheroid_ms4 passes them.  Not for
 * av_degrid_tiled_adjoint.  At most 2^31 - 1 samples. */
int av_tiled_plan_shared(const double *uvw, const double *freq, const int32_t *chan_map,
                         int64_t n_u, int64_t n_v, double delta_l, double delta_m, int support,
                         int oversampling, int64_t nt, int64_t nb, int64_t nchan,
                         int64_t n_img_chan, void *workspace, size_t workspace_bytes,
                         void *stream);
/* No counterpart in the reference (diagnostics): out[0] = usable records of
 * a tiled plan (gridder, degridder or shared), out[1] = samples a shared plan
 * lists for the degridder's FP64 pass (0 for the others).  Synchronises. */
int av_tiled_plan_counts(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u, int64_t n_v,
                         int64_t n_img_chan, int support, const void *workspace,
                         size_t workspace_bytes, uint32_t *out, void *stream);

/* No counterpart in the reference: bitwise-reproducible gridding.
 * av_tiled_plan_order_rows orders each cell key's records of a built tiled
 * plan (gridder or shared; a shared plan's degridder marks move with them)
 * by row, so the order of a cell's samples no longer depends on the plan
 * build's atomics.  av_grid_tiled_execute_det then grids like
 * av_grid_tiled_execute (same arguments; supports 3-8, the FP64 tensor-core
 * kernel) with every sum past a run's FP64 sum in 64-bit fixed point: the
 * grid and sum_weight it adds are bit-identical from call to call for the
 * same plan, inputs and launch settings (AV_TUNE_GRID_CHUNKS_PER_SM), and
 * agree with av_grid_tiled_execute's to within the FP64 summation order
 * (the tests hold both to 1e-13, norm-wise, of the FP64 oracle).  It needs
 * det_workspace (256-byte aligned) of av_grid_tiled_det_workspace_size
 * bytes, synchronises the stream once (to report an unordered plan or an
 * infinite value, AV_ERR_ARG) and runs about twice as long as
 * av_grid_tiled_execute. */
int av_tiled_plan_order_rows(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u, int64_t n_v,
                             int64_t n_img_chan, int support, void *workspace,
                             size_t workspace_bytes, void *stream);
size_t av_grid_tiled_det_workspace_size(int64_t n_img_chan, int64_t n_img_pol, int64_t n_u,
                                        int64_t n_v);
int av_grid_tiled_execute_det(void *grid, int grid_dtype, double *sum_weight, int do_psf,
                              const void *vis, int vis_dtype, const void *weight,
                              int weight_dtype, const int32_t *pol_map, const double *cgk,
                              int64_t n_u, int64_t n_v, int support, int oversampling, int64_t nt,
                              int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                              int64_t n_img_pol, void *workspace, size_t workspace_bytes,
                              void *det_workspace, size_t det_workspace_bytes, void *stream);

/* ----------------------------------------------------------- degridding -- */
/* dgrid_numba, standard_degrid.py:388-485: values (nt, nb, nvchan, nvpol) of
 * values_dtype (AV_C64 / AV_C128) += sum_k w_k grid_k conj(phasor) / sum_k w_k
 * for unflagged samples whose support lies inside the grid.
 *   flag (nt, nb, nvchan, nvpol) uint8 (0 = use); may be NULL (no flags)
 *   dphase (nt, nb) float64; may be NULL (zero phase)
 *   scale_x/y, offset_x/y: the first two entries of the reference's scale and
 *              offset arrays (standard_degrid.py:572-573), by value
 *   grid (g_nchan, g_npol, g_n2, g_n3) of grid_dtype (AV_C64 / AV_C128)
 *   convFunc the 1-D half kernel (doubles); chanmap (nvchan), polmap (nvpol)
 *   int32 */
/* Plain FP64 degridder: one thread per sample and polarisation, the
 * reference's summation order (bit-identical to it in FP64). */
int av_degrid_plain(const double *uvw, const double *dphase, void *values, int values_dtype,
                    const uint8_t *flag, double scale_x, double scale_y, double offset_x, double offset_y,
                    const void *grid, int grid_dtype, int64_t g_nchan, int64_t g_npol,
                    int64_t g_n2, int64_t g_n3, const double *freq, double c, int support,
                    int sampling, const double *convFunc, const int32_t *chanmap,
                    const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                    int64_t nvpol, void *stream);

/* Adjoint of av_degrid_plain (FP64, the degridder's exact positions and
 * maps): grid (c128 / c64, +=) gets w_k / (sum_k w_k) * phasor * values for
 * every unflagged sample - the gradient of the degridder with respect to the
 * grid.  No counterpart function in the reference: it is the transpose of
 * dgrid_numba (standard_degrid.py:388-485). */
int av_degrid_plain_adjoint(const double *uvw, const double *dphase, const void *values,
                            int values_dtype, const uint8_t *flag, double scale_x, double scale_y,
                            double offset_x, double offset_y, void *grid, int grid_dtype,
                            int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                            const double *freq, double c, int support, int sampling,
                            const double *convFunc, const int32_t *chanmap,
                            const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                            int64_t nvpol, void *stream);

size_t av_degrid_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nvchan, int64_t g_n2,
                                      int64_t g_n3, int64_t g_nchan, int support);

/* FP32 tiled degridder: samples binned by uv cell, each CTA stages a tile's
 * sub-grid in shared memory, one thread per sample, FP32 products and sums.
 * Requires nvpol <= 4, g_npol <= 4, support <= 9, sampling <= 254. */
/* The two halves of av_degrid_tiled (plan from uvw / freq / chanmap and the
 * degridder's scale and offset; execute per model grid), reusable like the
 * gridder's. */
int av_degrid_tiled_plan(const double *uvw, const double *freq, const int32_t *chanmap,
                         double scale_x, double scale_y, double offset_x, double offset_y,
                         int64_t g_nchan, int64_t g_n2, int64_t g_n3, int support, int sampling,
                         int64_t nt, int64_t nb, int64_t nvchan, void *workspace,
                         size_t workspace_bytes, void *stream);
int av_degrid_tiled_execute(const double *dphase, void *values, int values_dtype,
                            int accumulate, const uint8_t *flag, const void *grid, int grid_dtype,
                            int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                            const double *freq, int support, int sampling,
                            const double *convFunc, const int32_t *polmap, int64_t nt,
                            int64_t nb, int64_t nvchan, int64_t nvpol, void *workspace,
                            size_t workspace_bytes, void *stream);
/* Whether a launch of the tensor-memory degridder (AV_DEGRID_LANES_TC05) on
 * the current device gave up a bounded wait for its MMAs since the flag was
 * last cleared: *out = 1 if so (the samples of that launch's warpgroup are
 * then partly unwritten), 0 otherwise; clear != 0 resets it.  Synchronises
 * the stream.  No counterpart in the reference (its degridder runs on the
 * CPU). */
int av_degrid_fault_read(int *out, int clear, void *stream);
int av_degrid_tiled(const double *uvw, const double *dphase, void *values, int values_dtype,
                    int accumulate, const uint8_t *flag, double scale_x, double scale_y,
                    double offset_x, double offset_y, const void *grid, int grid_dtype,
                    int64_t g_nchan, int64_t g_npol, int64_t g_n2, int64_t g_n3,
                    const double *freq, double c, int support, int sampling,
                    const double *convFunc, const int32_t *chanmap, const int32_t *polmap,
                    int64_t nt, int64_t nb, int64_t nvchan, int64_t nvpol, void *workspace,
                    size_t workspace_bytes, void *stream);

/* Adjoint of the tiled degridder (zero phase), run on a plan built by
 * av_degrid_tiled_plan in the same workspace: grid (+=) gets
 * w_k / (sum_k w_k) * values for every unflagged sample (complex64 values,
 * FP64 accumulation).  The transpose of dgrid_numba
 * (standard_degrid.py:388-485); no counterpart function in the reference. */
int av_degrid_tiled_adjoint(void *grid, int grid_dtype, const void *values, int values_dtype,
                            const uint8_t *flag, int64_t g_nchan, int64_t g_npol, int64_t g_n2,
                            int64_t g_n3, int support, int sampling, const double *convFunc,
                            const int32_t *polmap, int64_t nt, int64_t nb, int64_t nvchan,
                            int64_t nvpol, void *workspace, size_t workspace_bytes,
                            void *stream);

/* ------------------------------------------------- image formation / FFT -- */
size_t av_fft_workspace_size(int64_t nplanes, int64_t nx, int64_t ny, int precision);

/* grid2image_spheroid_ms4's image step, standard_grid.py:693-708:
 * image[p] = Re(fftshift(ifft2(ifftshift(grid[p])))) / corrTerm * nx*ny /
 * sum_weight[p] for nplanes planes of (nx, ny).  grid AV_C64 or AV_C128;
 * the transform is always an FP64 cuFFT Z2Z; image AV_F32 or AV_F64.
 * sum_weight may be NULL (no division). apply_corr = 0 skips corrTerm. */
size_t av_grid_to_image_workspace_size(int64_t nplanes, int64_t nx, int64_t ny);
int av_grid_to_image(const void *grid, int grid_dtype, const double *sum_weight,
                     void *image, int image_dtype, int64_t nplanes, int64_t nx, int64_t ny,
                     int apply_corr, void *workspace, size_t workspace_bytes, void *stream);

/* fft_lm_to_uv(image / corrTerm) (fft.py:5, gcf_prolate_spheroidal.py:73-79)
 * for nplanes real (nx, ny) planes (AV_F32 / AV_F64) into a complex grid
 * (AV_C64 / AV_C128), FP64 transform; apply_corr = 0 skips the division.  The
 * image -> grid step of the degridding forward model and the adjoint of
 * av_grid_to_image without sum_weight. */
int av_image_to_grid(const void *image, int image_dtype, void *grid, int grid_dtype,
                     int64_t nplanes, int64_t nx, int64_t ny, int apply_corr, void *workspace,
                     size_t workspace_bytes, void *stream);

/* fft_lm_to_uv (fft.py:5) with inverse = 0 and ifft_uv_to_lm (ifft.py:5)
 * with inverse = 1, over the last two axes of nplanes (nx, ny) planes:
 * out = fftshift(fft2 / ifft2(ifftshift(in))).  in/out AV_C64 or AV_C128
 * (same dtype); inverse output is complex (take .real on the host side). */
int av_fft_shifted(const void *in, void *out, int dtype, int64_t nplanes, int64_t nx,
                   int64_t ny, int inverse, void *workspace, size_t workspace_bytes,
                   void *stream);

/* -------------------------------------------------------- imaging weights -- */
/* grid_imaging_weights_jit, grid_imaging_weights.py:93-206, fused with the
 * flag->NaN and polarisation averaging of calculate_imaging_weights.py:183-198:
 * wt (nt, nb, nchan, npol) of wt_dtype; flag same shape uint8 or NULL.
 * density (nchan, 1, n_u, n_v) float64 and sum_weight (nchan, 1) float64 are
 * accumulated.  npol in {1, 2, 4}: 2 averages pols (0,1), 4 averages (0,3). */
int av_weight_density(double *density, double *sum_weight, const double *uvw,
                      const double *freq, const void *wt, int wt_dtype, const uint8_t *flag,
                      int64_t n_u, int64_t n_v, double delta_l, double delta_m, int64_t nt,
                      int64_t nb, int64_t nchan, int64_t npol, void *stream);

/* calculate_briggs_params, briggs_weighting.py:1-31 ("briggs"):
 * factors (2, nplanes): [0] = (5*10^-robust)^2 / (sum(G^2)/sum_weight), [1] = 1.
 * sum(G^2) is an FP64 reduction in a fixed order (deterministic). */
size_t av_briggs_factors_workspace_size(int64_t nplanes);
int av_briggs_factors(const double *density, const double *sum_weight, double *factors,
                      int64_t nplanes, int64_t n_u, int64_t n_v, double robust,
                      void *workspace, size_t workspace_bytes, void *stream);

/* No counterpart in the reference.  av_briggs_factors for callers that may
 * not allocate device memory: a host program that hands this library buffers
 * from a pool it sized at start-up and allows no cudaMalloc/cudaFree on its
 * processing path (an allocation there synchronises the device and can fail
 * mid-run), or a plugin running inside another framework that owns all device
 * memory and passes it only inputs and outputs.  Same arguments and result as
 * av_briggs_factors, without the workspace: the partial sums live in a
 * static device array of this library (AV_BRIGGS_NOALLOC_MAX_PLANES planes,
 * 512 KiB, held on every GPU that loads the library until the process exits).
 * nplanes above the maximum returns AV_ERR_ARG; the call makes no
 * allocation.  The first call on a device looks up that device's copy of the
 * array: make it before any stream capture.  The lookup is kept for the life
 * of the process and does not survive cudaDeviceReset (after a reset the
 * array may sit elsewhere): do not call this function after resetting a
 * device it has been called on.  The stream must belong to the current
 * device (AV_ERR_ARG otherwise).  All calls share the one array,
 * so calls that overlap on the GPU (other streams, other host threads) race;
 * serialise them.  Every partial a call reads it first writes, so the
 * previous call's contents never leak into a result. */
#define AV_BRIGGS_NOALLOC_MAX_PLANES 1024
int av_briggs_factors_noalloc(const double *density, const double *sum_weight, double *factors,
                              int64_t nplanes, int64_t n_u, int64_t n_v, double robust,
                              void *stream);

/* degrid_imaging_weights_jit, grid_imaging_weights.py:285-443, with the
 * input preparation and the tiling to n_pol of calculate_imaging_weights.py
 * (:228-261): out (nt, nb, nchan, npol) of out_dtype gets the imaging weight
 * of each sample (0 off-grid, NaN where flagged).  *err_flag (device int32,
 * zeroed by the caller) is set to 1 where the reference raises ValueError
 * ("NaN in briggs_factors", a NaN factor on a used cell). */
int av_briggs_apply(void *out, int out_dtype, const double *density, const double *factors,
                    const double *uvw, const double *freq, const void *wt, int wt_dtype,
                    const uint8_t *flag, int64_t n_u, int64_t n_v, double delta_l,
                    double delta_m, int64_t nt, int64_t nb, int64_t nchan, int64_t npol,
                    int32_t *err_flag, void *stream);

/* standard_imaging_weight_degrid_jit, standard_grid.py:487-604 (called by
 * standard_imaging_weight_degrid_numpy_wrap, :441-484): imaging_weight (nt,
 * nb, nchan, npol, float64) gets, for every sample whose nearest cell
 * (int(x + 0.5), bounds [0, n)) is on the grid, each polarisation's natural
 * weight (the mean of polarisations 0 and 1 when npol == 2) divided by
 * briggs_factors[0][a] * G[a][cell] + briggs_factors[1][a], a = (chan_map[c],
 * pol_map[p]), where that polarisation's natural weight and G[a][cell] are
 * neither NaN nor zero.  Entries of samples off the grid or with NaN uv are
 * left unchanged (the wrapper passes zeros).  grid_imaging_weight is
 * (g_chan, g_pol, n_u, n_v) of grid_dtype, briggs_factors (2, g_chan, g_pol);
 * chan_map (nchan) and pol_map (npol) are device int32 arrays whose entries
 * the caller keeps in [0, g_chan) and [0, g_pol). */
int av_imaging_weight_degrid(double *imaging_weight, const void *grid_imaging_weight,
                             int grid_dtype, int64_t g_chan, int64_t g_pol,
                             const double *briggs_factors, const double *uvw, const double *freq,
                             const int32_t *chan_map, const int32_t *pol_map,
                             const void *natural_weight, int wt_dtype, int64_t n_u, int64_t n_v,
                             double delta_l, double delta_m, int64_t nt, int64_t nb,
                             int64_t nchan, int64_t npol, void *stream);

/* ------------------------------------------------------------ Hogbom CLEAN -- */
/* hclean::maximg, hclean.cpp:51-81: out[0] = min, out[1] = max over pixels
 * with mask > 0.5 (mask may be NULL).  dtype AV_F32 / AV_F64; out of dtype. */
int av_maximg(const void *image, const void *mask, int dtype, int64_t nx, int64_t ny,
              void *out, void *stream);

/* Persistent state of one Hogbom run (device memory, 256 bytes). */
size_t av_hogbom_state_size(void);
size_t av_hogbom_workspace_size(int64_t nx, int64_t ny, int dtype);

/* hclean::clean, hclean.cpp:106-210 (bindings.cpp:63-208 for the box):
 * runs iterations [iter_begin, iter_end) of Hogbom CLEAN on residual (ny, nx)
 * in place, adding components to model (ny, nx); psf (pny, pnx) with its
 * centre at (pny/2, pnx/2) - pnx = nx, pny = ny is the reference exactly.
 * One cooperative persistent launch; each iteration fuses the PSF
 * subtraction with the next peak search, with one bounded grid barrier.
 * state carries the current peak between calls: pass init_state = 1 on the
 * first call.  On return the host reads (via av_hogbom_state_read) the next
 * iteration number, the peak (px, py, value, |value|) and whether the
 * threshold stopped the loop.  Arithmetic is bit-identical to the reference
 * (no fused multiply-add, first-maximum tie break). */
int av_hogbom_run(void *model, void *residual, const void *psf, const void *mask, int dtype,
                  int64_t nx, int64_t ny, int64_t pnx, int64_t pny, int xbeg, int xend,
                  int ybeg, int yend, int niter, int siter, int iter_begin, int iter_end,
                  double gain, double threshold, double speedup, void *state, int init_state,
                  void *workspace, size_t workspace_bytes, void *stream);

/* Copies the state to the host: out_i[0] = next iteration, [1] = px,
 * [2] = py, [3] = stopped by threshold, [4] = device error code;
 * out_d[0] = peak value, out_d[1] = |peak|.  Synchronises the stream. */
int av_hogbom_state_read(const void *state, int32_t *out_i, double *out_d, void *stream);

/* Sum of |model| over pixels in row-major order with sequential FP32/FP64
 * addition (the total_flux_cleaned of bindings.cpp:181-186).  out one value
 * of dtype. */
size_t av_abs_sum_workspace_size(int64_t n, int dtype);
int av_abs_sum_ordered(const void *model, int dtype, int64_t n, void *out, void *workspace,
                       size_t workspace_bytes, void *stream);

/* ------------------------------------------------- major/minor-cycle imager -- */
/* corr_to_stokes / stokes_to_corr (corr_to_stokes.py:71-138) as used by
 * image_corr_to_stokes and image_stokes_to_corr (:141-305, :307-487):
 * out[k, o, p] = sum_i M[o][i] in[k, i, p] for in (n_outer, n_in, n_pix) and
 * out (n_outer, n_out, n_pix); matrix is the complex n_out x n_in matrix M,
 * row-major, as (re, im) pairs in host memory.  Element types AV_F32 / AV_F64
 * / AV_C64 / AV_C128; a real output keeps the real part (the .real of
 * image_corr_to_stokes for real images).  Terms with a zero coefficient are
 * left out and nothing is fused, so the reference's tables give numpy's
 * results exactly. */
int av_pol_transform(const void *in, int in_dtype, void *out, int out_dtype,
                     const double *matrix, int n_in, int n_out, int64_t n_outer, int64_t n_pix,
                     void *stream);

/* np.argmax(np.abs(x)) (mode 0) or np.argmax(x) (mode 1) over n values
 * (AV_F32 / AV_F64): first index of the maximum, NaN above every number.
 * Device outputs: *out_index, and *out_value = x at that index (signed), the
 * value image_peak_residual returns (image_statistics.py:83-86). */
size_t av_argmax_workspace_size(int64_t n);
int av_argmax(const void *x, int dtype, int64_t n, int mode, int64_t *out_index,
              double *out_value, void *workspace, size_t workspace_bytes, void *stream);

/* max_sidelobe of extract_main_lobe(npix_window = (win0, win1), threshold,
 * psf) (psf_gaussian_fit.py:46-126) for one (ny, nx) PSF plane: the main lobe
 * is the 4-connected set of pixels above threshold x peak, inside the window
 * around the PSF peak, that holds the window maximum; the result is the
 * maximum over the plane with the main lobe counted as 0.  out (device, 2
 * doubles): out[0] = max_sidelobe, out[1] = 0, or out[0] = NaN and out[1] = 1
 * for a negative threshold x peak (the reference would label the whole image
 * outside the window).  Windows up to 16384 pixels. */
size_t av_psf_sidelobe_workspace_size(int64_t ny, int64_t nx, int win0, int win1);
int av_psf_sidelobe(const void *psf, int dtype, int64_t ny, int64_t nx, int win0, int win1,
                    double threshold, double *out, void *workspace, size_t workspace_bytes,
                    void *stream);

/* Per-plane sums in FP64 of x (n_planes, n_pix), AV_F32 / AV_F64: the model
 * flux of deconvolve (deconvolution.py:262, np.sum of a plane); out (device)
 * n_planes doubles.  Up to 65535 planes. */
size_t av_plane_sum_workspace_size(int64_t n_planes, int64_t n_pix);
int av_plane_sum(const void *x, int dtype, int64_t n_planes, int64_t n_pix, double *out,
                 void *workspace, size_t workspace_bytes, void *stream);

/* correct_fft_to_uv / correct_ifft_to_lm (standard_image_grid_preparation.py:
 * 380-492): x (n_planes, n_pix) of AV_F32 / AV_F64 / AV_C64 / AV_C128, in
 * place.  mode 0: x /= s (correct_fft_to_uv, s = u x v); mode 1: x *= s
 * (correct_ifft_to_lm without the spheroid correction, s = l x m); mode 2:
 * x *= s / (corr[pix] * w[plane]) (with it: corr the grid-correction term of
 * create_prolate_spheroidal_kernel, n_pix doubles, w the planes'
 * normalisations, n_planes doubles).  Modes 0 and 1 compute in the data's
 * precision, mode 2 forms its factor and the product in FP64, as numpy does;
 * a complex x is scaled as numpy divides or multiplies it by the complex
 * (s, 0) (division: both parts times the reciprocal of s), which also fixes
 * the signs of zeros and the NaNs of infinite parts. */
int av_plane_rescale(void *x, int dtype, int64_t n_planes, int64_t n_pix, int mode, double s,
                     const double *corr, const double *w, void *stream);

/* apply_pb (standard_image_grid_preparation.py:236-275) through _mult_div
 * (:278-309): x (nt, nc, np, n_pix) of AV_F32 / AV_F64 / AV_C64 / AV_C128
 * multiplied (multiply != 0) or divided in place by the primary beam pb
 * (pt, pc, pp, n_pix) of AV_F32 / AV_F64; x's plane (t, c, p) uses pb's plane
 * with each index 0 where pb's extent differs from x's (equal shapes map
 * plane to plane).  numpy's arithmetic for x op= pb (the promoted precision,
 * rounded to x's type; a complex x as numpy multiplies or divides by
 * (pb, 0)); dividing by a zero beam leaves NaN, (NaN, 0) for a complex x. */
int av_apply_pb(void *x, int x_dtype, int64_t nt, int64_t nc, int64_t npl, const void *pb,
                int pb_dtype, int64_t pt, int64_t pc, int64_t pp, int64_t n_pix, int multiply,
                void *stream);

/* compute_residual_visibilities (imager.py:82-85): out = vis - model over n
 * complex values (AV_C64 / AV_C128); out may alias vis or model. */
int av_vis_residual(const void *vis, const void *model, void *out, int dtype, int64_t n,
                    void *stream);

/* ------------------------------------------------- mosaic / A-projection -- */
/* conv_kernel x phase_gradient[0] (mosaic_grid.py:56-58, :384): out
 * (n_cf, conv_u, conv_v) complex128 from a float64 or complex128 kernel of
 * that shape and one (conv_u, conv_v) complex128 phase gradient; products
 * without fused multiply-add. */
int av_cf_phase_product(const void *conv_kernel, int kernel_dtype, const void *phase_gradient,
                        void *out, int64_t n_cf, int64_t conv_u, int64_t conv_v, void *stream);

/* Airy-disk primary beams of make_pb_symmetric.py: airy_disk (:1-58) and
 * casa_airy_disk (:61-125) with rorder = 0, out (nx, ny, n_freq, n_pol,
 * n_dish); airy_disk_rorder (:128-190) and casa_airy_disk_rorder (:193-280)
 * with rorder = 1, out (n_dish, n_freq, n_pol, nx, ny); casa selects the
 * CASA blockage formula.  Pixel offsets from (cx, cy) times (cell_x, cell_y)
 * radians, freq (n_freq) device float64 in Hz, dish and blockage diameters
 * (n_dish <= 16) in host memory, metres; the pattern raised to ipower (0-8),
 * 1 at the centre; J1 is CUDA's j1 (a few ulp from scipy's). */
int av_airy_pattern(double *out, const double *dish_diameters, const double *blockage_diameters,
                    int64_t n_dish, const double *freq, int64_t n_freq, int64_t n_pol,
                    int64_t nx, int64_t ny, int64_t cx, int64_t cy, double cell_x,
                    double cell_y, int ipower, int casa, int rorder, void *stream);

/* mosaic_grid_jit (mosaic_grid.py:307-486): grid (n_img_chan, n_img_pol,
 * n_u, n_v) complex128 and sum_weight (n_img_chan, n_img_pol) += the
 * samples' windows of the convolution function cf (n_cf_baseline,
 * n_cf_chan, n_cf_pol, conv_u, conv_v) complex128 (phase gradient applied,
 * see av_cf_phase_product), chosen per sample by cf_baseline_map (nb),
 * cf_chan_map (nchan) and cf_pol_map (npol); window sizes support
 * (n_cf_baseline, n_cf_chan, n_cf_pol, 2); max_support = np.max(support)
 * sets the grid-edge test.  vis (nt, nb, nchan, npol) complex128 (NULL with
 * do_psf), weight float64 of the same shape, uvw (nt, nb, 3), freq (nchan).
 * sum_weight gets w Re(norm) with do_psf, else w Re(norm^2), norm the sum of
 * the window.  Window taps that fall outside cf (the reference reads past the
 * array there) are left out. */
int av_mosaic_grid(void *grid, double *sum_weight, int do_psf, const void *vis,
                   const double *weight, const double *uvw, const double *freq,
                   const int32_t *chan_map, const int32_t *pol_map,
                   const int32_t *cf_baseline_map, const int32_t *cf_chan_map,
                   const int32_t *cf_pol_map, const void *cf, int64_t n_cf_baseline,
                   int64_t n_cf_chan, int64_t n_cf_pol, int64_t conv_u, int64_t conv_v,
                   const int32_t *support, int max_support, int64_t n_u, int64_t n_v,
                   double delta_l, double delta_m, int os_u, int os_v, int64_t nt, int64_t nb,
                   int64_t nchan, int64_t npol, int64_t n_img_chan, int64_t n_img_pol,
                   void *stream);

/* Binned mosaic gridding, the same sums as av_mosaic_grid: _plan bins the
 * samples (cells and kernel offsets, the mosaic's edge margin of
 * max_support cells) into the workspace, _execute grids with that plan; a
 * persistent CTA per SM keeps an FP64 sub-grid per tile in shared memory.
 * Needs max_support <= 32 (the largest window; support entries above it are
 * skipped), os_u == os_v <= 254, n_img_pol <= 4 and
 * (31 + max_support)^2 x n_img_pol x 16 bytes of shared memory <= 220 KiB.
 * Executes on one plan must not overlap (stream order is enough). */
size_t av_mosaic_tiled_workspace_size(int64_t nt, int64_t nb, int64_t nchan, int64_t n_u,
                                      int64_t n_v, int64_t n_img_chan, int max_support);
int av_mosaic_tiled_plan(const double *uvw, const double *freq, const int32_t *chan_map,
                         int64_t n_u, int64_t n_v, double delta_l, double delta_m,
                         int max_support, int oversampling, int64_t nt, int64_t nb,
                         int64_t nchan, int64_t n_img_chan, void *workspace,
                         size_t workspace_bytes, void *stream);
int av_mosaic_tiled_execute(void *grid, double *sum_weight, int do_psf, const void *vis,
                            const double *weight, const double *uvw, const double *freq,
                            const int32_t *chan_map, const int32_t *pol_map,
                            const int32_t *cf_baseline_map, const int32_t *cf_chan_map,
                            const int32_t *cf_pol_map, const void *cf, int64_t n_cf_baseline,
                            int64_t n_cf_chan, int64_t n_cf_pol, int64_t conv_u, int64_t conv_v,
                            const int32_t *support, int max_support, int64_t n_u, int64_t n_v,
                            double delta_l, double delta_m, int os_u, int os_v, int64_t nt,
                            int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                            int64_t n_img_pol, void *workspace, size_t workspace_bytes,
                            void *stream);

/* aperture_grid_jit (mosaic_grid.py:13-153): every sample that passes the
 * grid-edge test adds weight x its function window at the grid centre
 * (and weight x Re(norm) to sum_weight); the weights are summed per
 * (cf baseline, channel, polarisation) first.  Same arguments as
 * av_mosaic_grid (do_psf and vis unused) plus a workspace of
 * av_aperture_grid_workspace_size bytes. */
size_t av_aperture_grid_workspace_size(int64_t n_cf_baseline, int64_t nchan, int64_t npol);
int av_aperture_grid(void *grid, double *sum_weight, int do_psf, const void *vis,
                     const double *weight, const double *uvw, const double *freq,
                     const int32_t *chan_map, const int32_t *pol_map,
                     const int32_t *cf_baseline_map, const int32_t *cf_chan_map,
                     const int32_t *cf_pol_map, const void *cf, int64_t n_cf_baseline,
                     int64_t n_cf_chan, int64_t n_cf_pol, int64_t conv_u, int64_t conv_v,
                     const int32_t *support, int max_support, int64_t n_u, int64_t n_v,
                     double delta_l, double delta_m, int os_u, int os_v, int64_t nt,
                     int64_t nb, int64_t nchan, int64_t npol, int64_t n_img_chan,
                     int64_t n_img_pol, void *workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AV200_H */
