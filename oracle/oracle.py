"""ctypes + numpy front end of the CPU oracle (test infrastructure only).

Function names and argument meanings follow the reference functions they
restate; every array is converted to the contiguous dtype the C code expects.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i = ctypes.c_int
_d = ctypes.c_double
_f = ctypes.c_float

C_LIGHT = 299792458.0


def lib():
    """Load (building first if needed) liboracle.so."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "av_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["sh", os.path.join(_HERE, "build.sh")])
    L = ctypes.CDLL(path)
    L.orc_pswf.argtypes = [_dp, _i64, _dp, _dp]
    L.orc_cgk_1d.argtypes = [_i, _i, _dp]
    L.orc_corr_term.argtypes = [_i64, _i64, _dp]
    L.orc_standard_grid.argtypes = [_vp, _i, _dp, _i, _i, _vp, _dp, _dp, _i64p, _i64p, _dp,
                                    _dp, _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64, _i64,
                                    _i64]
    L.orc_standard_grid_mt.argtypes = [_vp, _dp, _i, _vp, _dp, _dp, _i64p, _i64p, _dp, _dp,
                                       _i64, _i64, _d, _d, _i, _i, _i64, _i64, _i64, _i64,
                                       _i64, _i64, _i]
    L.orc_standard_grid_mt.restype = _i
    L.orc_dgrid.argtypes = [_dp, _dp, _vp, _u8p, _dp, _dp, _vp, _i64, _i64, _i64, _i64, _dp,
                            _d, _i, _i, _dp, _i64p, _i64p, _i64, _i64, _i64, _i64, _i]
    L.orc_dgrid_adjoint.argtypes = [_dp, _dp, _vp, _u8p, _dp, _dp, _vp, _i64, _i64, _i64, _i64,
                                    _dp, _d, _i, _i, _dp, _i64p, _i64p, _i64, _i64, _i64, _i64]
    L.orc_grid_imaging_weights.argtypes = [_dp, _i64, _dp, _dp, _dp, _i64p, _dp, _i64, _i64,
                                           _d, _d, _i64, _i64, _i64, _i64]
    L.orc_degrid_imaging_weights.argtypes = [_dp, _dp, _i64, _i64, _dp, _dp, _dp, _i64p,
                                             _i64p, _i64, _dp, _i64, _i64, _d, _d, _i64, _i64,
                                             _i64, _i64]
    L.orc_degrid_imaging_weights.restype = _i
    L.orc_imaging_weight_degrid.argtypes = [_dp, _dp, _i64, _i64, _dp, _dp, _dp, _i64p, _i64p,
                                            _dp, _i64, _i64, _d, _d, _i64, _i64, _i64, _i64]
    L.orc_imaging_weight_degrid.restype = None
    L.orc_hogbom_f32.argtypes = [_fp, _fp, _fp, _i, _i, _i, _fp, _i, _i, _i, _i, _i, _i, _i,
                                 _i, _f, _f, _f, _dp, _i32p, _dp]
    L.orc_hogbom_f32.restype = _i
    L.orc_hogbom_f64.argtypes = [_dp, _dp, _dp, _i, _i, _i, _dp, _i, _i, _i, _i, _i, _i, _i,
                                 _i, _d, _d, _d, _dp, _i32p, _dp]
    L.orc_hogbom_f64.restype = _i
    L.orc_maximg_f32.argtypes = [_fp, _i, _fp, _i, _i, _fp, _fp]
    L.orc_maximg_f64.argtypes = [_dp, _i, _dp, _i, _i, _dp, _dp]
    L.orc_num_threads.restype = _i
    L.orc_mosaic_grid.argtypes = [_vp, _dp, _i, _vp, _dp, _dp, _i64p, _i64p, _i64p, _i64p,
                                  _i64p, _dp, _vp, _i64, _i64, _i64, _i64, _i64p, _i64, _i64,
                                  _i64, _d, _d, _i64, _i64, _i64, _i64, _i64, _i64, _i64]
    _LIB = L
    return L


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a, t):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------------------
# PSWF (gcf_prolate_spheroidal.py)
# ----------------------------------------------------------------------------
def prolate_spheroidal_function(u):
    """Restates gcf_prolate_spheroidal.py:102-158: returns (grdsf, (1-u^2) grdsf)."""
    u = _c(u, np.float64)
    g = np.empty_like(u)
    k = np.empty_like(u)
    lib().orc_pswf(_p(u, _dp), u.size, _p(g, _dp), _p(k, _dp))
    return g, k


def create_prolate_spheroidal_kernel_1D(oversampling, support):
    """Restates gcf_prolate_spheroidal.py:87-99."""
    out = np.empty(oversampling * (support // 2 + 1), dtype=np.float64)
    lib().orc_cgk_1d(int(oversampling), int(support), _p(out, _dp))
    return out


def corr_term(n_uv):
    """Grid-correction image of gcf_prolate_spheroidal.py:73-79, shape (nx, ny)."""
    nx, ny = int(n_uv[0]), int(n_uv[1])
    out = np.empty((nx, ny), dtype=np.float64)
    lib().orc_corr_term(nx, ny, _p(out, _dp))
    return out


# ----------------------------------------------------------------------------
# Gridder (standard_grid.py)
# ----------------------------------------------------------------------------
def standard_grid_jit(grid, sum_weight, do_psf, do_imaging_weight, vis_data, uvw, freq_chan,
                      chan_map, pol_map, weight, cgk_1D, n_uv, delta_lm, support,
                      oversampling):
    """Restates standard_grid_jit (standard_grid.py:246-432); updates grid and
    sum_weight in place.  grid must be C-contiguous complex128 or float64."""
    assert grid.flags.c_contiguous and grid.dtype in (np.complex128, np.float64)
    assert sum_weight.flags.c_contiguous and sum_weight.dtype == np.float64
    nt, nb = uvw.shape[:2]
    nchan, npol = weight.shape[2], weight.shape[3]
    vis = _c(vis_data if not do_psf else np.zeros(weight.shape, np.complex128), np.complex128)
    uvw = _c(uvw, np.float64)
    freq = _c(freq_chan, np.float64)
    cm = _c(chan_map, np.int64)
    pm = _c(pol_map, np.int64)
    w = _c(weight, np.float64)
    cgk = _c(cgk_1D, np.float64)
    lib().orc_standard_grid(grid.ctypes.data, int(grid.dtype == np.complex128),
                            _p(sum_weight, _dp), int(bool(do_psf)),
                            int(bool(do_imaging_weight)), vis.ctypes.data, _p(uvw, _dp),
                            _p(freq, _dp), _p(cm, _i64p), _p(pm, _i64p), _p(w, _dp),
                            _p(cgk, _dp), int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                            float(delta_lm[1]), int(support), int(oversampling), nt, nb, nchan,
                            npol, grid.shape[1])


def standard_grid(vis_data, uvw, weight, freq_chan, cgk_1D, image_size, cell_size,
                  oversampling=100, support=7, do_psf=False, chan_mode="continuum",
                  nthreads=1, rows=False):
    """standard_grid_numpy_wrap (standard_grid.py:88-165) on fresh arrays:
    returns (grid complex128, sum_weight).  nthreads > 1 (or 0: every OpenMP
    thread) uses the row-owner OpenMP variant: the grid is bit-identical to
    the serial one, sum_weight may differ in the last bits (it is summed per
    thread first).  rows=True takes that variant at one thread too (the CPU
    baseline's one-thread rate)."""
    nchan, npol = weight.shape[2], weight.shape[3]
    if chan_mode == "cube":
        n_img_chan, chan_map = nchan, np.arange(nchan, dtype=np.int64)
    else:
        n_img_chan, chan_map = 1, np.zeros(nchan, dtype=np.int64)
    pol_map = np.arange(npol, dtype=np.int64)
    nu, nv = int(image_size[0]), int(image_size[1])
    grid = np.zeros((n_img_chan, npol, nu, nv), dtype=np.complex128)
    sw = np.zeros((n_img_chan, npol), dtype=np.float64)
    if nthreads == 1 and not rows:
        standard_grid_jit(grid, sw, do_psf, False, vis_data, uvw, freq_chan, chan_map, pol_map,
                          weight, cgk_1D, np.array([nu, nv]), cell_size, support, oversampling)
        return grid, sw
    nt, nb = uvw.shape[:2]
    vis = _c(vis_data if not do_psf else np.zeros(weight.shape, np.complex128), np.complex128)
    uvw = _c(uvw, np.float64)
    freq = _c(freq_chan, np.float64)
    w = _c(weight, np.float64)
    cgk = _c(cgk_1D, np.float64)
    got = lib().orc_standard_grid_mt(grid.ctypes.data, _p(sw, _dp), int(bool(do_psf)),
                                     vis.ctypes.data, _p(uvw, _dp), _p(freq, _dp),
                                     _p(chan_map, _i64p), _p(pol_map, _i64p), _p(w, _dp),
                                     _p(cgk, _dp), nu, nv, float(cell_size[0]),
                                     float(cell_size[1]), int(support), int(oversampling), nt,
                                     nb, nchan, npol, n_img_chan, npol, int(nthreads))
    if got == -2:
        raise ValueError(f"oracle: support {support} outside the row-owner gridder's range")
    if got < 0:
        raise MemoryError("oracle: the per-sample cell table could not be allocated")
    return grid, sw


def grid_to_image(grid, sum_weight, n_uv=None):
    """Image formation of grid2image_spheroid_ms4 (standard_grid.py:693-708):
    Re(fftshift(ifft2(ifftshift(g)))) / corrTerm * nx * ny / sumwt per plane."""
    nx, ny = grid.shape[-2:]
    ct = corr_term((nx, ny))
    out = np.empty(grid.shape, dtype=np.float64)
    for c in range(grid.shape[0]):
        for p in range(grid.shape[1]):
            out[c, p] = (np.real(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(grid[c, p]))))
                         / ct * nx * ny / sum_weight[c, p])
    return out


def fft_lm_to_uv(ary, axes):
    """fft.py:5-18."""
    return np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(ary, axes=axes), axes=axes), axes=axes)


def ifft_uv_to_lm(ary, axes):
    """ifft.py:5-18."""
    return np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(ary, axes=axes), axes=axes),
                           axes=axes).real


# ----------------------------------------------------------------------------
# Degridder (standard_degrid.py)
# ----------------------------------------------------------------------------
def dgrid_numba(uvw, dphase, values, flag, scale, offset, grid, freq, c, support, sampling,
                convFunc, chanmap, polmap, nthreads=1):
    """Restates dgrid_numba (standard_degrid.py:388-485); values += in place.
    values must be C-contiguous complex128."""
    assert values.flags.c_contiguous and values.dtype == np.complex128
    nt, nb, nvchan, nvpol = values.shape
    g = _c(grid, np.complex128)
    uvw = _c(uvw, np.float64)
    dph = _c(dphase, np.float64)
    fl = _c(flag, np.uint8)
    sc = _c(scale, np.float64)
    off = _c(offset, np.float64)
    fr = _c(freq, np.float64)
    cf = _c(convFunc, np.float64)
    cm = _c(chanmap, np.int64)
    pm = _c(polmap, np.int64)
    lib().orc_dgrid(_p(uvw, _dp), _p(dph, _dp), values.ctypes.data, _p(fl, _u8p), _p(sc, _dp),
                    _p(off, _dp), g.ctypes.data, g.shape[0], g.shape[1], g.shape[2], g.shape[3],
                    _p(fr, _dp), float(c), int(support), int(sampling), _p(cf, _dp),
                    _p(cm, _i64p), _p(pm, _i64p), nt, nb, nvchan, nvpol, int(nthreads))


def degrid(grid, uvw, freq, pixelincr, flag=None, support=7, sampling=100, nthreads=1):
    """degrid_spheroid_ms4's call of dgrid_numba (standard_degrid.py:568-602) on
    plain arrays: returns the model visibilities (nt, nb, nfreq, npol)."""
    nt, nb = uvw.shape[:2]
    nfreq = len(freq)
    if flag is None:
        raise ValueError("flag array required (shape nt, nb, nfreq, npol)")
    npolv = flag.shape[3]
    nx, ny = grid.shape[-2:]
    scale = np.array([-pixelincr[0] * nx, -pixelincr[1] * ny, 0.0], dtype=np.float64)
    offset = np.array([nx / 2, ny / 2, 0.0], dtype=np.float64)
    cf = create_prolate_spheroidal_kernel_1D(sampling, support)
    nchan, npol = grid.shape[0], grid.shape[1]
    chanmap = (np.arange(nfreq) / nfreq * nchan).astype(np.int64)
    polmap = np.round(np.arange(npolv) % npol).astype(np.int64)
    values = np.zeros((nt, nb, nfreq, npolv), dtype=np.complex128)
    dgrid_numba(uvw, np.zeros((nt, nb)), values, flag, scale, offset, grid, freq, C_LIGHT,
                support, sampling, cf, chanmap, polmap, nthreads=nthreads)
    return values


def dgrid_adjoint(uvw, values, flag, scale, offset, grid_shape, freq, support, sampling,
                  convFunc, chanmap, polmap, dphase=None, c=C_LIGHT):
    """Transpose of dgrid_numba: a fresh complex128 grid of grid_shape."""
    g = np.zeros(grid_shape, dtype=np.complex128)
    nt, nb, nvchan, nvpol = values.shape
    v = _c(values, np.complex128)
    uvw = _c(uvw, np.float64)
    fl = None if flag is None else _c(flag, np.uint8)
    dph = None if dphase is None else _c(dphase, np.float64)
    lib().orc_dgrid_adjoint(_p(uvw, _dp), None if dph is None else _p(dph, _dp), v.ctypes.data,
                            None if fl is None else _p(fl, _u8p), _p(_c(scale, np.float64), _dp),
                            _p(_c(offset, np.float64), _dp), g.ctypes.data, g.shape[0], g.shape[1],
                            g.shape[2], g.shape[3], _p(_c(freq, np.float64), _dp), float(c),
                            int(support), int(sampling), _p(_c(convFunc, np.float64), _dp),
                            _p(_c(chanmap, np.int64), _i64p), _p(_c(polmap, np.int64), _i64p), nt,
                            nb, nvchan, nvpol)
    return g


# ----------------------------------------------------------------------------
# Imaging weights (grid_imaging_weights.py, briggs_weighting.py)
# ----------------------------------------------------------------------------
def grid_imaging_weights_jit(grid, sum_weight, uvw, freq_chan, chan_map, data_weights, n_uv,
                             delta_lm):
    """Restates grid_imaging_weights_jit (grid_imaging_weights.py:93-206)."""
    assert grid.flags.c_contiguous and grid.dtype == np.float64
    nt, nb = uvw.shape[:2]
    nchan, npol = data_weights.shape[2], data_weights.shape[3]
    uvw = _c(uvw, np.float64)
    fr = _c(freq_chan, np.float64)
    cm = _c(chan_map, np.int64)
    dw = _c(data_weights, np.float64)
    lib().orc_grid_imaging_weights(_p(grid, _dp), grid.shape[1], _p(sum_weight, _dp),
                                   _p(uvw, _dp), _p(fr, _dp), _p(cm, _i64p), _p(dw, _dp),
                                   int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                                   float(delta_lm[1]), nt, nb, nchan, npol)


def degrid_imaging_weights_jit(imaging_weight, grid_imaging_weight, briggs_factors, uvw,
                               freq_chan, chan_map, pol_map, data_weight, n_uv, delta_lm):
    """Restates degrid_imaging_weights_jit (grid_imaging_weights.py:285-443)."""
    assert imaging_weight.flags.c_contiguous and imaging_weight.dtype == np.float64
    nt, nb = uvw.shape[:2]
    nchan, npol = data_weight.shape[2], data_weight.shape[3]
    g = _c(grid_imaging_weight, np.float64)
    bf = _c(briggs_factors, np.float64).reshape(2, g.shape[0], g.shape[1])
    uvw = _c(uvw, np.float64)
    fr = _c(freq_chan, np.float64)
    cm = _c(chan_map, np.int64)
    pm = _c(pol_map, np.int64)
    dw = _c(data_weight, np.float64)
    rc = lib().orc_degrid_imaging_weights(_p(imaging_weight, _dp), _p(g, _dp), g.shape[0],
                                          g.shape[1], _p(bf, _dp), _p(uvw, _dp), _p(fr, _dp),
                                          _p(cm, _i64p), _p(pm, _i64p), len(pm), _p(dw, _dp),
                                          int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                                          float(delta_lm[1]), nt, nb, nchan, npol)
    if rc != 0:
        raise ValueError("NaN in briggs_factors")


def standard_imaging_weight_degrid_jit(imaging_weight, grid_imaging_weight, briggs_factors, uvw,
                                       freq_chan, chan_map, pol_map, natural_imaging_weight,
                                       n_uv, delta_lm):
    """Restates standard_imaging_weight_degrid_jit (standard_grid.py:487-604),
    in place into the float64 array imaging_weight."""
    assert imaging_weight.flags.c_contiguous and imaging_weight.dtype == np.float64
    nt, nb = uvw.shape[:2]
    nchan, npol = natural_imaging_weight.shape[2], natural_imaging_weight.shape[3]
    g = _c(grid_imaging_weight, np.float64)
    bf = _c(briggs_factors, np.float64).reshape(2, g.shape[0], g.shape[1])
    uvw = _c(uvw, np.float64)
    fr = _c(freq_chan, np.float64)
    cm = _c(chan_map, np.int64)
    pm = _c(pol_map, np.int64)
    nw = _c(natural_imaging_weight, np.float64)
    lib().orc_imaging_weight_degrid(_p(imaging_weight, _dp), _p(g, _dp), g.shape[0], g.shape[1],
                                    _p(bf, _dp), _p(uvw, _dp), _p(fr, _dp), _p(cm, _i64p),
                                    _p(pm, _i64p), _p(nw, _dp), int(n_uv[0]), int(n_uv[1]),
                                    float(delta_lm[0]), float(delta_lm[1]), nt, nb, nchan, npol)


def standard_imaging_weight_degrid_numpy_wrap(grid_imaging_weight, uvw, natural_imaging_weight,
                                              briggs_factors, freq_chan, grid_params):
    """Restates standard_imaging_weight_degrid_numpy_wrap (standard_grid.py:441-484)."""
    n_chan, n_pol = natural_imaging_weight.shape[2], natural_imaging_weight.shape[3]
    out = np.zeros(natural_imaging_weight.shape, dtype=np.double)
    standard_imaging_weight_degrid_jit(out, grid_imaging_weight, briggs_factors, uvw, freq_chan,
                                       np.arange(n_chan), np.arange(n_pol),
                                       natural_imaging_weight, grid_params["image_size_padded"],
                                       grid_params["cell_size"])
    return out


def calculate_briggs_params(grid, sum_weight, params):
    """Restates briggs_weighting.py:1-31."""
    if params["weighting"] == "briggs":
        robust = params["robust"]
        bf = np.ones((2,) + sum_weight.shape)
        sq = np.sum(grid ** 2, axis=(2, 3))
        with np.errstate(invalid="ignore", divide="ignore"):
            bf[0, :, :] = (np.square(5.0 * 10.0 ** (-robust)) / (sq / sum_weight))[None, None]
        return bf
    if params["weighting"] == "briggs_abs":
        robust = params["robust"]
        bf = np.ones((2,) + sum_weight.shape)
        bf[0] = bf[0] * np.square(robust)
        bf[1] = bf[1] * 2.0 * np.square(params["briggs_abs_noise"])
        return bf
    bf = np.zeros((2, 1, 1) + sum_weight.shape)
    bf[0] = np.ones((1, 1, 1) + sum_weight.shape)
    return bf


def imaging_weights(uvw, weight, flag, freq, image_size, cell_size, robust=0.5):
    """calculate_imaging_weights (calculate_imaging_weights.py:166-261) on plain
    arrays for Briggs weighting: returns (imaging weights tiled to n_pol,
    density grid, sum_weight, briggs factors)."""
    w = np.array(weight, dtype=np.float64, copy=True)
    w[flag == 1] = np.nan
    if w.shape[3] == 2:
        w = ((w[..., 0] + w[..., 1]) / 2)[..., None]
    elif w.shape[3] == 4:
        w = ((w[..., 0] + w[..., 3]) / 2)[..., None]
    nchan = len(freq)
    nu, nv = int(image_size[0]), int(image_size[1])
    G = np.zeros((nchan, 1, nu, nv), dtype=np.float64)
    sw = np.zeros((nchan, 1), dtype=np.float64)
    grid_imaging_weights_jit(G, sw, uvw, freq, np.arange(nchan), w, np.array([nu, nv]),
                             cell_size)
    bf = calculate_briggs_params(G, sw, {"weighting": "briggs", "robust": robust})
    iw = np.zeros(w.shape, dtype=np.float64)
    degrid_imaging_weights_jit(iw, G, bf, uvw, freq, np.arange(nchan), np.arange(1), w,
                               np.array([nu, nv]), cell_size)
    npol = weight.shape[3]
    return np.tile(iw, (1, 1, 1, npol)), G, sw, bf


# ----------------------------------------------------------------------------
# Hogbom (hclean.cpp)
# ----------------------------------------------------------------------------
def hogbom_clean(dirty, psf, mask=None, clean_box=(-1, -1, -1, -1), max_iter=100,
                 start_iter=0, gain=0.1, threshold=0.0, speedup=0.0):
    """Restates hclean::clean (hclean.cpp:106-210) with the box parsing of
    bindings.cpp:110-128.  psf may be larger than dirty (centre at its
    (ny/2, nx/2)).  Returns dict(model_image, residual_image,
    iterations_performed, components (n, 3): px, py, pv)."""
    f32 = dirty.dtype == np.float32
    dt = np.float32 if f32 else np.float64
    r = np.array(dirty, dtype=dt, copy=True, order="C")
    ps = _c(psf, dt)
    ny, nx = r.shape
    pny, pnx = ps.shape
    model = np.zeros_like(r)
    xbeg, xend, ybeg, yend = 0, nx, 0, ny
    if len(clean_box) == 4:
        xbeg, xend, ybeg, yend = (int(v) for v in clean_box)
        xbeg = 0 if xbeg == -1 else xbeg
        xend = nx if xend == -1 else xend
        ybeg = 0 if ybeg == -1 else ybeg
        yend = ny if yend == -1 else yend
        xbeg = max(0, min(xbeg, nx - 1))
        xend = max(xbeg + 1, min(xend, nx))
        ybeg = max(0, min(ybeg, ny - 1))
        yend = max(ybeg + 1, min(yend, ny))
    domask = 0
    m = np.zeros(1, dtype=dt)
    if mask is not None and np.asarray(mask).size > 0:
        domask = 1
        m = _c(mask, dt)
    comps = np.zeros((max(max_iter - start_iter, 1), 3), dtype=np.float64)
    peak = (ctypes.c_int * 2)()
    mv = ctypes.c_double()
    fp = _fp if f32 else _dp
    fn = lib().orc_hogbom_f32 if f32 else lib().orc_hogbom_f64
    it = fn(_p(model, fp), _p(r, fp), _p(ps, fp), pnx, pny, domask, _p(m, fp), nx, ny, xbeg,
            xend, ybeg, yend, int(max_iter), int(start_iter), gain, threshold, speedup,
            _p(comps, _dp), peak, ctypes.byref(mv))
    return {"model_image": model, "residual_image": r, "iterations_performed": it,
            "components": comps[:max(it - start_iter, 0)], "last_peak": (peak[0], peak[1]),
            "last_value": mv.value}


def maximg(image, mask=None):
    """Restates hclean::maximg (hclean.cpp:51-81): returns (fmin, fmax)."""
    f32 = image.dtype == np.float32
    dt = np.float32 if f32 else np.float64
    im = _c(image, dt)
    ny, nx = im.shape
    domask = 0
    m = np.zeros(1, dtype=dt)
    if mask is not None and np.asarray(mask).size > 0:
        domask = 1
        m = _c(mask, dt)
    if f32:
        a, b = ctypes.c_float(), ctypes.c_float()
        lib().orc_maximg_f32(_p(im, _fp), domask, _p(m, _fp), nx, ny, ctypes.byref(a),
                             ctypes.byref(b))
        return np.float32(a.value), np.float32(b.value)
    a, b = ctypes.c_double(), ctypes.c_double()
    lib().orc_maximg_f64(_p(im, _dp), domask, _p(m, _dp), nx, ny, ctypes.byref(a),
                         ctypes.byref(b))
    return a.value, b.value


def mosaic_grid(grid, sum_weight, do_psf, vis, uvw, freq, chan_map, pol_map, cfb_map, cfc_map,
                cfp_map, weight, cf, support, n_uv, delta_lm, oversampling):
    """Restates mosaic_grid_jit (mosaic_grid.py:307-486) with cf the
    convolution function already multiplied by phase_gradient[0]; grid
    (complex128) and sum_weight are updated in place."""
    assert grid.flags.c_contiguous and grid.dtype == np.complex128
    nt, nb, nchan, npol = weight.shape
    v = _c(vis if not do_psf else np.zeros(weight.shape, np.complex128), np.complex128)
    cfa = _c(cf, np.complex128)
    sup = _c(support, np.int64)
    n_cfb, n_cfc, n_cfp, cu, cv = cfa.shape
    os_ = np.broadcast_to(np.asarray(oversampling, dtype=np.int64), (2,))
    maps = [_c(m, np.int64) for m in (chan_map, pol_map, cfb_map, cfc_map, cfp_map)]
    lib().orc_mosaic_grid(grid.ctypes.data, _p(sum_weight, _dp), int(bool(do_psf)),
                          v.ctypes.data, _p(_c(uvw, np.float64), _dp),
                          _p(_c(freq, np.float64), _dp), *[_p(m, _i64p) for m in maps],
                          _p(_c(weight, np.float64), _dp), cfa.ctypes.data, n_cfc, n_cfp, cu, cv,
                          _p(sup, _i64p), int(np.max(sup)), int(n_uv[0]), int(n_uv[1]),
                          float(delta_lm[0]), float(delta_lm[1]), int(os_[0]), int(os_[1]), nt,
                          nb, nchan, npol, grid.shape[1])


def num_threads():
    return lib().orc_num_threads()
