"""CPU restatement of the reference's major/minor-cycle imager (test
infrastructure: only tests and the benchmark's CPU baseline use it).

Follows src/astroviper/core/imaging/imager.py:108-351 step by step with the
oracle's C kernels for gridding, degridding and Hogbom CLEAN and numpy for
the rest:
  * corr_to_stokes.py:71-487   polarisation products (numpy matmul after a
                               moveaxis, the 2-pol case through zero-filled
                               cross hands);
  * psf_gaussian_fit.py:46-126 max_sidelobe of extract_main_lobe
                               (scipy.ndimage.label, 4-connectivity);
  * deconvolution.py:123-329   per-plane Hogbom with the statistics;
  * standard_grid.py:607-708,  make_point_spread_function.py:1-79,
    standard_degrid.py:488-608 the measurement-set level grid / PSF /
                               predict steps with their side effects.
The iteration controller is passed in by the caller (it is host logic,
pinned against the reference's own controller separately).
"""
import numpy as np
from scipy.ndimage import label

from . import oracle as O

LIN_C2S = np.array([[1, 0, 0, 1], [1, 0, 0, -1], [0, 1, 1, 0], [0, -1j, 1j, 0]], dtype=complex)
CIR_C2S = np.array([[1, 0, 0, 1], [0, 1, 1, 0], [0, -1j, 1j, 0], [1, 0, 0, -1]], dtype=complex)
LIN_S2C = np.array([[0.5, 0.5, 0, 0], [0, 0, 0.5, 0.5j], [0, 0, 0.5, -0.5j], [0.5, -0.5, 0, 0]],
                   dtype=complex)
CIR_S2C = np.array([[0.5, 0, 0, 0.5], [0, 0.5, 0.5j, 0], [0, 0.5, -0.5j, 0], [0.5, 0, 0, -0.5]],
                   dtype=complex)
SIDX = {"I": 0, "Q": 1, "U": 2, "V": 3}


def image_corr_to_stokes(data, corr_type, pol_axis, stokes_out):
    """corr_to_stokes.py:141-305 for numpy input."""
    ax = pol_axis % data.ndim
    moved = np.moveaxis(data, ax, -1)
    n_corr = moved.shape[-1]
    if n_corr == 2:
        full4 = np.zeros(moved.shape[:-1] + (4,), dtype=moved.dtype)
        full4[..., 0] = moved[..., 0]
        full4[..., 3] = moved[..., 1]
        moved = full4
    m = LIN_C2S if corr_type == "linear" else CIR_C2S
    full = moved @ m.T
    if set(stokes_out) == {"I", "Q", "U", "V"}:
        conv = full
    else:
        conv = np.take(full, [SIDX[s] for s in stokes_out], axis=-1)
    out = np.moveaxis(conv, -1, ax)
    return out.real if np.isrealobj(data) else out


def image_stokes_to_corr(data, corr_type, pol_axis, stokes_in):
    """corr_to_stokes.py:307-487 (corr_out from the Stokes count)."""
    ax = pol_axis % data.ndim
    moved = np.moveaxis(data, ax, -1)
    n = moved.shape[-1]
    if n != 4:
        idx = {s: i for i, s in enumerate(stokes_in)}
        partner = "Q" if corr_type == "linear" else "V"
        conv = np.zeros(moved.shape[:-1] + (2,), dtype=moved.dtype)
        i_ = moved[..., idx["I"]]
        if partner in idx:
            p_ = moved[..., idx[partner]]
            conv[..., 0] = (i_ + p_) / 2
            conv[..., 1] = (i_ - p_) / 2
        else:
            conv[..., 0] = i_ / 2
            conv[..., 1] = i_ / 2
    else:
        conv = moved @ (LIN_S2C if corr_type == "linear" else CIR_S2C).T
    return np.moveaxis(conv, -1, ax)


def psf_max_sidelobe(psf, window=(41, 41), threshold=0.35):
    """max_sidelobe of extract_main_lobe (psf_gaussian_fit.py:46-126) for one
    (ny, nx) plane."""
    img = np.asarray(psf, dtype=np.float64)[None, None, None]
    peak = np.max(img)
    if peak == 0:
        return 0.0
    _, _, _, py, px = np.unravel_index(np.argmax(img), img.shape)
    win = np.zeros_like(img)
    r0, r1 = max(0, px - window[0] // 2), min(img.shape[3], px + window[0] // 2)
    c0, c1 = max(0, py - window[1] // 2), min(img.shape[4], py + window[1] // 2)
    win[:, :, :, r0:r1, c0:c1] = img[:, :, :, r0:r1, c0:c1]
    labels, _ = label(win > peak * threshold)
    main = labels[np.unravel_index(np.argmax(win), win.shape)]
    return float(np.max(img * (labels != main)))


def _peak(plane):
    return plane.flat[np.abs(plane).argmax()]


def deconvolve_planes(dirty, psf, gain, niter, threshold, start_model=None):
    """deconvolution.py:123-329 on arrays: dirty (T, C, P, ny, nx), psf
    (T, C, Pp, ny, nx).  Returns (records, model, residual); records are the
    per-plane statistics in (time, chan, pol) order, each with its key."""
    nt, nc, npol = dirty.shape[:3]
    bc = psf.shape[2] == 1 and npol > 1
    model = np.zeros_like(dirty)
    resid = np.array(dirty, copy=True)
    recs = []
    for tt in range(nt):
        for nn in range(nc):
            sl = psf_max_sidelobe(psf[tt, nn, 0])
            for pp in range(npol):
                d = dirty[tt, nn, pp]
                # the empty float32 mask of hogbom_clean selects the FP32 CLEAN
                r = O.hogbom_clean(d.astype(np.float32), psf[tt, nn, 0 if bc else pp].astype(
                    np.float32), max_iter=int(niter), gain=float(np.float32(gain)),
                    threshold=float(np.float32(threshold)))
                model[tt, nn, pp] = r["model_image"]
                resid[tt, nn, pp] = r["residual_image"]
                recs.append({
                    "key": (tt, pp, nn),
                    "iter_done": int(r["iterations_performed"]),
                    "max_psf_sidelobe": sl,
                    "start_peakres": float(_peak(d)),
                    "peakres": float(_peak(resid[tt, nn, pp])),
                    "model_flux": float(np.sum(r["model_image"])),
                    "start_model_flux": 0.0 if start_model is None else
                    float(np.sum(start_model[tt, nn, pp])),
                    "masksum": int(d.shape[0] * d.shape[1]),
                })
    return recs, model, resid


def run_imaging_loop(vis, uvw, weight, flag, freq, params, controller, merge, ReturnDict,
                     initial_model=None):
    """imager.py:108-351 on arrays (vis (nt, nb, nchan, npol) complex128).
    weight / flag / uvw are modified in place as the reference modifies the
    measurement set.  Returns dict(model, residual, cycles, vis_model,
    residual_vis, controller, combined)."""
    image_size = params["image_size"]
    cell = np.asarray(params["cell_size"], dtype=float)
    support, os_ = params.get("support", 7), params.get("oversampling", 100)
    gain = params.get("gain", 0.1)
    corr_type = params.get("corr_type", "linear")
    chan_mode = params.get("chan_mode", "cube")
    n_corr = vis.shape[3]
    stokes = params.get("stokes") or (
        (["I", "Q"] if corr_type == "linear" else ["I", "V"]) if n_corr == 2
        else ["I", "Q", "U", "V"])
    ny, nx = image_size
    cgk = O.create_prolate_spheroidal_kernel_1D(os_, support)

    def grid_image(data, pixelincr, dopsf, n_uv):
        weight[flag] = 0.0
        weight[np.isnan(uvw[:, :, 0]) | np.isnan(uvw[:, :, 1])] = 0.0
        g, sw = O.standard_grid(data, uvw, weight, freq, cgk, n_uv, pixelincr, os_, support,
                                do_psf=dopsf, chan_mode=chan_mode)
        return O.grid_to_image(g, sw)

    psf_corr = grid_image(None, np.array([-cell[0], cell[1]]), True, (image_size[1],
                                                                       image_size[0]))
    psf_i = image_corr_to_stokes(psf_corr[None], corr_type, 2, ["I"])
    model = np.zeros((len(freq), len(stokes), ny, nx)) if initial_model is None else \
        np.array(initial_model, dtype=float)
    combined = ReturnDict()
    column = vis
    out = {"cycles": []}
    vis_model = None
    major = 0
    residual = None
    while controller.stopcode.major == 0:
        major += 1
        dirty = image_corr_to_stokes(grid_image(column, cell, False, (ny, nx)), corr_type, 1,
                                     stokes)
        if major == 1:
            t = ReturnDict()
            pk = float(np.max(np.abs(dirty)))
            t.add({"peakres": pk, "peakres_nomask": pk, "masksum": ny * nx, "iter_done": 0,
                   "max_psf_sidelobe": 0.2, "loop_gain": gain}, time=0, pol=0, chan=0)
            cn, ct = controller.calculate_cycle_controls(t)
        else:
            cn, ct = controller.calculate_cycle_controls(combined)
        start = model[None] if np.any(model != 0) else None
        recs, m5, r5 = deconvolve_planes(dirty[None], psf_i, gain, cn, ct, start)
        model, residual = m5[0], r5[0]
        rd = ReturnDict()
        for rec in recs:
            tt, pp, nn = rec["key"]
            rd.add({k: v for k, v in rec.items() if k != "key"} | {
                "loop_gain": gain, "niter": cn, "threshold": ct,
                "peakres_nomask": rec["peakres"],
                "start_peakres_nomask": rec["start_peakres"]}, time=tt, pol=pp, chan=nn)
        out["cycles"].append({"niter": cn, "threshold": ct, "records": recs})
        controller.update_counts(rd)
        combined = merge([combined, rd])
        code, _ = controller.check_convergence(rd)
        if code.major != 0:
            break
        mcorr = image_stokes_to_corr(model, corr_type, 1, stokes)
        grid = O.fft_lm_to_uv(mcorr, axes=[2, 3])
        nan_rows = np.isnan(uvw).any(axis=-1)
        flag[nan_rows] = True
        uvw[nan_rows] = 1e9
        g_nchan, g_npol = grid.shape[:2]
        gx, gy = grid.shape[-2:]
        vis_model = np.zeros(vis.shape, dtype=np.complex128)
        O.dgrid_numba(uvw, np.zeros(uvw.shape[:2]), vis_model, flag,
                      np.array([-cell[0] * gx, -cell[1] * gy, 0.0]),
                      np.array([gx / 2, gy / 2, 0.0]), grid, freq, 299792458.0, support, os_,
                      cgk, (np.arange(vis.shape[2]) / vis.shape[2] * g_nchan).astype(int),
                      np.round(np.arange(vis.shape[3]) % g_npol).astype(int))
        column = vis - vis_model
    out.update(model=model, residual=residual, vis_model=vis_model,
               residual_vis=None if vis_model is None else vis - vis_model,
               controller=controller, combined=combined)
    return out


# ----------------------------------------------------------------------------
# Normalisation helpers (standard_image_grid_preparation.py:312-492)
# ----------------------------------------------------------------------------
def correct_fft_to_uv_planes(x, u_size, v_size):
    """standard_image_grid_preparation.py:405-409: x /= u * v in place, in
    numpy's own arithmetic for the array's dtype."""
    x /= u_size * v_size
    return x


def correct_ifft_to_lm_planes(x, nx, ny, corr=None, norm=None):
    """standard_image_grid_preparation.py:458-492 on x (time, frequency,
    polarization, l, m), in place: x *= nx * ny, or with the spheroid
    correction each plane x[t, f, p] *= (nx * ny) / (corr * norm[t, f, p])
    (corr the (l, m) grid-correction term)."""
    if corr is None:
        x *= nx * ny
        return x
    for t in range(x.shape[0]):
        for f in range(x.shape[1]):
            for p in range(x.shape[2]):
                x[t, f, p] *= (nx * ny) / (corr * norm[t, f, p])
    return x


def mult_div_planes(x, pb, multiply=True):
    """_mult_div of apply_pb (standard_image_grid_preparation.py:278-309) on
    numpy arrays, in place: x *= pb or x /= pb with NaN where pb == 0, for
    equal shapes at once, else per (time, frequency, polarization) plane with
    pb's index 0 along each axis whose extent differs from x's."""
    if x.shape == pb.shape:
        if multiply:
            x *= pb
        else:
            x /= pb
            x[pb == 0.0] = np.nan
        return x
    te, ce, pe = (x.shape[k] == pb.shape[k] for k in range(3))
    for t in range(x.shape[0]):
        for c in range(x.shape[1]):
            for p in range(x.shape[2]):
                w = pb[t if te else 0, c if ce else 0, p if pe else 0]
                if multiply:
                    x[t, c, p] *= w
                else:
                    x[t, c, p] /= w
                    x[t, c, p][w == 0] = np.nan
    return x


def grid_ms4_into_image(nodes, grid, sumwt, cell, support=7, sampling=100, do_psf=False,
                        chan_mode="continuum"):
    """grid2xradio_spheroid_ms4 (standard_image_grid_preparation.py:495-580)
    on arrays: every node (vis, uvw, weight, flag, freq) gridded with the
    oracle's standard_grid_jit into each time plane of grid (time, frequency,
    polarization, u, v) complex128 and sumwt (time, frequency, polarization),
    in place; flagged weights set to 0 in the nodes' weight arrays."""
    cgk = O.create_prolate_spheroidal_kernel_1D(sampling, support)
    nu, nv = grid.shape[-2:]
    for it in range(grid.shape[0]):
        for vis, uvw, weight, flag, freq in nodes:
            weight[flag] = 0.0
            nchan, npol = weight.shape[2], weight.shape[3]
            chan_map = (np.arange(nchan) if chan_mode == "cube" else np.zeros(nchan)).astype(int)
            O.standard_grid_jit(grid[it], sumwt[it], do_psf, False, vis, uvw, freq, chan_map,
                                np.arange(npol), weight, cgk, np.array([nu, nv]),
                                np.asarray(cell), support, sampling)
    return grid, sumwt
