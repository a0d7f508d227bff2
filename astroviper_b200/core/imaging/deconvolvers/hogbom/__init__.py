"""Hogbom CLEAN on B200: drop-in for the reference's ``_hogbom_ext`` module
(src/astroviper/core/imaging/deconvolvers/hogbom/python/bindings.cpp).

Same functions, arguments, defaults, errors and result dictionary.  The
minor cycle runs as one persistent cooperative kernel (av_hogbom_run) whose
arithmetic is bit-identical to hclean.cpp; with callbacks it runs in segments
that end exactly where the reference calls them.

dtype selection follows the reference's pybind11 overloads (FP32 registered
first, then FP64, with forcecast): the FP64 path is taken only when every
array argument is float64 (an explicit empty float32 mask therefore selects
FP32, as in the reference); anything else is converted to float32.
"""
import numpy as np
import torch

from ..... import _kernels as K

__all__ = ["maximg", "clean", "clean_nc", "get_dtype_name", "is_float32", "is_float64"]


_TORCH_OF = {np.float32: torch.float32, np.float64: torch.float64}


def _is_dtype(a, dt):
    if isinstance(a, torch.Tensor):
        return a.dtype == _TORCH_OF[dt]
    return isinstance(a, np.ndarray) and a.dtype == dt


def _size(a):
    return a.numel() if isinstance(a, torch.Tensor) else np.asarray(a).size


def _t(a):
    """Device tensor of a converted array (numpy arrays are staged)."""
    return a if isinstance(a, torch.Tensor) else torch.from_numpy(a)


def _out(t, on_device):
    return t if on_device else t.cpu().numpy()


def _pick_dtype(*arrays):
    given = [a for a in arrays if a is not None]
    if all(_is_dtype(a, np.float32) for a in given):
        return np.float32
    if all(_is_dtype(a, np.float64) for a in given):
        return np.float64
    return np.float32


def _as(a, dt):
    if isinstance(a, torch.Tensor):
        return a.to(device=K.device(), dtype=_TORCH_OF[dt]).contiguous()
    return np.ascontiguousarray(np.asarray(a), dtype=dt)


def maximg(image, mask=None):
    """(fmin, fmax) over pixels with mask > 0.5 (hclean.cpp:51-81,
    bindings.cpp:16-58)."""
    dt = _pick_dtype(image, mask)
    img = _as(image, dt)
    if img.ndim != 2:
        raise RuntimeError("Image must be 2D array")
    m = None
    if mask is not None and _size(mask) > 0:
        m = _as(mask, dt)
        if m.ndim != 2:
            raise RuntimeError("Mask must be 2D array")
        if tuple(m.shape) != tuple(img.shape):
            raise RuntimeError("Mask dimensions must match image spatial dimensions")
    out = K.maximg(_t(img), None if m is None else _t(m))
    o = out.cpu().numpy()
    return (float(o[0]), float(o[1]))


def _box(clean_box, nx, ny):
    xbeg, xend, ybeg, yend = 0, nx, 0, ny
    if len(clean_box) == 4:
        xbeg, xend, ybeg, yend = (int(v) for v in clean_box)
        if xbeg == -1:
            xbeg = 0
        if xend == -1:
            xend = nx
        if ybeg == -1:
            ybeg = 0
        if yend == -1:
            yend = ny
        xbeg = max(0, min(xbeg, nx - 1))
        xend = max(xbeg + 1, min(xend, nx))
        ybeg = max(0, min(ybeg, ny - 1))
        yend = max(ybeg + 1, min(yend, ny))
    return xbeg, xend, ybeg, yend


def _final_stats(run):
    """(min, max) of the residual (maximg) and the ordered sum of the model's
    |x| as one host array (FP64 holds the FP32 results exactly)."""
    mm = K.maximg(run.resid, run.mask)
    total = K.abs_sum_ordered(run.model)
    return torch.cat([mm.reshape(-1).to(torch.float64),
                      total.reshape(-1)[:1].to(torch.float64)]).cpu().numpy()


def clean(dirty_image, psf, mask=None, clean_box=(-1, -1, -1, -1), max_iter=100, start_iter=0,
          gain=0.1, threshold=0.0, speedup=0.0, progress_callback=None, stop_callback=None, *,
          large_psf=False):
    """hclean_impl (bindings.cpp:63-208) + hclean::clean (hclean.cpp:106-210).

    Returns {model_image, residual_image, iterations_performed, final_peak,
    total_flux_cleaned, converged}.  With large_psf=True a PSF larger than
    the image is accepted (centre at its (ny/2, nx/2)); the reference requires
    equal shapes.  torch tensors are accepted too (same dtype rule, torch
    float32 / float64 in place of numpy's); the model and residual then stay
    on the device."""
    on_device = isinstance(dirty_image, torch.Tensor)
    m_given = mask if (mask is not None and _size(mask) > 0) else None
    dt = _pick_dtype(dirty_image, psf, mask)
    d = _as(dirty_image, dt)
    p = _as(psf, dt)
    if d.ndim != 2:
        raise RuntimeError("Dirty image must be 2D [ny, nx]")
    if p.ndim != 2:
        raise RuntimeError("PSF must be 2D [ny, nx]")
    ny, nx = d.shape
    if large_psf:
        if p.shape[0] < ny or p.shape[1] < nx:
            raise RuntimeError("PSF must be at least as large as the image")
    elif tuple(p.shape) != tuple(d.shape):
        raise RuntimeError("PSF dimensions must match image spatial dimensions")
    m = None
    if m_given is not None:
        m = _as(m_given, dt)
        if m.ndim != 2 or tuple(m.shape) != tuple(d.shape):
            raise RuntimeError("Mask must be 2D with same spatial dimensions as image")
    box = _box(tuple(clean_box), nx, ny)
    tdt = np.dtype(dt).type
    niter, siter = int(max_iter), int(start_iter)
    gain_t, thres_t, speed_t = tdt(gain), tdt(threshold), tdt(speedup)
    run = K.HogbomRun(_t(d), _t(p), mask=None if m is None else _t(m), box=box, niter=niter,
                      siter=siter, gain=float(gain_t), threshold=float(thres_t),
                      speedup=float(speed_t))
    callbacks = progress_callback is not None or stop_callback is not None
    if not callbacks:
        run.run(siter, niter)
        # the final statistics are queued before the state is read, so the
        # host waits once
        stats = _final_stats(run)
        st = run.read_state()
    else:
        cycle = max(1, int((niter - siter) / 10)) if niter - siter >= 0 else 1
        run.run(siter, siter)  # peak of the first iteration only
        st = run.read_state()
        last = None
        while True:
            it = st["iter"]
            if st["stopped"] or it >= niter:
                break
            cth = thres_t
            if speed_t > 0:
                cth = tdt(thres_t * np.power(tdt(2), tdt(it - siter) / speed_t))
            if tdt(st["absval"]) < cth:
                break
            if it == siter or (it % cycle) == 1:
                if progress_callback is not None:
                    progress_callback(it, st["px"], st["py"], float(tdt(st["peak"])))
                if stop_callback is not None and bool(stop_callback()):
                    break
            nxt = it + 1
            while nxt < niter and (nxt % cycle) != 1:
                nxt += 1
            end = min(nxt, niter)
            if end == niter and it < niter - 1:
                # stop one short so the peak of the last iteration is kept
                run.run(it, niter - 1)
                st = run.read_state()
                continue
            if it == niter - 1:
                last = st
            run.run(it, end)
            st = run.read_state()
        if st["iter"] > siter and progress_callback is not None:
            # a loop that ran out of iterations reports the peak its last
            # iteration subtracted (hclean.cpp:124,202-203)
            rep = last if (st["iter"] >= niter and last is not None) else st
            progress_callback(st["iter"], rep["px"], rep["py"], float(tdt(rep["peak"])))
        stats = _final_stats(run)
    final_iter = min(st["iter"], niter) if st["iter"] > niter else st["iter"]
    mm = stats[:2]
    final_peak = max(abs(mm[0]), abs(mm[1]))
    total = stats[2]
    return {
        "model_image": _out(run.model, on_device),
        "residual_image": _out(run.resid, on_device),
        "iterations_performed": int(final_iter),
        "final_peak": float(final_peak),
        "total_flux_cleaned": float(total),
        "converged": bool(final_peak <= thres_t),
    }


def clean_nc(dirty_image, psf, gain=0.1, threshold=0.0, max_iter=100,
             clean_box=(-1, -1, -1, -1)):
    """hclean_simple_impl (bindings.cpp:213-228): no mask, no callbacks."""
    return clean(dirty_image, psf, None, clean_box, max_iter, 0, gain, threshold, 0.0, None,
                 None)


def get_dtype_name(arr):
    """String name of an array's dtype (bindings.cpp:290-292)."""
    return str(np.asarray(arr).dtype)


def is_float32(arr):
    return np.asarray(arr).dtype == np.float32


def is_float64(arr):
    return np.asarray(arr).dtype == np.float64
