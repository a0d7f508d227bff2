"""Device-tensor front end of libav200: one function per C-ABI entry point.

All tensors are CUDA tensors (C-contiguous); results stay on the device.  The
numpy/xarray drop-in modules under ``astroviper_b200.core`` stage host arrays
through these functions.  Scratch space comes from torch's caching allocator
and is handed to the library as (pointer, bytes).
"""
import math

import numpy as np
import torch

from . import _lib
from ._lib import AV_C64, AV_C128, AV_F32, AV_F64, check, lib

C_LIGHT = 299792458.0

_DT = {torch.float32: AV_F32, torch.float64: AV_F64, torch.complex64: AV_C64,
       torch.complex128: AV_C128}


def require_gpu():
    if not torch.cuda.is_available():
        raise RuntimeError("astroviper_b200 needs a CUDA device (B200, sm_100a); none is visible")
    lib()


def device():
    require_gpu()
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr():
    return torch.cuda.current_stream().cuda_stream


def dcode(t):
    try:
        return _DT[t.dtype]
    except KeyError:
        raise TypeError(f"unsupported dtype {t.dtype}") from None


def p(t):
    """Device pointer of a tensor (None passes NULL)."""
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return t.data_ptr()


def workspace(nbytes):
    """Scratch buffer (256-byte aligned) from torch's caching allocator."""
    n = int(max(nbytes, 256))
    buf = torch.empty(n + 256, dtype=torch.uint8, device=device())
    off = (-buf.data_ptr()) % 256
    return buf, buf.data_ptr() + off, n


def on_device(x, dtype=None):
    """Contiguous CUDA tensor from a tensor or array-like."""
    dev = device()
    if isinstance(x, torch.Tensor):
        t = x.to(device=dev, dtype=dtype or x.dtype, non_blocking=True)
    else:
        t = torch.as_tensor(x, dtype=dtype, device=dev)
    return t.contiguous()


# --------------------------------------------------------------------- PSWF --
def pswf(u):
    u = on_device(u, torch.float64)
    g = torch.empty_like(u)
    k = torch.empty_like(u)
    check(lib().av_pswf(p(u), u.numel(), p(g), p(k), stream_ptr()), "av_pswf")
    return g, k


def pswf_table(oversampling, support):
    out = torch.empty(oversampling * (support // 2 + 1), dtype=torch.float64, device=device())
    check(lib().av_pswf_table(p(out), int(oversampling), int(support), stream_ptr()),
          "av_pswf_table")
    return out


def corr_term(nx, ny):
    out = torch.empty((int(nx), int(ny)), dtype=torch.float64, device=device())
    check(lib().av_corr_term(p(out), int(nx), int(ny), stream_ptr()), "av_corr_term")
    return out


def pswf_kernel4d(oversampling, support):
    n_os = oversampling + 1 if oversampling % 2 == 0 else oversampling
    out = torch.empty((n_os, n_os, support, support), dtype=torch.float64, device=device())
    check(lib().av_pswf_kernel4d(p(out), int(oversampling), int(support), stream_ptr()),
          "av_pswf_kernel4d")
    return out


# ----------------------------------------------------------------- gridding --
def grid_tiled_ok(precision, do_imaging_weight, support, oversampling, npol, n_img_pol):
    """Whether grid() runs the tiled kernel for these options."""
    return not (precision == "fp64" or do_imaging_weight or support > 9 or support < 3
                or oversampling > 254 or npol > 4 or n_img_pol > 4)


def degrid_tiled_ok(precision, support, sampling, g_npol, c):
    """Whether degrid() runs the tiled kernel for these options."""
    return (precision != "fp64" and 3 <= support <= 9 and sampling <= 254 and g_npol <= 4
            and float(c) == C_LIGHT)


def grid(vis, weight, uvw, freq, chan_map, pol_map, cgk, n_uv, delta_lm, support,
         oversampling, n_img_chan, n_img_pol, grid_out=None, sum_weight=None, do_psf=False,
         do_imaging_weight=False, precision="fp32"):
    """Accumulate samples into grid_out / sum_weight (allocated when None).

    precision "fp32": the tiled kernel (reads complex64 visibilities and
    float32 weights, accumulates in FP64; complex128 grid unless a complex64
    grid is passed); "fp64": the plain FP64 kernel (FP64 inputs, every option
    of the reference, complex128 grid)."""
    dev = device()
    nu, nv = int(n_uv[0]), int(n_uv[1])
    nt, nb = int(uvw.shape[0]), int(uvw.shape[1])
    nchan, npol = int(weight.shape[2]), int(weight.shape[3])
    uvw = on_device(uvw, torch.float64)
    freq = on_device(freq, torch.float64)
    cm = on_device(chan_map, torch.int32)
    pm = on_device(pol_map, torch.int32)
    cgk = on_device(cgk, torch.float64)
    fp64 = not grid_tiled_ok(precision, do_imaging_weight, support, oversampling, npol,
                             n_img_pol)
    if grid_out is None:
        grid_out = torch.zeros((n_img_chan, n_img_pol, nu, nv), dtype=torch.complex128,
                               device=dev)
    if sum_weight is None:
        sum_weight = torch.zeros((n_img_chan, n_img_pol), dtype=torch.float64, device=dev)
    assert grid_out.is_contiguous() and sum_weight.is_contiguous()
    if fp64:
        w = on_device(weight)
        if w.dtype not in (torch.float32, torch.float64):
            w = w.to(torch.float64)
        v = None if do_psf else on_device(vis)
        if v is not None and v.dtype not in (torch.complex64, torch.complex128):
            v = v.to(torch.complex128)
        rc = lib().av_grid_plain(
            p(grid_out), dcode(grid_out), p(sum_weight), int(bool(do_psf)),
            int(bool(do_imaging_weight)), p(v), dcode(v) if v is not None else AV_C128, p(w),
            dcode(w), p(uvw), p(freq), p(cm), p(pm), p(cgk), nu, nv, float(delta_lm[0]),
            float(delta_lm[1]), int(support), int(oversampling), nt, nb, nchan, npol,
            int(n_img_chan), int(n_img_pol), stream_ptr())
        check(rc, "av_grid_plain")
        return grid_out, sum_weight
    w = on_device(weight, torch.float32)
    v = None if do_psf else on_device(vis, torch.complex64)
    ws_bytes = lib().av_grid_tiled_workspace_size(nt, nb, nchan, nu, nv, int(n_img_chan),
                                                  int(support))
    _buf, wptr, wbytes = workspace(ws_bytes)
    rc = lib().av_grid_tiled(
        p(grid_out), dcode(grid_out), p(sum_weight), int(bool(do_psf)), p(v), AV_C64, p(w),
        AV_F32, p(uvw), p(freq), p(cm), p(pm), p(cgk), nu, nv, float(delta_lm[0]),
        float(delta_lm[1]), int(support), int(oversampling), nt, nb, nchan, npol,
        int(n_img_chan), int(n_img_pol), wptr, wbytes, stream_ptr())
    check(rc, "av_grid_tiled")
    return grid_out, sum_weight


def degrid(grid_t, uvw, freq, scale, offset, chanmap, polmap, cgk, support, sampling,
           values=None, flag=None, dphase=None, c=C_LIGHT, nvchan=None, nvpol=None,
           precision="fp32", accumulate=True):
    """values (nt, nb, nvchan, nvpol) += degridded model (accumulate) or =
    model with zeros for skipped samples (not accumulate, tiled kernel only);
    values are allocated (complex64 / complex128) when None."""
    dev = device()
    g = on_device(grid_t)
    if g.dtype not in (torch.complex64, torch.complex128):
        g = g.to(torch.complex128)
    nt, nb = int(uvw.shape[0]), int(uvw.shape[1])
    if values is not None:
        nvchan, nvpol = int(values.shape[2]), int(values.shape[3])
    uvw = on_device(uvw, torch.float64)
    freq = on_device(freq, torch.float64)
    cm = on_device(chanmap, torch.int32)
    pm = on_device(polmap, torch.int32)
    cgk = on_device(cgk, torch.float64)
    fl = None if flag is None else on_device(flag).to(torch.uint8).contiguous()
    dph = None if dphase is None else on_device(dphase, torch.float64)
    g_nchan, g_npol, g_n2, g_n3 = (int(s) for s in g.shape)
    tiled_ok = degrid_tiled_ok(precision, support, sampling, g_npol, c)
    if values is None:
        vdt = torch.complex64 if tiled_ok else torch.complex128
        if tiled_ok and not accumulate:
            values = torch.empty((nt, nb, nvchan, nvpol), dtype=vdt, device=dev)
        else:
            values = torch.zeros((nt, nb, nvchan, nvpol), dtype=vdt, device=dev)
            accumulate = True
    assert values.is_contiguous()
    if not tiled_ok:
        if not accumulate:
            values.zero_()
        args_common = (p(uvw), p(dph), p(values), dcode(values), p(fl), float(scale[0]),
                       float(scale[1]), float(offset[0]), float(offset[1]))
        rc = lib().av_degrid_plain(*args_common, p(g), dcode(g), g_nchan, g_npol, g_n2, g_n3,
                                   p(freq), float(c), int(support), int(sampling), p(cgk), p(cm),
                                   p(pm), nt, nb, nvchan, nvpol, stream_ptr())
        check(rc, "av_degrid_plain")
        return values
    ws_bytes = lib().av_degrid_tiled_workspace_size(nt, nb, nvchan, g_n2, g_n3, g_nchan,
                                                    int(support))
    _buf, wptr, wbytes = workspace(ws_bytes)
    rc = lib().av_degrid_tiled(p(uvw), p(dph), p(values), dcode(values), int(bool(accumulate)),
                               p(fl), float(scale[0]), float(scale[1]), float(offset[0]),
                               float(offset[1]), p(g), dcode(g), g_nchan, g_npol, g_n2, g_n3,
                               p(freq), float(c), int(support), int(sampling), p(cgk), p(cm),
                               p(pm), nt, nb, nvchan, nvpol, wptr, wbytes, stream_ptr())
    check(rc, "av_degrid_tiled")
    return values


# ------------------------------------------------- streamed host inputs ----
# Large host (numpy) inputs go to the device in time chunks on a copy stream
# while the previous chunk is planned and gridded / degridded on the current
# stream (and, for the degridder, the chunk before that is copied back on a
# third stream): the kernels and the copies in both directions overlap.  The
# overlap needs page-locked host arrays; pageable ones are copied
# synchronously, with the same results.
STREAM_CHUNK_BYTES = 128 << 20
DEGRID_STREAM_SLOTS = 3
_streams = {}


def _side_stream(name):
    key = (name, torch.cuda.current_device())
    if key not in _streams:
        _streams[key] = torch.cuda.Stream()
    return _streams[key]


def time_chunks(nt, bytes_per_t, chunk_bytes=None):
    """[(t0, t1), ...] covering range(nt) in about chunk_bytes pieces
    (STREAM_CHUNK_BYTES when None)."""
    chunk_bytes = STREAM_CHUNK_BYTES if chunk_bytes is None else chunk_bytes
    n = int(max(1, min(nt, -(-int(nt * bytes_per_t) // int(chunk_bytes)))))
    edges = [nt * i // n for i in range(n + 1)]
    return list(zip(edges[:-1], edges[1:]))


def _h2d(dst, host_slice):
    dst.copy_(torch.from_numpy(np.ascontiguousarray(host_slice)), non_blocking=True)


def grid_streamed(vis, weight, uvw, freq, chan_map, pol_map, cgk, n_uv, delta_lm, support,
                  oversampling, n_img_chan, n_img_pol, grid_out, sum_weight, do_psf=False,
                  chunk_bytes=None):
    """grid() of host arrays vis / weight / uvw (tiled kernel), copied to the
    device in time chunks that overlap the gridding of the previous chunk.
    Accumulates into the device arrays grid_out / sum_weight."""
    nt = int(uvw.shape[0])
    per_t = weight[0].nbytes + (0 if do_psf else vis[0].nbytes) + uvw[0].nbytes
    chunks = time_chunks(nt, per_t, chunk_bytes)
    tmax = max(t1 - t0 for t0, t1 in chunks)
    dev = device()
    freq = on_device(freq, torch.float64)
    chan_map = on_device(chan_map, torch.int32)
    pol_map = on_device(pol_map, torch.int32)
    cgk = on_device(cgk, torch.float64)
    cur = torch.cuda.current_stream()
    cp = _side_stream("h2d")
    mk = lambda a: torch.empty((tmax,) + tuple(a.shape[1:]),
                               dtype=torch.from_numpy(a[:1]).dtype, device=dev)
    slots = [dict(w=mk(weight), u=mk(uvw), v=None if do_psf else mk(vis)) for _ in range(2)]
    free = [None, None]
    cp.wait_stream(cur)
    for i, (t0, t1) in enumerate(chunks):
        sl = slots[i % 2]
        n = t1 - t0
        with torch.cuda.stream(cp):
            if free[i % 2] is not None:
                cp.wait_event(free[i % 2])
            _h2d(sl["w"][:n], weight[t0:t1])
            _h2d(sl["u"][:n], uvw[t0:t1])
            if not do_psf:
                _h2d(sl["v"][:n], vis[t0:t1])
            ready = torch.cuda.Event()
            ready.record(cp)
        cur.wait_event(ready)
        grid(None if do_psf else sl["v"][:n], sl["w"][:n], sl["u"][:n], freq, chan_map, pol_map,
             cgk, n_uv, delta_lm, support, oversampling, n_img_chan, n_img_pol,
             grid_out=grid_out, sum_weight=sum_weight, do_psf=do_psf, precision="fp32")
        ev = torch.cuda.Event()
        ev.record(cur)
        free[i % 2] = ev
    return grid_out, sum_weight


def degrid_streamed(grid_t, uvw, freq, scale, offset, chanmap, polmap, cgk, support, sampling,
                    values, flag=None, dphase=None, chunk_bytes=None):
    """values (host array, updated in place) += degridded model of the device
    grid grid_t (tiled kernel), in time chunks: chunk i+1 is copied in while
    chunk i is degridded and chunk i-1 copied back.  Three device slots, so
    that copying a chunk in never waits for the copy back of the one before
    it: the two directions of the host link then run at once.  Returns when
    values holds the result."""
    nt = int(uvw.shape[0])
    per_t = values[0].nbytes * 2 + uvw[0].nbytes + (0 if flag is None else flag[0].nbytes)
    chunks = time_chunks(nt, per_t, chunk_bytes)
    tmax = max(t1 - t0 for t0, t1 in chunks)
    dev = device()
    grid_t = on_device(grid_t)
    freq = on_device(freq, torch.float64)
    chanmap = on_device(chanmap, torch.int32)
    polmap = on_device(polmap, torch.int32)
    cgk = on_device(cgk, torch.float64)
    cur = torch.cuda.current_stream()
    cin = _side_stream("h2d")
    cout = _side_stream("d2h")
    vt = torch.from_numpy(values[:1]).dtype
    n_slots = DEGRID_STREAM_SLOTS
    slots = []
    for _ in range(n_slots):
        slots.append(dict(
            v=torch.empty((tmax,) + tuple(values.shape[1:]), dtype=vt, device=dev),
            u=torch.empty((tmax,) + tuple(uvw.shape[1:]), dtype=torch.float64, device=dev),
            f=None if flag is None else torch.empty((tmax,) + tuple(flag.shape[1:]),
                                                    dtype=torch.uint8, device=dev),
            d=None if dphase is None else torch.empty((tmax,) + tuple(np.shape(dphase)[1:]),
                                                      dtype=torch.float64, device=dev)))
    vals_t = torch.from_numpy(values)
    free = [None] * n_slots
    cin.wait_stream(cur)
    for i, (t0, t1) in enumerate(chunks):
        sl = slots[i % n_slots]
        n = t1 - t0
        with torch.cuda.stream(cin):
            if free[i % n_slots] is not None:
                cin.wait_event(free[i % n_slots])
            _h2d(sl["v"][:n], values[t0:t1])
            _h2d(sl["u"][:n], np.asarray(uvw[t0:t1], dtype=np.float64))
            if flag is not None:
                f = np.asarray(flag[t0:t1])
                _h2d(sl["f"][:n], f.view(np.uint8) if f.dtype == np.bool_ else f.astype(np.uint8))
            if dphase is not None:
                _h2d(sl["d"][:n], np.asarray(dphase[t0:t1], dtype=np.float64))
            ready = torch.cuda.Event()
            ready.record(cin)
        cur.wait_event(ready)
        degrid(grid_t, sl["u"][:n], freq, scale, offset, chanmap, polmap, cgk, support,
               sampling, values=sl["v"][:n], flag=None if flag is None else sl["f"][:n],
               dphase=None if dphase is None else sl["d"][:n], accumulate=True)
        done = torch.cuda.Event()
        done.record(cur)
        with torch.cuda.stream(cout):
            cout.wait_event(done)
            vals_t[t0:t1].copy_(sl["v"][:n], non_blocking=True)
            back = torch.cuda.Event()
            back.record(cout)
        free[i % n_slots] = back
    cur.wait_stream(cout)
    cout.synchronize()
    return values


# ------------------------------------------------------------------- images --
def grid_to_image(grid_t, sum_weight=None, apply_corr=True, out_dtype=None):
    """Re(fftshift(ifft2(ifftshift(grid)))) / corrTerm * nx*ny / sum_weight per
    plane of a (..., nx, ny) complex grid."""
    g = on_device(grid_t)
    if g.dtype not in (torch.complex64, torch.complex128):
        g = g.to(torch.complex128)
    nx, ny = int(g.shape[-2]), int(g.shape[-1])
    npl = int(g.numel() // (nx * ny))
    if out_dtype is None:
        out_dtype = torch.float32 if g.dtype == torch.complex64 else torch.float64
    img = torch.empty(g.shape, dtype=out_dtype, device=g.device)
    sw = None
    if sum_weight is not None:
        sw = on_device(sum_weight, torch.float64).reshape(-1)
        assert sw.numel() == npl
    ws = lib().av_grid_to_image_workspace_size(npl, nx, ny)
    _buf, wptr, wbytes = workspace(ws)
    check(lib().av_grid_to_image(p(g), dcode(g), p(sw), p(img), dcode(img), npl, nx, ny,
                                 int(bool(apply_corr)), wptr, wbytes, stream_ptr()),
          "av_grid_to_image")
    return img


def fft_shifted(x, inverse):
    """fftshift(fft2 / ifft2(ifftshift(x))) over the last two axes (complex)."""
    t = on_device(x)
    if not t.is_complex():
        t = t.to(torch.complex128 if t.dtype == torch.float64 else torch.complex64)
    nx, ny = int(t.shape[-2]), int(t.shape[-1])
    npl = int(t.numel() // max(1, nx * ny))
    out = torch.empty_like(t)
    ws = lib().av_fft_workspace_size(npl, nx, ny, dcode(t))
    _buf, wptr, wbytes = workspace(ws)
    check(lib().av_fft_shifted(p(t), p(out), dcode(t), npl, nx, ny, int(bool(inverse)), wptr,
                               wbytes, stream_ptr()), "av_fft_shifted")
    return out


# ------------------------------------------------------------------ weights --
def weight_density(uvw, freq, weight, flag, n_uv, delta_lm, density=None, sum_weight=None):
    """Nearest-cell weight-density grid (nchan, 1, nu, nv) and sum_weight."""
    dev = device()
    nt, nb, nchan, npol = (int(s) for s in weight.shape)
    nu, nv = int(n_uv[0]), int(n_uv[1])
    w = on_device(weight)
    if w.dtype not in (torch.float32, torch.float64):
        w = w.to(torch.float64)
    fl = None if flag is None else on_device(flag).to(torch.uint8).contiguous()
    if density is None:
        density = torch.zeros((nchan, 1, nu, nv), dtype=torch.float64, device=dev)
    if sum_weight is None:
        sum_weight = torch.zeros((nchan, 1), dtype=torch.float64, device=dev)
    # device copies are held in locals until the launch: a temporary freed
    # right after taking its pointer could be handed to the next one
    uvw_d = on_device(uvw, torch.float64)
    freq_d = on_device(freq, torch.float64)
    check(lib().av_weight_density(p(density), p(sum_weight), p(uvw_d),
                                  p(freq_d), p(w), dcode(w), p(fl), nu,
                                  nv, float(delta_lm[0]), float(delta_lm[1]), nt, nb, nchan,
                                  npol, stream_ptr()), "av_weight_density")
    return density, sum_weight


def briggs_factors(density, sum_weight, robust):
    d = on_device(density, torch.float64)
    sw = on_device(sum_weight, torch.float64)
    npl = int(d.shape[0] * d.shape[1])
    nu, nv = int(d.shape[2]), int(d.shape[3])
    out = torch.empty((2,) + tuple(sw.shape), dtype=torch.float64, device=d.device)
    _buf, wptr, wbytes = workspace(lib().av_briggs_factors_workspace_size(npl))
    check(lib().av_briggs_factors(p(d), p(sw), p(out), npl, nu, nv, float(robust), wptr, wbytes,
                                  stream_ptr()), "av_briggs_factors")
    return out


def briggs_apply(density, factors, uvw, freq, weight, flag, n_uv, delta_lm,
                 out_dtype=torch.float64):
    nt, nb, nchan, npol = (int(s) for s in weight.shape)
    w = on_device(weight)
    if w.dtype not in (torch.float32, torch.float64):
        w = w.to(torch.float64)
    fl = None if flag is None else on_device(flag).to(torch.uint8).contiguous()
    out = torch.empty((nt, nb, nchan, npol), dtype=out_dtype, device=w.device)
    err = torch.zeros(1, dtype=torch.int32, device=w.device)
    dens_d = on_device(density, torch.float64)
    fac_d = on_device(factors, torch.float64)
    uvw_d = on_device(uvw, torch.float64)
    freq_d = on_device(freq, torch.float64)
    check(lib().av_briggs_apply(p(out), dcode(out), p(dens_d), p(fac_d), p(uvw_d), p(freq_d),
                                p(w), dcode(w), p(fl),
                                int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                                float(delta_lm[1]), nt, nb, nchan, npol, p(err), stream_ptr()),
          "av_briggs_apply")
    return out, err


def imaging_weight_degrid(imaging_weight, grid_imaging_weight, briggs_factors, uvw, freq,
                          chan_map, pol_map, natural_weight, n_uv, delta_lm):
    """av_imaging_weight_degrid into the float64 device tensor imaging_weight
    (nt, nb, nchan, npol), in place; returns it."""
    w = on_device(natural_weight)
    if w.dtype not in (torch.float32, torch.float64):
        w = w.to(torch.float64)
    G = on_device(grid_imaging_weight)
    if G.dtype not in (torch.float32, torch.float64):
        G = G.to(torch.float64)
    G = G.contiguous()
    nt, nb, nchan, npol = (int(s) for s in w.shape)
    g_chan, g_pol = int(G.shape[0]), int(G.shape[1])
    cm = np.asarray(chan_map).astype(np.int64).ravel()
    pm = np.asarray(pol_map).astype(np.int64).ravel()
    if cm.size != nchan or pm.size != npol:
        raise ValueError("chan_map / pol_map must have one entry per channel / polarisation")
    if cm.size and (cm.min() < 0 or cm.max() >= g_chan):
        raise ValueError("chan_map entries must index grid_imaging_weight's channels")
    if pm.size and (pm.min() < 0 or pm.max() >= g_pol):
        raise ValueError("pol_map entries must index grid_imaging_weight's polarisations")
    bf = on_device(briggs_factors, torch.float64).contiguous()
    if bf.numel() != 2 * g_chan * g_pol:
        raise ValueError("briggs_factors must have shape (2, n_chan, n_pol) of the grid")
    uvw_d = on_device(uvw, torch.float64)
    freq_d = on_device(freq, torch.float64)
    cm_d = torch.as_tensor(cm.astype(np.int32), device=w.device)
    pm_d = torch.as_tensor(pm.astype(np.int32), device=w.device)
    check(lib().av_imaging_weight_degrid(p(imaging_weight), p(G), dcode(G), g_chan, g_pol, p(bf),
                                         p(uvw_d), p(freq_d), p(cm_d), p(pm_d), p(w), dcode(w),
                                         int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                                         float(delta_lm[1]), nt, nb, nchan, npol, stream_ptr()),
          "av_imaging_weight_degrid")
    return imaging_weight


# ------------------------------------------------------------------- Hogbom --
def maximg(image, mask=None):
    im = on_device(image)
    m = None if mask is None else on_device(mask, im.dtype)
    out = torch.empty(2, dtype=im.dtype, device=im.device)
    ny, nx = int(im.shape[0]), int(im.shape[1])
    check(lib().av_maximg(p(im), p(m), dcode(im), nx, ny, p(out), stream_ptr()), "av_maximg")
    return out


def abs_sum_ordered(x):
    t = on_device(x)
    out = torch.empty(1, dtype=t.dtype, device=t.device)
    n = t.numel()
    _buf, wptr, wbytes = workspace(lib().av_abs_sum_workspace_size(n, dcode(t)))
    check(lib().av_abs_sum_ordered(p(t), dcode(t), n, p(out), wptr, wbytes, stream_ptr()),
          "av_abs_sum_ordered")
    return out


class HogbomRun:
    """Device state of one Hogbom CLEAN run (residual, model, PSF)."""

    def __init__(self, dirty, psf, mask=None, box=None, niter=100, siter=0, gain=0.1,
                 threshold=0.0, speedup=0.0):
        self.resid = on_device(dirty).clone()
        self.dtype = self.resid.dtype
        assert self.dtype in (torch.float32, torch.float64)
        self.psf = on_device(psf, self.dtype)
        self.mask = None if mask is None else on_device(mask, self.dtype)
        self.model = torch.zeros_like(self.resid)
        self.ny, self.nx = (int(s) for s in self.resid.shape)
        self.pny, self.pnx = (int(s) for s in self.psf.shape)
        self.box = box if box is not None else (0, self.nx, 0, self.ny)
        self.niter, self.siter = int(niter), int(siter)
        self.gain, self.threshold, self.speedup = float(gain), float(threshold), float(speedup)
        self.state = torch.zeros(int(lib().av_hogbom_state_size()) // 8, dtype=torch.float64,
                                 device=self.resid.device)
        self._ws = workspace(lib().av_hogbom_workspace_size(self.nx, self.ny, dcode(self.resid)))
        self.started = False

    def run(self, iter_begin, iter_end):
        xb, xe, yb, ye = self.box
        init = 0 if self.started else 1
        _buf, wptr, wbytes = self._ws
        check(lib().av_hogbom_run(p(self.model), p(self.resid), p(self.psf), p(self.mask),
                                  dcode(self.resid), self.nx, self.ny, self.pnx, self.pny, xb, xe,
                                  yb, ye, self.niter, self.siter, int(iter_begin), int(iter_end),
                                  self.gain, self.threshold, self.speedup, p(self.state), init,
                                  wptr, wbytes, stream_ptr()), "av_hogbom_run")
        self.started = True

    def read_state(self):
        import ctypes
        oi = (ctypes.c_int32 * 5)()
        od = (ctypes.c_double * 2)()
        check(lib().av_hogbom_state_read(p(self.state), oi, od, stream_ptr()),
              "av_hogbom_state_read")
        return dict(iter=oi[0], px=oi[1], py=oi[2], stopped=oi[3], err=oi[4], peak=od[0],
                    absval=od[1])


# ------------------------------------------------------------------ imager --
def pol_transform(x, matrix, pol_axis, out_dtype):
    """out[..., o, ...] = sum_i matrix[o, i] x[..., i, ...] along pol_axis
    (av_pol_transform); matrix (n_out, n_in) complex, out_dtype a torch
    dtype (real output keeps the real part)."""
    t = on_device(x)
    if t.dtype not in (torch.float32, torch.float64, torch.complex64, torch.complex128):
        t = t.to(torch.float64)
    m = np.asarray(matrix, dtype=np.complex128)
    n_out, n_in = m.shape
    ax = pol_axis % t.ndim
    if int(t.shape[ax]) != n_in:
        raise ValueError(f"polarisation axis has {int(t.shape[ax])} entries, matrix takes {n_in}")
    n_outer = int(np.prod(t.shape[:ax], dtype=np.int64))
    n_pix = int(np.prod(t.shape[ax + 1:], dtype=np.int64))
    shape = list(t.shape)
    shape[ax] = n_out
    out = torch.empty(shape, dtype=out_dtype, device=t.device)
    flat = np.ascontiguousarray(np.stack([m.real, m.imag], axis=-1).reshape(-1))
    check(lib().av_pol_transform(p(t), dcode(t), p(out), dcode(out),
                                 flat.ctypes.data, n_in, n_out, n_outer,
                                 n_pix, stream_ptr()), "av_pol_transform")
    return out


def argmax(x, mode):
    """(index, value) of np.argmax(np.abs(x)) (mode 0) / np.argmax(x) (mode 1)
    over the flattened x; value is x at that index.  Synchronises."""
    t = on_device(x)
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    n = t.numel()
    res = torch.empty(2, dtype=torch.float64, device=t.device)
    idx = torch.empty(1, dtype=torch.int64, device=t.device)
    _buf, wptr, wbytes = workspace(lib().av_argmax_workspace_size(n))
    check(lib().av_argmax(p(t), dcode(t), n, int(mode), p(idx), p(res), wptr, wbytes,
                          stream_ptr()), "av_argmax")
    return int(idx.item()), float(res[0].item())


def psf_sidelobe(psf, window=(41, 41), threshold=0.35):
    """max_sidelobe of extract_main_lobe(window, threshold, psf plane)."""
    t = on_device(psf)
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    ny, nx = int(t.shape[-2]), int(t.shape[-1])
    if t.numel() != ny * nx:
        raise ValueError("psf_sidelobe takes one (ny, nx) plane")
    out = torch.empty(2, dtype=torch.float64, device=t.device)
    w0, w1 = int(window[0]), int(window[1])
    _buf, wptr, wbytes = workspace(lib().av_psf_sidelobe_workspace_size(ny, nx, w0, w1))
    check(lib().av_psf_sidelobe(p(t), dcode(t), ny, nx, w0, w1, float(threshold), p(out), wptr,
                                wbytes, stream_ptr()), "av_psf_sidelobe")
    r = out.cpu().numpy()
    if r[1] != 0:
        raise ValueError("PSF peak x threshold is negative: the main lobe is undefined")
    return float(r[0])


def plane_sum(x):
    """FP64 sums of each (..., ny, nx) plane of x, as a device tensor of the
    leading shape."""
    t = on_device(x)
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    ny, nx = int(t.shape[-2]), int(t.shape[-1])
    npl = int(t.numel() // max(1, ny * nx))
    out = torch.empty(tuple(t.shape[:-2]), dtype=torch.float64, device=t.device)
    _buf, wptr, wbytes = workspace(lib().av_plane_sum_workspace_size(npl, ny * nx))
    check(lib().av_plane_sum(p(t), dcode(t), npl, ny * nx, p(out), wptr, wbytes, stream_ptr()),
          "av_plane_sum")
    return out


def vis_residual(vis, model, out=None):
    """vis - model (complex64 / complex128 device tensors of one shape)."""
    v = on_device(vis)
    m = on_device(model, v.dtype)
    if out is None:
        out = torch.empty_like(v)
    check(lib().av_vis_residual(p(v), p(m), p(out), dcode(v), v.numel(), stream_ptr()),
          "av_vis_residual")
    return out


# ------------------------------------------------------------------ mosaic --
def cf_phase_product(conv_kernel, phase_gradient):
    """conv_kernel (..., cu, cv) x phase_gradient (cu, cv): complex128."""
    k = on_device(conv_kernel)
    if k.dtype not in (torch.float64, torch.complex128):
        k = k.to(torch.complex128 if k.is_complex() else torch.float64)
    pg = on_device(phase_gradient, torch.complex128)
    cu, cv = int(k.shape[-2]), int(k.shape[-1])
    if tuple(pg.shape) != (cu, cv):
        raise ValueError(f"phase gradient {tuple(pg.shape)} does not match the kernel's "
                         f"({cu}, {cv})")
    out = torch.empty(k.shape, dtype=torch.complex128, device=k.device)
    n_cf = int(k.numel() // (cu * cv))
    check(lib().av_cf_phase_product(p(k), dcode(k), p(pg), p(out), n_cf, cu, cv, stream_ptr()),
          "av_cf_phase_product")
    return out


def mosaic_tiled_ok(support, oversampling, n_img_pol):
    """Whether the binned mosaic gridder covers these functions."""
    ms = int(np.max(np.asarray(support)))
    os_ = np.broadcast_to(np.asarray(oversampling), (2,))
    return (1 <= ms <= 32 and int(os_[0]) == int(os_[1]) and 1 <= int(os_[0]) <= 254
            and int(n_img_pol) <= 4 and (31 + ms) ** 2 * int(n_img_pol) * 16 <= 220 * 1024
            and int(np.min(np.asarray(support))) >= 1)


def mosaic_grid(grid, sum_weight, do_psf, vis, weight, uvw, freq, chan_map, pol_map, cfb_map,
                cfc_map, cfp_map, cf, support, n_uv, delta_lm, oversampling, aperture=False,
                tiled=None):
    """av_mosaic_grid / av_aperture_grid into the device arrays grid
    (complex128) and sum_weight (float64).  tiled (default: when
    mosaic_tiled_ok) bins the samples first and grids tile by tile
    (av_mosaic_tiled_plan + _execute)."""
    w = on_device(weight, torch.float64)
    nt, nb, nchan, npol = (int(s) for s in w.shape)
    v = None if (do_psf or aperture) else on_device(vis, torch.complex128)
    uvw_d = on_device(uvw, torch.float64)
    freq_d = on_device(freq, torch.float64)
    maps = [on_device(np.asarray(m), torch.int32) for m in
            (chan_map, pol_map, cfb_map, cfc_map, cfp_map)]
    sup = on_device(np.asarray(support), torch.int32)
    n_cfb, n_cfc, n_cfp, cu, cv = (int(s) for s in cf.shape)
    os_u, os_v = (int(oversampling[0]), int(oversampling[1])) if np.ndim(oversampling) else \
        (int(oversampling), int(oversampling))
    max_sup = int(np.max(np.asarray(support)))
    args = [p(grid), p(sum_weight), int(bool(do_psf)), p(v), p(w), p(uvw_d), p(freq_d)] + \
        [p(m) for m in maps] + [p(cf), n_cfb, n_cfc, n_cfp, cu, cv, p(sup), max_sup,
                                int(n_uv[0]), int(n_uv[1]), float(delta_lm[0]),
                                float(delta_lm[1]), os_u, os_v, nt, nb, nchan, npol,
                                int(grid.shape[0]), int(grid.shape[1])]
    if aperture:
        _buf, wptr, wbytes = workspace(lib().av_aperture_grid_workspace_size(n_cfb, nchan, npol))
        check(lib().av_aperture_grid(*args, wptr, wbytes, stream_ptr()), "av_aperture_grid")
        return grid, sum_weight
    if tiled is None:
        tiled = mosaic_tiled_ok(support, oversampling, grid.shape[1])
    if not tiled:
        check(lib().av_mosaic_grid(*args, stream_ptr()), "av_mosaic_grid")
        return grid, sum_weight
    n_img_chan = int(grid.shape[0])
    need = lib().av_mosaic_tiled_workspace_size(nt, nb, nchan, int(n_uv[0]), int(n_uv[1]),
                                                n_img_chan, max_sup)
    _buf, wptr, wbytes = workspace(need)
    check(lib().av_mosaic_tiled_plan(p(uvw_d), p(freq_d), p(maps[0]), int(n_uv[0]), int(n_uv[1]),
                                     float(delta_lm[0]), float(delta_lm[1]), max_sup, os_u, nt,
                                     nb, nchan, n_img_chan, wptr, wbytes, stream_ptr()),
          "av_mosaic_tiled_plan")
    check(lib().av_mosaic_tiled_execute(*args, wptr, wbytes, stream_ptr()),
          "av_mosaic_tiled_execute")
    return grid, sum_weight


def airy_pattern(freq, n_pol, dish, blockage, image_size, image_center, cell, ipower, casa,
                 rorder):
    """Primary-beam patterns of make_pb_symmetric (device float64)."""
    f = on_device(np.atleast_1d(np.asarray(freq, dtype=np.float64)), torch.float64)
    dish = np.ascontiguousarray(np.asarray(dish, dtype=np.float64).ravel())
    blk = np.ascontiguousarray(np.asarray(blockage, dtype=np.float64).ravel())
    nd, nf = len(dish), int(f.numel())
    nx, ny = int(image_size[0]), int(image_size[1])
    shape = (nd, nf, int(n_pol), nx, ny) if rorder else (nx, ny, nf, int(n_pol), nd)
    out = torch.empty(shape, dtype=torch.float64, device=f.device)
    check(lib().av_airy_pattern(p(out), dish.ctypes.data, blk.ctypes.data, nd, p(f), nf,
                                int(n_pol), nx, ny, int(image_center[0]), int(image_center[1]),
                                float(cell[0]), float(cell[1]), int(ipower), int(bool(casa)),
                                int(bool(rorder)), stream_ptr()), "av_airy_pattern")
    return out


def plane_rescale(t, mode, s, corr=None, w=None):
    """In place on the contiguous device tensor t (..., ny, nx):
    av_plane_rescale mode 0 (t /= s), 1 (t *= s) or 2
    (t *= s / (corr * w[plane]), corr (ny, nx) and w one value per plane)."""
    assert t.is_contiguous() and t.is_cuda
    ny, nx = int(t.shape[-2]), int(t.shape[-1])
    npl = int(t.numel() // max(1, ny * nx))
    c = None if corr is None else on_device(corr, torch.float64)
    ww = None if w is None else on_device(w, torch.float64).reshape(-1)
    if mode == 2:
        assert c.numel() == ny * nx and ww.numel() == npl
    check(lib().av_plane_rescale(p(t), dcode(t), npl, ny * nx, int(mode), float(s), p(c), p(ww),
                                 stream_ptr()), "av_plane_rescale")
    return t


def apply_pb(t, pb, multiply):
    """In place on the contiguous device tensor t (nt, nc, np, ny, nx), or of
    any shape when pb has the same shape: av_apply_pb with the contiguous
    real device tensor pb (pt, pc, pp, ny, nx)."""
    assert t.is_contiguous() and t.is_cuda and pb.is_contiguous() and pb.is_cuda
    if tuple(t.shape) == tuple(pb.shape):
        n_pix = int(t.shape[-1]) * int(t.shape[-2]) if t.ndim >= 2 else int(t.numel())
        npl = int(t.numel() // max(1, n_pix))
        dims, pdims = (1, 1, npl), (1, 1, npl)
    else:
        if t.ndim != 5 or pb.ndim != 5 or tuple(t.shape[3:]) != tuple(pb.shape[3:]):
            raise ValueError("a primary beam of another shape must be 5-D like the image, "
                             "with the same (l, m) extent")
        n_pix = int(t.shape[3]) * int(t.shape[4])
        dims, pdims = tuple(int(d) for d in t.shape[:3]), tuple(int(d) for d in pb.shape[:3])
    if pb.dtype not in (torch.float32, torch.float64):
        raise TypeError("apply_pb: the primary beam must be float32 or float64")
    check(lib().av_apply_pb(p(t), dcode(t), *dims, p(pb), dcode(pb), *pdims, n_pix,
                            int(bool(multiply)), stream_ptr()), "av_apply_pb")
    return t
