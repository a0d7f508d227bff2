"""Seeded synthetic interferometer data for the standard-gridder workloads.

The reference measures on downloaded measurement sets (Antennae, NGC5921) that
are not available offline; these generators stand in for them with the array
geometry, sizes and value distributions of the benchmark workloads:

* ``array_uvw``: antennas uniform in a disk (r = R sqrt(U), theta = 2 pi U),
  all baselines i < j, Earth-rotation uvw for a source at declination ``dec``
  seen from latitude ``lat`` in 10 s steps symmetric about transit.
* ``point_source_vis``: sum of point sources S_k exp(-2 pi i (u l_k + v m_k))
  plus independent N(0, sigma) noise on the real and imaginary parts.
  The sign puts a source at pixel offset (dx, dy) from the image centre of the
  reference's ``grid2image_spheroid_ms4`` when l = -dx * pixelincr[0],
  m = -dy * pixelincr[1] (see ``source_lm``).

Everything is drawn from ``numpy.random.default_rng(seed)``.
"""
import math

import numpy as np

C_LIGHT = 299792458.0
OMEGA_EARTH = 7.2921150e-5  # rad / s
ARCSEC = math.pi / (180.0 * 3600.0)


def antenna_disk(n_ant, radius_m, rng):
    """East/north/up positions (n_ant, 3), uniform in a disk of radius_m."""
    r = radius_m * np.sqrt(rng.uniform(size=n_ant))
    th = 2.0 * np.pi * rng.uniform(size=n_ant)
    return np.stack([r * np.cos(th), r * np.sin(th), np.zeros(n_ant)], axis=1)


def baselines(enu):
    i, j = np.triu_indices(enu.shape[0], k=1)
    return enu[j] - enu[i]


def array_uvw(n_ant=64, n_time=50, dt_s=10.0, radius_m=2000.0, dec_deg=-30.0,
              lat_deg=-30.0, seed=20260101):
    """uvw (n_time, n_baseline, 3) in metres, float64."""
    rng = np.random.default_rng(seed)
    enu = antenna_disk(n_ant, radius_m, rng)
    b = baselines(enu)
    lat = math.radians(lat_deg)
    dec = math.radians(dec_deg)
    e, n, u_ = b[:, 0], b[:, 1], b[:, 2]
    X = -math.sin(lat) * n + math.cos(lat) * u_
    Y = e
    Z = math.cos(lat) * n + math.sin(lat) * u_
    t = (np.arange(n_time) - (n_time - 1) / 2.0) * dt_s
    H = (OMEGA_EARTH * t)[:, None]
    sH, cH = np.sin(H), np.cos(H)
    uu = sH * X + cH * Y
    vv = -math.sin(dec) * cH * X + math.sin(dec) * sH * Y + math.cos(dec) * Z
    ww = math.cos(dec) * cH * X - math.cos(dec) * sH * Y + math.sin(dec) * Z
    return np.ascontiguousarray(np.stack([uu, vv, ww], axis=-1), dtype=np.float64), rng


def source_lm(dx_pix, dy_pix, pixelincr):
    """Direction cosines that image at pixel offset (dx, dy) from the centre."""
    return -np.asarray(dx_pix) * pixelincr[0], -np.asarray(dy_pix) * pixelincr[1]


def random_sources(rng, n_src, flux_lo, flux_hi, max_offset_pix):
    flux = np.exp(rng.uniform(np.log(flux_lo), np.log(flux_hi), size=n_src))
    dx = rng.uniform(-max_offset_pix, max_offset_pix, size=n_src)
    dy = rng.uniform(-max_offset_pix, max_offset_pix, size=n_src)
    return flux, dx, dy


def point_source_vis(uvw, freq, n_pol, flux, l, m, noise_sigma, rng, dtype=np.complex128,
                     device=None):
    """Visibilities (nt, nb, nchan, n_pol).  With ``device`` (a torch device) the
    sky term is evaluated there in float64 (for the large workloads) and a
    torch tensor is returned; the noise is drawn there with a generator seeded
    from ``rng``."""
    nt, nb = uvw.shape[:2]
    nchan = len(freq)
    if device is None:
        out = np.zeros((nt, nb, nchan), dtype=np.complex128)
        for k in range(len(flux)):
            ph = (uvw[:, :, 0:1] * l[k] + uvw[:, :, 1:2] * m[k]) * (freq[None, None, :] / C_LIGHT)
            out += flux[k] * np.exp(-2j * np.pi * ph)
        vis = np.repeat(out[..., None], n_pol, axis=-1)
        if noise_sigma > 0:
            vis = vis + (rng.normal(0.0, noise_sigma, vis.shape)
                         + 1j * rng.normal(0.0, noise_sigma, vis.shape))
        return np.ascontiguousarray(vis.astype(dtype))
    import torch
    cdt = torch.complex64 if dtype == np.complex64 else torch.complex128
    U = torch.as_tensor(uvw, dtype=torch.float64, device=device)
    F = torch.as_tensor(np.asarray(freq) / C_LIGHT, dtype=torch.float64, device=device)
    out = torch.empty((nt, nb, nchan, n_pol), dtype=cdt, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(int(rng.integers(0, 2**62)))
    step = max(1, (1 << 24) // max(1, nb * nchan))
    for t0 in range(0, nt, step):
        t1 = min(nt, t0 + step)
        sky = torch.zeros((t1 - t0, nb, nchan), dtype=torch.complex128, device=device)
        for k in range(len(flux)):
            ph = (U[t0:t1, :, 0:1] * float(l[k]) + U[t0:t1, :, 1:2] * float(m[k])) * F
            sky += float(flux[k]) * torch.exp(torch.complex(torch.zeros_like(ph),
                                                            -2.0 * math.pi * ph))
        blk = sky[..., None].expand(-1, -1, -1, n_pol)
        if noise_sigma > 0:
            nr = torch.randn(blk.shape, generator=g, dtype=torch.float64, device=device)
            ni = torch.randn(blk.shape, generator=g, dtype=torch.float64, device=device)
            blk = blk + noise_sigma * torch.complex(nr, ni)
        out[t0:t1] = blk.to(cdt)
    return out


# ----------------------------------------------------------------------------
# Named workloads
# ----------------------------------------------------------------------------
def workload_small(seed=20260101, n_time=50):
    """64 antennas in a 2 km disk, 2016 baselines x ``n_time`` steps of 10 s,
    1 channel at 1.4 GHz, 2 polarisations, complex128; 5 point sources
    (0.1-1 Jy log-uniform, offsets within +-200 arcsec) + N(0, 0.01) noise;
    unit weights, natural weighting; 512^2 image of 2 arcsec cells."""
    uvw, rng = array_uvw(64, n_time, seed=seed)
    freq = np.array([1.4e9])
    cell = 2.0 * ARCSEC
    pixelincr = np.array([-cell, cell])
    flux, dx, dy = random_sources(rng, 5, 0.1, 1.0, 200.0 / 2.0)
    l, m = source_lm(dx, dy, pixelincr)
    vis = point_source_vis(uvw, freq, 2, flux, l, m, 0.01, rng)
    weight = np.ones(vis.shape, dtype=np.float64)
    return dict(uvw=uvw, freq=freq, vis=vis, weight=weight, flag=np.zeros(vis.shape, bool),
                pixelincr=pixelincr, image_size=np.array([512, 512]), support=7,
                oversampling=100, sources=(flux, dx, dy))


def workload_large(seed=20260102, n_time=256, n_chan=64, n_pol=4, device=None,
                   time_slice=None):
    """Same array at ``n_time`` steps x ``n_chan`` channels (1.0-1.5 GHz) x
    ``n_pol`` polarisations, complex64 data, unit weights, no flags; 2048^2
    image of 1 arcsec cells, Briggs robust 0.5 (weights computed by the
    caller), support 7, oversampling 100.  With ``device`` the visibilities are
    made on that torch device.  With ``time_slice`` (a slice of the time
    steps) only those steps' visibilities are made; ``uvw`` still holds every
    step (``uvw_all``) and ``uvw`` the sliced ones."""
    uvw_all, rng = array_uvw(64, n_time, seed=seed)
    uvw = uvw_all if time_slice is None else np.ascontiguousarray(uvw_all[time_slice])
    freq = np.linspace(1.0e9, 1.5e9, n_chan)
    cell = 1.0 * ARCSEC
    pixelincr = np.array([-cell, cell])
    flux, dx, dy = random_sources(rng, 5, 0.1, 1.0, 200.0)
    l, m = source_lm(dx, dy, pixelincr)
    vis = point_source_vis(uvw, freq, n_pol, flux, l, m, 0.01, rng, dtype=np.complex64,
                           device=device)
    return dict(uvw=uvw, uvw_all=uvw_all, freq=freq, vis=vis, pixelincr=pixelincr,
                image_size=np.array([2048, 2048]), support=7, oversampling=100, robust=0.5,
                sources=(flux, dx, dy))


def workload_batched(seed=20260105, n_time=496, n_chan=128, n_pol=2, image=1024,
                     flag_lo=0.0, flag_hi=0.6, device=None):
    """Batched uneven gridding: the same array at ``n_time`` steps x
    ``n_chan`` channels (1.0-1.5 GHz) x ``n_pol`` polarisations, complex64,
    cube mode (every channel its own image plane, every polarisation its own
    grid: n_chan x n_pol independent ``image``^2 grids of 2 arcsec cells).
    Each (channel, polarisation) grid has its own flag fraction, uniform in
    [flag_lo, flag_hi); flags are i.i.d. per sample and enter as zero
    weights, so per-grid sample counts are uneven.  With ``device`` the
    visibilities and weights are made on that torch device."""
    uvw, rng = array_uvw(64, n_time, seed=seed)
    freq = np.linspace(1.0e9, 1.5e9, n_chan)
    cell = 2.0 * ARCSEC
    pixelincr = np.array([-cell, cell])
    flux, dx, dy = random_sources(rng, 5, 0.1, 1.0, 100.0)
    l, m = source_lm(dx, dy, pixelincr)
    vis = point_source_vis(uvw, freq, n_pol, flux, l, m, 0.01, rng, dtype=np.complex64,
                           device=device)
    frac = rng.uniform(flag_lo, flag_hi, size=(n_chan, n_pol))
    shape = (len(uvw), uvw.shape[1], n_chan, n_pol)
    if device is None:
        weight = (rng.uniform(size=shape) >= frac[None, None]).astype(np.float32)
    else:
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(int(rng.integers(0, 2**62)))
        u = torch.rand(shape, generator=g, dtype=torch.float32, device=device)
        weight = (u >= torch.as_tensor(frac, dtype=torch.float32, device=device)).to(torch.float32)
    return dict(uvw=uvw, freq=freq, vis=vis, weight=weight, flag_fraction=frac,
                pixelincr=pixelincr, image_size=np.array([image, image]), support=7,
                oversampling=100)


def workload_forward(seed=20260104, n_ant=128, n_time=128, n_chan=4, image=1024, n_blob=200,
                     device=None):
    """Differentiable imaging forward model: ``n_ant`` antennas in the 2 km
    disk, ``n_time`` steps x ``n_chan`` channels (1.0-1.5 GHz) x 1
    polarisation (4.16M visibilities at the defaults), an ``image``^2 truth of
    ``n_blob`` Gaussian blobs (sigma 1-5 px, peak log-uniform 0.01-1,
    centres in the inner 80 % of the field), 1 arcsec cells.  Returns the
    truth as a float32 array (1, 1, image, image)."""
    uvw, rng = array_uvw(n_ant, n_time, seed=seed)
    freq = np.linspace(1.0e9, 1.5e9, n_chan)
    cell = 1.0 * ARCSEC
    truth = np.zeros((image, image), dtype=np.float64)
    yy, xx = np.mgrid[0:image, 0:image]
    lo, hi = 0.1 * image, 0.9 * image
    for _ in range(n_blob):
        cx, cy = rng.uniform(lo, hi, 2)
        sig = rng.uniform(1.0, 5.0)
        amp = 10.0 ** rng.uniform(-2.0, 0.0)
        r = int(np.ceil(5 * sig))
        x0, x1 = max(0, int(cx) - r), min(image, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(image, int(cy) + r + 1)
        truth[y0:y1, x0:x1] += amp * np.exp(-((xx[y0:y1, x0:x1] - cx) ** 2 +
                                              (yy[y0:y1, x0:x1] - cy) ** 2) / (2 * sig * sig))
    return dict(uvw=uvw, freq=freq, cell=np.array([-cell, cell]),
                truth=truth.astype(np.float32)[None, None], noise_sigma=0.01,
                image_size=np.array([image, image]), seed_rng=rng)


def sampling_psf(uvw, freq, image_size, pixelincr):
    """A PSF from the uv sampling of ``uvw`` x ``freq``: nearest-cell counts of
    the samples and their conjugates, inverse FFT, peak-normalised to 1
    (float64, shape image_size)."""
    nx, ny = int(image_size[0]), int(image_size[1])
    u = (uvw[:, :, 0:1] * (freq / C_LIGHT)).ravel()
    v = (uvw[:, :, 1:2] * (freq / C_LIGHT)).ravel()
    iu = np.rint(-u * pixelincr[0] * nx).astype(np.int64)
    iv = np.rint(-v * pixelincr[1] * ny).astype(np.int64)
    g = np.zeros((nx, ny), dtype=np.float64)
    ok = (np.abs(iu) < nx // 2) & (np.abs(iv) < ny // 2)
    np.add.at(g, ((iu[ok] + nx // 2), (iv[ok] + ny // 2)), 1.0)
    np.add.at(g, ((-iu[ok] + nx // 2), (-iv[ok] + ny // 2)), 1.0)
    psf = np.real(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(g))))
    return psf / psf.max()


def clean_workload(nx=2048, psf_factor=2, n_src=50, seed=20260103, n_time=50):
    """Hogbom workload: PSF of the small array's sampling at (psf_factor*nx)^2
    with 1 arcsec cells, peak 1, float32; dirty (nx, nx) = sum of ``n_src``
    point sources (0.005-1 Jy log-uniform, positions uniform in the inner
    0.73 nx) each convolved with the PSF (centre at its (pny/2, pnx/2))."""
    uvw, rng = array_uvw(64, n_time, seed=seed)
    freq = np.array([1.4e9])
    pn = psf_factor * nx
    cell = ARCSEC
    psf = sampling_psf(uvw, freq, (pn, pn), np.array([-cell, cell])).astype(np.float32)
    flux = np.exp(rng.uniform(np.log(0.005), np.log(1.0), size=n_src))
    inner = int(round(0.732421875 * nx))  # 1500 px of 2048
    lo = (nx - inner) // 2
    xs = rng.integers(lo, lo + inner, size=n_src)
    ys = rng.integers(lo, lo + inner, size=n_src)
    dirty = np.zeros((nx, nx), dtype=np.float64)
    for k in range(n_src):
        # dirty[y, x] += S psf[pn/2 + y - ys, pn/2 + x - xs] where inside the PSF
        y0 = pn // 2 - ys[k]
        x0 = pn // 2 - xs[k]
        ya, yb = max(0, -y0), min(nx, pn - y0)
        xa, xb = max(0, -x0), min(nx, pn - x0)
        dirty[ya:yb, xa:xb] += flux[k] * psf[y0 + ya:y0 + yb, x0 + xa:x0 + xb].astype(np.float64)
    return dict(dirty=dirty.astype(np.float32), psf=psf, flux=flux, xs=xs, ys=ys)


class _Column:
    def __init__(self, values, dims):
        self.values = values
        self.data = values
        self.dims = tuple(dims)
        self.coords = {}

    def __len__(self):
        return len(self.values)


class Ms4Node:
    """A measurement-set node shaped like an xradio MSv4 DataTree node as
    far as the imaging path reads one: VISIBILITY / UVW / WEIGHT / FLAG
    columns with .data / .values / .dims, the frequency / polarization / time
    coordinates, dims and the phase_center attribute; columns can be added
    (VISIBILITY_MODEL, RESIDUAL)."""

    def __init__(self, vis, uvw, weight, flag, freq, pols, phase_center=(0.0, 0.0), dt_s=10.0):
        self._d = {}
        vdims = ("time", "baseline_id", "frequency", "polarization")
        self["VISIBILITY"] = _Column(vis, vdims)
        self["UVW"] = _Column(uvw, ("time", "baseline_id", "uvw_label"))
        self["WEIGHT"] = _Column(weight, vdims)
        self["FLAG"] = _Column(flag, vdims)
        self.frequency = _Column(np.asarray(freq), ("frequency",))
        self.coords = {"frequency": _Column(np.asarray(freq), ("frequency",)),
                       "polarization": _Column(np.asarray(pols), ("polarization",)),
                       "time": _Column(np.arange(vis.shape[0]) * dt_s, ("time",))}
        nt, nb, nc, npol = vis.shape
        self.dims = {"time": nt, "baseline_id": nb, "frequency": nc, "polarization": npol}
        self.attrs = {"phase_center": tuple(phase_center)}

    def __getitem__(self, k):
        return self._d[k]

    def __setitem__(self, k, v):
        self._d[k] = v
        setattr(self, k, v)

    def __contains__(self, k):
        return k in self._d


def ms4_small(seed=20260101, n_time=50):
    """workload_small as an Ms4Node (XX, YY) and its imaging parameters
    (512^2, 2 arcsec cells, support 7, oversampling 100)."""
    W = workload_small(seed=seed, n_time=n_time)
    node = Ms4Node(W["vis"].copy(), W["uvw"].copy(), W["weight"].copy(), W["flag"].copy(),
                   W["freq"], ["XX", "YY"])
    cell = np.abs(W["pixelincr"])
    return node, {"image_size": (512, 512), "cell_size": (float(cell[0]), float(cell[1])),
                  "support": 7, "oversampling": 100}
