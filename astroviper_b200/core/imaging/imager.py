"""Major/minor-cycle imaging loop on B200.

Drop-in for src/astroviper/core/imaging/imager.py: grid_visibilities
(:54-79), compute_residual_visibilities (:82-85), predict_model_visibilities
(:88-105) and run_imaging_loop (:108-351), same arguments, defaults,
results and side effects on the measurement set.

run_imaging_loop keeps the measurement set on the device for the whole
loop.  The visibilities, weights, flags and uvw are copied in once.  The
gridding and degridding plans (cells and kernel offsets of every sample)
depend only on uvw, the frequencies and the image geometry, so they are
built once and reused by every major cycle.  The dirty image, the Stokes
conversions, the CLEAN of every plane, the model FFT, the prediction and the
residual visibilities stay in HBM.  Each major cycle reads back only the
handful of statistics the iteration controller decides on.  The
VISIBILITY_MODEL and RESIDUAL columns go back to the measurement set once,
at the end.

The arithmetic follows the reference step by step, including two
behaviours of it that a caller can observe:
  * each deconvolve call returns only its own components, so the model of a
    major cycle, the one predicted and the one returned are those of the
    last minor cycle (deconvolution.py:228-256);
  * the PSF is gridded with pixel increment (-cell[0], cell[1])
    (make_point_spread_function.py:45-53) and the dirty images with cell
    itself.
precision "fp32" (default) runs the tiled kernels (complex64 samples, FP64
grid accumulation); "fp64" the plain FP64 kernels.
"""
import logging
from typing import Any, Dict, Optional, Tuple

import numpy as np
import torch

from ... import _kernels as K
from ...config import resolve_precision
from ...gridder import Gridder
from .deconvolution import deconvolve
from .fft import fft_lm_to_uv
from .imaging_utils.corr_to_stokes import image_corr_to_stokes, image_stokes_to_corr
from .imaging_utils.iteration_control import IterationController, merge_return_dicts
from .imaging_utils.return_dict import ReturnDict
from .imaging_utils.standard_degrid import _ModelArray, degrid_spheroid_ms4
from .imaging_utils.standard_grid import grid2image_spheroid_ms4
from .sky_image import make_sky_image

logger = logging.getLogger("astroviper_b200")

_DEFAULT_PARAMS = {
    "image_size": (256, 256),
    "cell_size": None,
    "support": 7,
    "oversampling": 100,
    "algorithm": "hogbom",
    "gain": 0.1,
    "niter": 1000,
    "threshold": 0.0,
    "nmajor": 10,
    "cyclefactor": 1.5,
    "cycleniter": -1,
    "minpsffraction": 0.05,
    "maxpsffraction": 0.8,
    "chan_mode": "cube",
    "corr_type": "linear",
    "stokes": None,
}


def _get_param(params: Dict, key: str):
    return params.get(key, _DEFAULT_PARAMS.get(key))


# ------------------------------------------------------ per-call drop-ins ----
def grid_visibilities(ms4, image_size, cell_size, support: int = 7, oversampling: int = 100,
                      chan_mode: str = "cube", column: str = "VISIBILITY", *, precision=None):
    """Dirty image (n_chan, n_pol, ny, nx) of one column (imager.py:54-79)."""
    n_chan = len(ms4.coords["frequency"])
    n_pol = len(ms4.coords["polarization"])
    ny, nx = image_size
    dirty = np.zeros([n_chan, n_pol, ny, nx], dtype=float)
    grid2image_spheroid_ms4(vis=ms4, resid_array=dirty, pixelincr=np.array(cell_size),
                            support=support, sampling=oversampling, dopsf=False, column=column,
                            chan_mode=chan_mode, precision=precision)
    return dirty


def _wrap_like(ms4, values):
    vis = ms4["VISIBILITY"]
    try:
        import xarray
        return xarray.DataArray(values, coords=vis.coords, dims=vis.dims)
    except ImportError:
        return _ModelArray(values, coords=getattr(vis, "coords", None),
                           dims=getattr(vis, "dims", None))


def compute_residual_visibilities(ms4) -> None:
    """ms4.RESIDUAL = VISIBILITY - VISIBILITY_MODEL (imager.py:82-85)."""
    vis = np.asarray(ms4["VISIBILITY"].data)
    mod = np.asarray(ms4["VISIBILITY_MODEL"].data)
    dt = np.result_type(vis.dtype, mod.dtype)
    a = torch.from_numpy(np.ascontiguousarray(vis, dtype=dt))
    b = torch.from_numpy(np.ascontiguousarray(mod, dtype=dt))
    out = K.vis_residual(a, b)
    ms4["RESIDUAL"] = _wrap_like(ms4, out.cpu().numpy())


def predict_model_visibilities(ms4, model_image, cell_size, support: int = 7,
                               oversampling: int = 100, incremental: bool = False, *,
                               precision=None) -> None:
    """FFT of the model image, degridded into ms4.VISIBILITY_MODEL
    (imager.py:88-105)."""
    model_grid = fft_lm_to_uv(model_image, axes=[2, 3])
    degrid_spheroid_ms4(vis=ms4, grid=model_grid, pixelincr=np.array(cell_size),
                        support=support, sampling=oversampling, incremental=incremental,
                        precision=precision)


# ------------------------------------------------ device-resident session ----
def _host(x):
    return x.data if hasattr(x, "data") and not isinstance(x, np.ndarray) else x


class _ResidentMs4:
    """One measurement set on the device for the imaging loop."""

    def __init__(self, ms4, image_size, cell_size, support, oversampling, chan_mode,
                 precision):
        self.ms4 = ms4
        self.precision = precision
        self.support, self.os = int(support), int(oversampling)
        self.chan_mode = chan_mode
        self.cell = np.array(cell_size, dtype=float)
        self.ny, self.nx = int(image_size[0]), int(image_size[1])
        self.freq = np.asarray(ms4.coords["frequency"].values, dtype=float)
        self.n_chan = len(self.freq)
        self.n_pol = len(ms4.coords["polarization"])
        # side effects of grid2image_spheroid_ms4 on the caller's arrays
        # (standard_grid.py:665-668), applied before the first gridding
        weight = _host(ms4.WEIGHT)
        flag = _host(ms4.FLAG)
        uvw = _host(ms4.UVW)
        weight[flag] = 0.0
        nan_uvw = np.isnan(uvw[:, :, 0]) | np.isnan(uvw[:, :, 1])
        weight[nan_uvw] = 0.0
        self._nan_rows = np.isnan(np.asarray(uvw)).any(axis=-1)
        wdt = torch.float32 if precision == "fp32" else torch.float64
        self.weight = torch.from_numpy(np.ascontiguousarray(weight)).to(K.device(), wdt)
        vdt = torch.complex64 if precision == "fp32" else torch.complex128
        self.vis = torch.from_numpy(np.ascontiguousarray(_host(ms4["VISIBILITY"]))).to(
            K.device(), vdt)
        self.nt, self.nb = int(self.vis.shape[0]), int(self.vis.shape[1])
        self.uvw_grid = torch.from_numpy(np.ascontiguousarray(uvw, dtype=np.float64)).to(
            K.device())
        # degridding sees NaN-uvw rows flagged with uvw 1e9, as
        # degrid_spheroid_ms4 leaves them (standard_degrid.py:557-566)
        uvw_d = np.array(uvw, dtype=np.float64, copy=True)
        uvw_d[self._nan_rows] = 1e9
        fl = np.array(flag, dtype=bool, copy=True)
        fl[self._nan_rows] = True
        self.uvw_degrid = torch.from_numpy(uvw_d).to(K.device())
        self.flag = torch.from_numpy(fl.view(np.uint8)).to(K.device())
        n_img_chan = self.n_chan if chan_mode == "cube" else 1
        if n_img_chan != self.n_chan:
            # grid2image_spheroid_ms4 into an (n_chan, ...) image
            raise RuntimeError(
                f"Shapes of gridded vis and image do no match "
                f"{(n_img_chan, self.n_pol, self.ny, self.nx)} and "
                f"{(self.n_chan, self.n_pol, self.ny, self.nx)}")
        self.chan_map = np.arange(self.n_chan) if chan_mode == "cube" else \
            np.zeros(self.n_chan, dtype=int)
        self.pol_map = np.arange(self.n_pol)
        self.cgk = K.pswf_table(self.os, self.support)
        self.g_dirty = None
        self.g_model = None
        if precision == "fp32":
            # plans of the dirty-image gridding and of the prediction, built
            # once for the whole loop
            self.g_dirty = Gridder(self.uvw_grid, self.freq, (self.ny, self.nx), self.cell,
                                   self.n_pol, support=self.support, oversampling=self.os,
                                   chan_mode=chan_mode)
            self.g_model = Gridder(self.uvw_degrid, self.freq, (self.ny, self.nx), self.cell,
                                   self.n_pol, support=self.support, oversampling=self.os,
                                   chan_mode=chan_mode)
            self.g_dirty._grid_plan()
            self.g_model._degrid_plan(self.n_chan)
        self.model_vis = None
        self.resid_vis = None
        self.predicted = False

    def psf(self):
        """make_psf: (n_freq, n_pol, image_size[1], image_size[0]) float64,
        gridded once with pixel increment (-cell[0], cell[1])."""
        cell = np.array([-self.cell[0], self.cell[1]])
        g, sw = K.grid(None, self.weight, self.uvw_grid, self.freq, self.chan_map,
                       self.pol_map, self.cgk, (self.nx, self.ny), cell, self.support, self.os,
                       len(np.unique(self.chan_map)), self.n_pol, do_psf=True,
                       precision=self.precision)
        return K.grid_to_image(g, sw, apply_corr=True, out_dtype=torch.float64)

    def dirty(self, column):
        """Dirty image of VISIBILITY or RESIDUAL; FP32 mode grids with the
        plan built once for the loop."""
        vis = self.vis if column == "VISIBILITY" else self.resid_vis
        if vis is None:
            raise KeyError(column)
        if self.precision == "fp32":
            g, sw = self.g_dirty.grid(vis, self.weight)
        else:
            g, sw = K.grid(vis, self.weight, self.uvw_grid, self.freq, self.chan_map,
                           self.pol_map, self.cgk, (self.ny, self.nx), self.cell, self.support,
                           self.os, len(np.unique(self.chan_map)), self.n_pol,
                           precision="fp64")
        return K.grid_to_image(g, sw, apply_corr=True, out_dtype=torch.float64)

    def predict(self, model_corr):
        """VISIBILITY_MODEL (store mode) and RESIDUAL of model_corr
        (n_chan, n_corr, ny, nx) on the device."""
        grid = K.fft_shifted(model_corr, inverse=False)
        if grid.dtype != torch.complex128:
            grid = grid.to(torch.complex128)
        if self.precision == "fp32":
            if self.model_vis is None:
                self.model_vis = torch.empty(self.vis.shape, dtype=torch.complex64,
                                             device=self.vis.device)
            self.g_model.degrid(grid, values=self.model_vis, flag=self.flag, accumulate=False)
        else:
            nx, ny = int(grid.shape[-2]), int(grid.shape[-1])
            scale = np.array([-self.cell[0] * nx, -self.cell[1] * ny, 0.0])
            offset = np.array([nx / 2, ny / 2, 0.0])
            g_nchan, g_npol = int(grid.shape[0]), int(grid.shape[1])
            chanmap = (np.arange(self.n_chan) / self.n_chan * g_nchan).astype(int)
            polmap = np.round(np.arange(self.n_pol) % g_npol).astype(int)
            self.model_vis = K.degrid(grid, self.uvw_degrid, self.freq, scale, offset, chanmap,
                                      polmap, self.cgk, self.support, self.os,
                                      values=torch.zeros(self.vis.shape,
                                                         dtype=torch.complex128,
                                                         device=self.vis.device),
                                      flag=self.flag, precision="fp64")
        self.resid_vis = K.vis_residual(self.vis, self.model_vis, out=self.resid_vis)
        if not self.predicted:
            # degrid_spheroid_ms4's side effects on the caller's FLAG and UVW
            flag = _host(self.ms4.FLAG)
            uvw = _host(self.ms4.UVW)
            it, ib = np.where(self._nan_rows)
            flag[it, ib, :, :] = True
            uvw[it, ib, :] = 1e9
        self.predicted = True

    def finish(self):
        """VISIBILITY_MODEL and RESIDUAL back into the measurement set."""
        if not self.predicted:
            return
        model = self.model_vis.to(torch.complex128)
        vis_host = np.asarray(_host(self.ms4["VISIBILITY"]))
        self.ms4["VISIBILITY_MODEL"] = _wrap_like(self.ms4, model.cpu().numpy())
        # VISIBILITY - VISIBILITY_MODEL in numpy's result type (complex128)
        v = torch.from_numpy(np.ascontiguousarray(vis_host)).to(K.device(), torch.complex128)
        resid = K.vis_residual(v, model)
        self.ms4["RESIDUAL"] = _wrap_like(self.ms4, resid.cpu().numpy())


def _abs_max(t):
    return abs(K.argmax(t, 0)[1])


def run_imaging_loop(ms4, params: Dict[str, Any], initial_model: Optional[np.ndarray] = None,
                     output_dir: str = ".", *, precision=None
                     ) -> Tuple[np.ndarray, np.ndarray, ReturnDict, IterationController]:
    """imager.py:108-351: major cycles of grid -> Stokes -> deconvolve ->
    predict -> residual until the IterationController stops; returns (model,
    residual, merged ReturnDict, controller), model and residual as
    (n_chan, n_stokes, ny, nx) float64 arrays."""
    p = {k: _get_param(params, k) for k in _DEFAULT_PARAMS}
    cell_size, image_size = p["cell_size"], p["image_size"]
    support, oversampling = p["support"], p["oversampling"]
    algorithm, gain, niter, threshold = p["algorithm"], p["gain"], p["niter"], p["threshold"]
    nmajor, cyclefactor, cycleniter = p["nmajor"], p["cyclefactor"], p["cycleniter"]
    minpsffraction, maxpsffraction = p["minpsffraction"], p["maxpsffraction"]
    chan_mode, corr_type, stokes = p["chan_mode"], p["corr_type"], p["stokes"]
    if cell_size is None:
        raise ValueError("cell_size must be specified in params")
    precision = resolve_precision(precision)
    ny, nx = image_size
    n_chan = len(ms4.coords["frequency"])
    n_corr = len(ms4.coords["polarization"])
    if stokes is None:
        if n_corr == 2:
            stokes = ["I", "Q"] if corr_type == "linear" else ["I", "V"]
        else:
            stokes = ["I", "Q", "U", "V"]
    n_stokes = len(stokes)
    attrs = getattr(ms4, "attrs", {}) or {}
    phase_center = attrs.get("phase_center", (0.0, 0.0))
    freq_coords = ms4.coords["frequency"].values
    time_coords = [float(ms4.coords["time"].values[0])]
    logger.info(f'Imaging: {ny}x{nx}, {cell_size[0]*206265:.4f}" cells, {n_chan} chan, '
                f"{n_corr}-corr ({corr_type}) -> {stokes}")
    logger.info(f"  niter={niter}, nmajor={nmajor}, threshold={threshold} Jy")

    controller = IterationController(niter=niter, nmajor=nmajor, threshold=threshold, gain=gain,
                                     cyclefactor=cyclefactor, minpsffraction=minpsffraction,
                                     maxpsffraction=maxpsffraction, cycleniter=cycleniter)
    session = _ResidentMs4(ms4, image_size, cell_size, support, oversampling, chan_mode,
                           precision)

    def sky(pol_coords):
        return make_sky_image(phase_center, image_size, cell_size, freq_coords, pol_coords,
                              time_coords)

    # Stokes-I PSF, one plane per frequency (make_psf + image_corr_to_stokes)
    psf_corr = session.psf()
    psf_i = image_corr_to_stokes(psf_corr.unsqueeze(0), corr_type=corr_type, pol_axis=2,
                                 stokes_out=["I"])
    psf_img = sky(["I"])
    psf_img["POINT_SPREAD_FUNCTION"] = psf_i

    if initial_model is not None:
        model_stokes = torch.from_numpy(np.array(initial_model, dtype=float)).to(K.device())
    else:
        model_stokes = torch.zeros((n_chan, n_stokes, ny, nx), dtype=torch.float64,
                                   device=K.device())
    residual_stokes = None
    combined = ReturnDict()
    dirty_img = None
    major_cycle = 0
    while controller.stopcode.major == 0:
        major_cycle += 1
        column = "VISIBILITY" if major_cycle == 1 else "RESIDUAL"
        logger.info(f"=== Major Cycle {major_cycle} === (gridding {column})")
        dirty_corr = session.dirty(column)
        dirty_stokes = image_corr_to_stokes(dirty_corr, corr_type=corr_type, pol_axis=1,
                                            stokes_out=stokes)
        if dirty_img is None:
            dirty_img = sky(stokes)
            dirty_img["RESIDUAL"] = dirty_stokes.unsqueeze(0)
        else:
            dirty_img["RESIDUAL"].values[0].copy_(dirty_stokes)
        if major_cycle == 1:
            temp = ReturnDict()
            temp.add({"peakres": _abs_max(dirty_stokes), "peakres_nomask": _abs_max(dirty_stokes),
                      "masksum": ny * nx, "iter_done": 0, "max_psf_sidelobe": 0.2,
                      "loop_gain": gain}, time=0, pol=0, chan=0)
            cycle_niter, cyclethresh = controller.calculate_cycle_controls(temp)
        else:
            cycle_niter, cyclethresh = controller.calculate_cycle_controls(combined)
        model_img = None
        if K.argmax(model_stokes, 0)[1] != 0:  # np.any(model != 0)
            model_img = sky(stokes)
            model_img["MODEL"] = model_stokes.unsqueeze(0)
        rd, new_model, resid_img = deconvolve(
            dirty_image_xds=dirty_img, psf_xds=psf_img, model_xds=model_img,
            algorithm=algorithm,
            deconv_params={"gain": gain, "niter": cycle_niter, "threshold": cyclethresh},
            output_dir=output_dir)
        model_stokes = new_model["MODEL"].values[0]
        residual_stokes = resid_img["RESIDUAL"].values[0]
        if logger.isEnabledFor(logging.INFO):
            logger.info(f"  peak={_abs_max(residual_stokes):.6f} Jy, "
                        f"model_flux={float(model_stokes[:, 0].sum()):.6f} Jy, "
                        f"niter={cycle_niter}")
        controller.update_counts(rd)
        combined = merge_return_dicts([combined, rd])
        stopcode, stopdesc = controller.check_convergence(rd)
        if stopcode.major != 0:
            logger.info(f"  *** CONVERGED: {stopdesc} ***")
            break
        model_corr = image_stokes_to_corr(model_stokes, corr_type=corr_type, pol_axis=1,
                                          stokes_in=stokes)
        session.predict(model_corr)
    session.finish()
    si = stokes.index("I") if "I" in stokes else 0
    if logger.isEnabledFor(logging.INFO):
        logger.info(f"=== Done: {controller.major_done} major, {controller.total_iter_done} "
                    f"iter, peak={_abs_max(residual_stokes):.6f} Jy, "
                    f"flux={float(model_stokes[:, si].sum()):.6f} Jy ===")
    return (model_stokes.cpu().numpy(), residual_stokes.cpu().numpy(), combined, controller)
