"""Device-resident gridding and degridding of one set of samples.

The reference re-derives every sample's cell and kernel offsets on each call
(standard_grid.py:318-352, standard_degrid.py:435-450).  They depend only on
uvw, the frequencies and the image geometry, so a Gridder bins the samples
once per convention (av_grid_tiled_plan / av_degrid_tiled_plan) and then
grids / degrids any number of visibility sets with av_*_tiled_execute - the
pattern of a major/minor-cycle imager, where the same uv coverage is gridded
and degridded every cycle.  All arrays stay on the device.
"""
import numpy as np
import torch

from . import _kernels as K
from ._lib import AV_C64, AV_F32, check, lib

C_LIGHT = 299792458.0


class Gridder:
    """Plans for gridding (standard_grid_jit conventions) and degridding
    (dgrid_numba conventions) of samples uvw (nt, nb, 3) at freq (nchan)
    onto (n_img_chan, n_img_pol, nx, ny) grids of cell_size (radians, as
    passed to the reference: pixelincr)."""

    def __init__(self, uvw, freq, image_size, cell_size, npol, support=7, oversampling=100,
                 chan_mode="continuum", n_img_pol=None, deterministic=False):
        """deterministic: grid() adds bit-identical results from call to call
        (plans ordered by row, fixed-point sums: av_grid_tiled_execute_det;
        supports 3-8, about twice the gridding time)."""
        self.dev = K.device()
        self.uvw = K.on_device(uvw, torch.float64)
        self.freq = K.on_device(freq, torch.float64)
        self.nt, self.nb = int(self.uvw.shape[0]), int(self.uvw.shape[1])
        self.nchan = int(self.freq.numel())
        self.npol = int(npol)
        self.nx, self.ny = int(image_size[0]), int(image_size[1])
        self.cell = (float(cell_size[0]), float(cell_size[1]))
        self.support, self.os = int(support), int(oversampling)
        if chan_mode == "cube":
            self.n_img_chan = self.nchan
            cm = np.arange(self.nchan)
        else:
            self.n_img_chan = 1
            cm = np.zeros(self.nchan, dtype=int)
        self._cm_host = np.asarray(cm)
        self.chan_map = K.on_device(cm, torch.int32)
        self.n_img_pol = int(n_img_pol if n_img_pol is not None else npol)
        self.pol_map = K.on_device(np.arange(self.npol) % self.n_img_pol, torch.int32)
        self.cgk = K.pswf_table(self.os, self.support)
        self._gplan = None
        self._dplan = None
        # plan() builds one plan for both directions where it can; False
        # builds the two separately
        self.shared_plan = True
        self.deterministic = bool(deterministic)
        if self.deterministic and not 3 <= self.support <= 8:
            raise ValueError("deterministic gridding covers supports 3-8")
        self._det_ws = None
        self._dpolmaps = {}

    # ------------------------------------------------------------- gridding
    def _grid_plan(self):
        if self._gplan is None:
            need = lib().av_grid_tiled_workspace_size(self.nt, self.nb, self.nchan, self.nx,
                                                      self.ny, self.n_img_chan, self.support)
            ws = K.workspace(need)
            check(lib().av_grid_tiled_plan(K.p(self.uvw), K.p(self.freq), K.p(self.chan_map),
                                           self.nx, self.ny, self.cell[0], self.cell[1],
                                           self.support, self.os, self.nt, self.nb, self.nchan,
                                           self.n_img_chan, ws[1], ws[2], K.stream_ptr()),
                  "av_grid_tiled_plan")
            self._order_rows(ws)
            self._gplan = ws
        return self._gplan

    def _order_rows(self, ws):
        if self.deterministic:
            check(lib().av_tiled_plan_order_rows(self.nt, self.nb, self.nchan, self.nx, self.ny,
                                                 self.n_img_chan, self.support, ws[1], ws[2],
                                                 K.stream_ptr()), "av_tiled_plan_order_rows")

    def clear_grid(self, grid):
        """Zeroes the cells this Gridder's gridding plan can touch (the
        footprint regions of its tiles): enough before gridding into a grid
        whose other cells are zero, such as one that held this Gridder's
        previous result (av_grid_tiled_clear)."""
        ws = self._grid_plan()
        check(lib().av_grid_tiled_clear(K.p(grid), K.dcode(grid), int(grid.shape[1]), self.nx,
                                        self.ny, self.support, self.nt, self.nb, self.nchan,
                                        self.n_img_chan, ws[1], ws[2], K.stream_ptr()),
              "av_grid_tiled_clear")
        return grid

    def new_grid(self, dtype=torch.complex128):
        return torch.zeros((self.n_img_chan, self.n_img_pol, self.nx, self.ny), dtype=dtype,
                           device=self.dev)

    def grid(self, vis, weight, grid=None, sum_weight=None, do_psf=False, replan=False):
        """grid += sum over samples (FP64 accumulation of complex64 vis x
        float32 weights); returns (grid, sum_weight)."""
        if replan:
            self._gplan = None
        ws = self._grid_plan()
        if grid is None:
            grid = self.new_grid()
        if sum_weight is None:
            sum_weight = torch.zeros((self.n_img_chan, self.n_img_pol), dtype=torch.float64,
                                     device=self.dev)
        w = K.on_device(weight, torch.float32)
        v = None if do_psf else K.on_device(vis, torch.complex64)
        if self.deterministic:
            need = lib().av_grid_tiled_det_workspace_size(self.n_img_chan, self.n_img_pol,
                                                          self.nx, self.ny)
            if self._det_ws is None or self._det_ws[2] < need:
                self._det_ws = K.workspace(need)
            dws = self._det_ws
            check(lib().av_grid_tiled_execute_det(
                K.p(grid), K.dcode(grid), K.p(sum_weight), int(bool(do_psf)), K.p(v), AV_C64,
                K.p(w), AV_F32, K.p(self.pol_map), K.p(self.cgk), self.nx, self.ny,
                self.support, self.os, self.nt, self.nb, self.nchan, self.npol, self.n_img_chan,
                self.n_img_pol, ws[1], ws[2], dws[1], dws[2], K.stream_ptr()),
                "av_grid_tiled_execute_det")
            return grid, sum_weight
        check(lib().av_grid_tiled_execute(K.p(grid), K.dcode(grid), K.p(sum_weight),
                                          int(bool(do_psf)), K.p(v), AV_C64, K.p(w), AV_F32,
                                          K.p(self.pol_map), K.p(self.cgk), self.nx, self.ny,
                                          self.support, self.os, self.nt, self.nb, self.nchan,
                                          self.npol, self.n_img_chan, self.n_img_pol, ws[1],
                                          ws[2], K.stream_ptr()), "av_grid_tiled_execute")
        return grid, sum_weight

    def plan(self, g_nchan=None):
        """Build the gridding and the degridding plan (for a grid of g_nchan
        channels, default n_img_chan).  When the degridder's channel map
        int(i / nchan * g_nchan) equals the gridder's (continuum and cube
        images), one shared plan serves both (av_tiled_plan_shared): the two
        conventions differ only in their rounding, and the rare samples where
        that matters are degridded apart in FP64.  Otherwise the two plans
        are built concurrently on two streams: both depend only on uvw, the
        frequencies and the geometry, and neither fills the GPU alone.  Later
        calls on the current stream see the plans."""
        key = int(self.n_img_chan if g_nchan is None else g_nchan)
        dmap = (np.arange(self.nchan) / self.nchan * key).astype(int)
        if (self.shared_plan and key == self.n_img_chan
                and np.array_equal(dmap, self._cm_host)):
            need = lib().av_grid_tiled_workspace_size(self.nt, self.nb, self.nchan, self.nx,
                                                      self.ny, self.n_img_chan, self.support)
            ws = K.workspace(need)
            check(lib().av_tiled_plan_shared(K.p(self.uvw), K.p(self.freq), K.p(self.chan_map),
                                             self.nx, self.ny, self.cell[0], self.cell[1],
                                             self.support, self.os, self.nt, self.nb,
                                             self.nchan, self.n_img_chan, ws[1], ws[2],
                                             K.stream_ptr()), "av_tiled_plan_shared")
            self._order_rows(ws)
            self._gplan = ws
            self._dplan = (key, ws)
            return
        cur = torch.cuda.current_stream(self.dev)
        if getattr(self, "_side", None) is None:
            self._side = torch.cuda.Stream(self.dev)
        self._side.wait_stream(cur)
        with torch.cuda.stream(self._side):
            ws = self._degrid_plan(self.n_img_chan if g_nchan is None else g_nchan)
            self._dchanmap.record_stream(cur)
        ws[0].record_stream(cur)
        self._grid_plan()
        cur.wait_stream(self._side)

    # ----------------------------------------------------------- degridding
    def _degrid_polmap(self, g_npol):
        """Device polarisation map i % g_npol, made once per grid: an upload
        from pageable memory on every call would wait for the stream."""
        pm = self._dpolmaps.get(g_npol)
        if pm is None:
            pm = K.on_device(np.arange(self.npol) % g_npol, torch.int32)
            self._dpolmaps[g_npol] = pm
        return pm

    def _degrid_plan(self, g_nchan):
        key = int(g_nchan)
        if self._dplan is None or self._dplan[0] != key:
            need = lib().av_degrid_tiled_workspace_size(self.nt, self.nb, self.nchan, self.nx,
                                                        self.ny, key, self.support)
            ws = K.workspace(need)
            self._dchanmap = K.on_device(
                (np.arange(self.nchan) / self.nchan * key).astype(int), torch.int32)
            sx, sy = -self.cell[0] * self.nx, -self.cell[1] * self.ny
            check(lib().av_degrid_tiled_plan(K.p(self.uvw), K.p(self.freq), K.p(self._dchanmap),
                                             sx, sy, self.nx / 2, self.ny / 2, key, self.nx,
                                             self.ny, self.support, self.os, self.nt, self.nb,
                                             self.nchan, ws[1], ws[2], K.stream_ptr()),
                  "av_degrid_tiled_plan")
            self._dplan = (key, ws)
        return self._dplan[1]

    def degrid(self, grid, values=None, flag=None, dphase=None, accumulate=False):
        """Model visibilities of grid with the conventions of
        degrid_spheroid_ms4 (chanmap int(i/nchan*g_nchan), polmap i % g_npol):
        values = model (zeros for skipped samples), or values += model with
        accumulate.  values (nt, nb, nchan, npol) complex64 / complex128 is
        allocated when None."""
        g = grid if grid.is_contiguous() else grid.contiguous()
        g_nchan, g_npol = int(g.shape[0]), int(g.shape[1])
        ws = self._degrid_plan(g_nchan)
        if values is None:
            values = torch.empty((self.nt, self.nb, self.nchan, self.npol),
                                 dtype=torch.complex64, device=self.dev)
            accumulate = False
        pm = self._degrid_polmap(g_npol)
        fl = None if flag is None else K.on_device(flag).to(torch.uint8).contiguous()
        dph = None if dphase is None else K.on_device(dphase, torch.float64)
        check(lib().av_degrid_tiled_execute(K.p(dph), K.p(values), K.dcode(values),
                                            int(bool(accumulate)), K.p(fl),
                                            K.p(g), K.dcode(g), g_nchan, g_npol, self.nx,
                                            self.ny, K.p(self.freq), self.support, self.os,
                                            K.p(self.cgk), K.p(pm), self.nt, self.nb,
                                            self.nchan, self.npol, ws[1], ws[2],
                                            K.stream_ptr()), "av_degrid_tiled_execute")
        return values

    # --------------------------------------------------------------- images
    def image(self, grid, sum_weight, out_dtype=torch.float64):
        """Grid-corrected image of grid2image_spheroid_ms4 (FP64 transform)."""
        return K.grid_to_image(grid, sum_weight, apply_corr=True, out_dtype=out_dtype)
