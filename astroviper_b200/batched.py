"""Batched gridding of many independent grids of uneven size in one launch.

Cube-mode gridding (standard_grid_jit, standard_grid.py:246-432, with
chan_mode "cube": every channel its own image plane) of n_chan x n_pol
independent grids.  Per-grid sample counts differ when weights are zero
(flagged samples; the reference skips zero-weighted data, standard_grid.py:378),
so the grids are uneven.

The binning plan is built once from uvw / freq.  Every call then runs the
persistent tiled gridder once over all grids: its CTAs take record chunks from
one counter, so grids with few samples free their SMs for the others with no
host involvement.  With ``drop_flagged=True`` each call also bins its own
batch's samples from the weights (av_grid_tiled_plan_weighted), leaving out
those whose every weight is zero or NaN, so heavily flagged grids take less
work.  Only the cells the plan can touch are cleared between calls
(av_grid_tiled_clear); the rest of the grids stays zero from construction.
With ``graph=True`` the call (the weighted plan when it applies, the clears and
the gridding launch) is captured as a CUDA graph on first use and replayed
afterwards; a replay takes a fresh batch of visibilities and weights for the
uv coverage given at construction, copied into the graph's static buffers.
Launch knobs come from the autotuner (astroviper_b200.autotune) when
``tune=True``.
"""
import numpy as np
import torch

from . import _kernels as K
from ._lib import AV_C64, AV_F32, check, lib


class BatchedGridder:
    def __init__(self, uvw, freq, image_size, cell_size, npol, support=7, oversampling=100,
                 graph=True, tune=False, grid_dtype=torch.complex128, drop_flagged=False,
                 alias_tol=1e-2):
        """support: the kernel support, or "auto" for the smallest of 7 and 9
        whose aliasing at the edge of the inner 80 % of the field is at most
        alias_tol (autotune.choose_support; it changes the result, so it is an
        explicit choice).  tune: let the autotuner choose the launch knobs."""
        self.dev = K.device()
        self.uvw = K.on_device(uvw, torch.float64)
        self.freq = K.on_device(freq, torch.float64)
        self.nt, self.nb = int(self.uvw.shape[0]), int(self.uvw.shape[1])
        self.nchan = int(self.freq.numel())
        self.npol = int(npol)
        self.n_u, self.n_v = int(image_size[0]), int(image_size[1])
        self.cell = (float(cell_size[0]), float(cell_size[1]))
        self.os = int(oversampling)
        self.alias = None
        if support == "auto":
            from . import autotune
            support, self.alias = autotune.choose_support((7, 9), self.os, alias_tol)
        self.support = int(support)
        self.graph = bool(graph)
        self.tune = bool(tune)
        self.drop_flagged = bool(drop_flagged)
        if self.npol < 1 or self.npol > 4:
            raise ValueError("npol must be in [1, 4]")
        self.chan_map = torch.arange(self.nchan, dtype=torch.int32, device=self.dev)
        self.pol_map = torch.arange(self.npol, dtype=torch.int32, device=self.dev)
        self.cgk = K.pswf_table(self.os, self.support)
        need = lib().av_grid_tiled_workspace_size(self.nt, self.nb, self.nchan, self.n_u, self.n_v,
                                                  self.nchan, self.support)
        # the plan of every sample: its tiles bound what any call can touch
        self._ws = K.workspace(need)
        check(lib().av_grid_tiled_plan(K.p(self.uvw), K.p(self.freq), K.p(self.chan_map),
                                       self.n_u, self.n_v, self.cell[0], self.cell[1],
                                       self.support, self.os, self.nt, self.nb, self.nchan,
                                       self.nchan, self._ws[1], self._ws[2], K.stream_ptr()),
              "av_grid_tiled_plan")
        # each call's plan without its fully flagged samples
        self._wws = K.workspace(need) if self.drop_flagged else None
        self._cleared = True  # the grids are all zero until the first launch
        self.grid = torch.zeros((self.nchan, self.npol, self.n_u, self.n_v), dtype=grid_dtype,
                                device=self.dev)
        self.sum_weight = torch.zeros((self.nchan, self.npol), dtype=torch.float64,
                                      device=self.dev)
        self._g = None
        self._vis = None
        self._wt = None

    @property
    def shape(self):
        return (self.nt, self.nb, self.nchan, self.npol)

    def tune_key(self):
        from . import autotune
        return autotune.key("grid", support=self.support, n_u=self.n_u, n_v=self.n_v,
                            npol=self.npol, planes=self.nchan)

    def _launch(self, vis, wt):
        if not self._cleared:
            # only the cells the full plan can touch were ever written
            check(lib().av_grid_tiled_clear(
                K.p(self.grid), K.dcode(self.grid), self.npol, self.n_u, self.n_v, self.support,
                self.nt, self.nb, self.nchan, self.nchan, self._ws[1], self._ws[2],
                K.stream_ptr()), "av_grid_tiled_clear")
        self._cleared = False
        self.sum_weight.zero_()
        ws = self._ws
        if self.drop_flagged:
            ws = self._wws
            check(lib().av_grid_tiled_plan_weighted(
                K.p(self.uvw), K.p(self.freq), K.p(self.chan_map), K.p(wt), self.npol, self.n_u,
                self.n_v, self.cell[0], self.cell[1], self.support, self.os, self.nt, self.nb,
                self.nchan, self.nchan, ws[1], ws[2], K.stream_ptr()),
                "av_grid_tiled_plan_weighted")
        check(lib().av_grid_tiled_execute(
            K.p(self.grid), K.dcode(self.grid), K.p(self.sum_weight), 0, K.p(vis), AV_C64,
            K.p(wt), AV_F32, K.p(self.pol_map), K.p(self.cgk), self.n_u, self.n_v, self.support,
            self.os, self.nt, self.nb, self.nchan, self.npol, self.nchan, self.npol,
            ws[1], ws[2], K.stream_ptr()), "av_grid_tiled_execute")

    def _inputs(self, vis, weight):
        v = K.on_device(vis, torch.complex64).contiguous()
        w = K.on_device(weight, torch.float32).contiguous()
        if tuple(v.shape) != self.shape or tuple(w.shape) != self.shape:
            raise ValueError(f"vis and weight must have shape {self.shape}")
        return v, w

    def __call__(self, vis, weight):
        """Grid all (channel, polarisation) grids; returns (grid, sum_weight),
        the object's own buffers (overwritten by the next call)."""
        v, w = self._inputs(vis, weight)
        if self.tune:
            from . import autotune
            autotune.ensure(self.tune_key(), lambda: self._launch(v, w))
        if not self.graph:
            self._launch(v, w)
            return self.grid, self.sum_weight
        if self._g is None:
            self._vis = v.clone()
            self._wt = w.clone()
            self._launch(self._vis, self._wt)  # first launch outside capture
            torch.cuda.synchronize(self.dev)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._launch(self._vis, self._wt)
            self._g = g
        else:
            if v.data_ptr() != self._vis.data_ptr():
                self._vis.copy_(v)
            if w.data_ptr() != self._wt.data_ptr():
                self._wt.copy_(w)
        self._g.replay()
        return self.grid, self.sum_weight

    def static_inputs(self):
        """The graph's input buffers (after the first call): writing the next
        batch into them directly skips the copy of __call__."""
        return self._vis, self._wt


class PerGridGridder:
    """The same grids, one launch per (channel, polarisation) grid with a plan
    per channel: the baseline the batched launch is compared with."""

    def __init__(self, uvw, freq, image_size, cell_size, npol, support=7, oversampling=100):
        self.dev = K.device()
        self.uvw = K.on_device(uvw, torch.float64)
        freq = np.asarray(freq, dtype=np.float64)
        self.nt, self.nb = int(self.uvw.shape[0]), int(self.uvw.shape[1])
        self.nchan, self.npol = len(freq), int(npol)
        self.n_u, self.n_v = int(image_size[0]), int(image_size[1])
        self.cell = (float(cell_size[0]), float(cell_size[1]))
        self.support, self.os = int(support), int(oversampling)
        self.cgk = K.pswf_table(self.os, self.support)
        self.zero_map = torch.zeros(1, dtype=torch.int32, device=self.dev)
        need = lib().av_grid_tiled_workspace_size(self.nt, self.nb, 1, self.n_u, self.n_v, 1,
                                                  self.support)
        self.freqs = [K.on_device(freq[c:c + 1], torch.float64) for c in range(self.nchan)]
        self.plans = []
        for c in range(self.nchan):
            ws = K.workspace(need)
            check(lib().av_grid_tiled_plan(K.p(self.uvw), K.p(self.freqs[c]), K.p(self.zero_map),
                                           self.n_u, self.n_v, self.cell[0], self.cell[1],
                                           self.support, self.os, self.nt, self.nb, 1, 1, ws[1],
                                           ws[2], K.stream_ptr()), "av_grid_tiled_plan")
            self.plans.append(ws)
        self.grid = torch.zeros((self.nchan, self.npol, self.n_u, self.n_v),
                                dtype=torch.complex128, device=self.dev)
        self.sum_weight = torch.zeros((self.nchan, self.npol), dtype=torch.float64,
                                      device=self.dev)

    @staticmethod
    def split(vis, weight):
        """Per-grid contiguous inputs [(vis (nt, nb, 1, 1), weight), ...] in
        (channel, polarisation) order: the layout this baseline reads."""
        v = torch.as_tensor(vis)
        w = torch.as_tensor(weight)
        out = []
        for c in range(v.shape[2]):
            for q in range(v.shape[3]):
                out.append((v[:, :, c:c + 1, q:q + 1].contiguous().to(torch.complex64),
                            w[:, :, c:c + 1, q:q + 1].contiguous().to(torch.float32)))
        return out

    def __call__(self, parts):
        self.grid.zero_()
        self.sum_weight.zero_()
        for idx, (v, w) in enumerate(parts):
            c, q = divmod(idx, self.npol)
            ws = self.plans[c]
            check(lib().av_grid_tiled_execute(
                K.p(self.grid[c, q]), K.dcode(self.grid), K.p(self.sum_weight[c, q:q + 1]), 0,
                K.p(v), AV_C64, K.p(w), AV_F32, K.p(self.zero_map), K.p(self.cgk), self.n_u,
                self.n_v, self.support, self.os, self.nt, self.nb, 1, 1, 1, 1, ws[1], ws[2],
                K.stream_ptr()), "av_grid_tiled_execute")
        return self.grid, self.sum_weight
