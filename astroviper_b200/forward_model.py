"""Differentiable degridding forward model and chi-squared image solve.

The model maps a real image x (n_img_chan, n_img_pol, nx, ny) to model
visibilities

    V = D F C^-1 x

with C the grid-correction image (gcf_prolate_spheroidal.py:73-79), F the
centred FFT of fft_lm_to_uv (fft.py:5) and D the degridder (dgrid_numba,
standard_degrid.py:388-485, with the maps of degrid_spheroid_ms4).  The
reference predicts with D F x (imager.py:88-105, no correction); dividing by
C first makes D F C^-1 the adjoint-consistent partner of the dirty image of
grid2image_spheroid_ms4.

It is a torch.autograd.Function whose backward is the hand-written adjoint

    x_bar = C^-1 Re(F^H D^H V_bar),

D^H being the gridding of V_bar with per-sample weight w / sum(w) at the
degridder's own positions (av_degrid_tiled_adjoint / av_degrid_plain_adjoint)
and F^H the unnormalised centred inverse FFT of av_grid_to_image.

precision "fp32": complex64 model visibilities from the tiled degridder, FP64
adjoint accumulation; "fp64": the plain FP64 kernels (for gradcheck).  The
FFTs are FP64 in both.
"""
import numpy as np
import torch

from . import _kernels as K
from ._lib import AV_C64, AV_C128, check, lib

C_LIGHT = 299792458.0


class ForwardModel:
    def __init__(self, uvw, freq, image_size, cell_size, npol=1, support=7, oversampling=100,
                 n_img_chan=1, n_img_pol=None, flag=None, precision="fp32"):
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self.precision = precision
        self.dev = K.device()
        self.uvw = K.on_device(uvw, torch.float64)
        self.freq = K.on_device(freq, torch.float64)
        self.nt, self.nb = int(self.uvw.shape[0]), int(self.uvw.shape[1])
        self.nchan = int(self.freq.numel())
        self.npol = int(npol)
        self.nx, self.ny = int(image_size[0]), int(image_size[1])
        self.cell = (float(cell_size[0]), float(cell_size[1]))
        self.support, self.os = int(support), int(oversampling)
        self.n_img_chan = int(n_img_chan)
        self.n_img_pol = int(n_img_pol if n_img_pol is not None else npol)
        # the maps of degrid_spheroid_ms4 (standard_degrid.py:580-584)
        self.chanmap = K.on_device(
            (np.arange(self.nchan) / self.nchan * self.n_img_chan).astype(int), torch.int32)
        self.polmap = K.on_device(np.round(np.arange(self.npol) % self.n_img_pol).astype(int),
                                  torch.int32)
        self.flag = None if flag is None else K.on_device(flag).to(torch.uint8).contiguous()
        self.cgk = K.pswf_table(self.os, self.support)
        self.scale = (-self.cell[0] * self.nx, -self.cell[1] * self.ny)
        self.offset = (self.nx / 2, self.ny / 2)
        self._plan = None
        if precision == "fp32":
            need = lib().av_degrid_tiled_workspace_size(self.nt, self.nb, self.nchan, self.nx,
                                                        self.ny, self.n_img_chan, self.support)
            self._plan = K.workspace(need)
            check(lib().av_degrid_tiled_plan(K.p(self.uvw), K.p(self.freq), K.p(self.chanmap),
                                             self.scale[0], self.scale[1], self.offset[0],
                                             self.offset[1], self.n_img_chan, self.nx, self.ny,
                                             self.support, self.os, self.nt, self.nb, self.nchan,
                                             self._plan[1], self._plan[2], K.stream_ptr()),
                  "av_degrid_tiled_plan")

    @property
    def image_shape(self):
        return (self.n_img_chan, self.n_img_pol, self.nx, self.ny)

    @property
    def vis_shape(self):
        return (self.nt, self.nb, self.nchan, self.npol)

    # ---------------------------------------------------------------- pieces
    def image_to_grid(self, image):
        """F C^-1 x as a complex128 grid."""
        img = image.detach().contiguous()
        assert tuple(img.shape) == self.image_shape and img.dtype in (torch.float32,
                                                                     torch.float64)
        grid = torch.empty(self.image_shape, dtype=torch.complex128, device=self.dev)
        npl = self.n_img_chan * self.n_img_pol
        _buf, wptr, wbytes = K.workspace(lib().av_grid_to_image_workspace_size(npl, self.nx,
                                                                               self.ny))
        check(lib().av_image_to_grid(K.p(img), K.dcode(img), K.p(grid), AV_C128, npl, self.nx,
                                     self.ny, 1, wptr, wbytes, K.stream_ptr()),
              "av_image_to_grid")
        return grid

    def degrid(self, grid):
        """D grid: model visibilities (complex64 in fp32, complex128 in fp64)."""
        if self.precision == "fp64":
            vals = torch.zeros(self.vis_shape, dtype=torch.complex128, device=self.dev)
            g = grid.to(torch.complex128).contiguous()
            check(lib().av_degrid_plain(K.p(self.uvw), None, K.p(vals), AV_C128, K.p(self.flag),
                                        self.scale[0], self.scale[1], self.offset[0],
                                        self.offset[1], K.p(g), AV_C128, self.n_img_chan,
                                        self.n_img_pol, self.nx, self.ny, K.p(self.freq),
                                        C_LIGHT, self.support, self.os, K.p(self.cgk),
                                        K.p(self.chanmap), K.p(self.polmap), self.nt, self.nb,
                                        self.nchan, self.npol, K.stream_ptr()), "av_degrid_plain")
            return vals
        vals = torch.empty(self.vis_shape, dtype=torch.complex64, device=self.dev)
        g = grid.contiguous()
        check(lib().av_degrid_tiled_execute(None, K.p(vals), AV_C64, 0, K.p(self.flag), K.p(g),
                                            K.dcode(g), self.n_img_chan, self.n_img_pol, self.nx,
                                            self.ny, K.p(self.freq), self.support, self.os,
                                            K.p(self.cgk), K.p(self.polmap), self.nt, self.nb,
                                            self.nchan, self.npol, self._plan[1], self._plan[2],
                                            K.stream_ptr()), "av_degrid_tiled_execute")
        return vals

    def degrid_adjoint(self, values):
        """D^H values: complex128 grid."""
        grid = torch.zeros(self.image_shape, dtype=torch.complex128, device=self.dev)
        if self.precision == "fp64":
            v = values.detach().to(torch.complex128).contiguous()
            check(lib().av_degrid_plain_adjoint(
                K.p(self.uvw), None, K.p(v), AV_C128, K.p(self.flag), self.scale[0],
                self.scale[1], self.offset[0], self.offset[1], K.p(grid), AV_C128,
                self.n_img_chan, self.n_img_pol, self.nx, self.ny, K.p(self.freq), C_LIGHT,
                self.support, self.os, K.p(self.cgk), K.p(self.chanmap), K.p(self.polmap),
                self.nt, self.nb, self.nchan, self.npol, K.stream_ptr()),
                "av_degrid_plain_adjoint")
            return grid
        v = values.detach().to(torch.complex64).contiguous()
        check(lib().av_degrid_tiled_adjoint(K.p(grid), AV_C128, K.p(v), AV_C64, K.p(self.flag),
                                            self.n_img_chan, self.n_img_pol, self.nx, self.ny,
                                            self.support, self.os, K.p(self.cgk),
                                            K.p(self.polmap), self.nt, self.nb, self.nchan,
                                            self.npol, self._plan[1], self._plan[2],
                                            K.stream_ptr()), "av_degrid_tiled_adjoint")
        return grid

    def grid_to_image(self, grid, dtype=torch.float64):
        """C^-1 Re(F^H grid) (the unnormalised transform, no sum of weights)."""
        return K.grid_to_image(grid, None, apply_corr=True, out_dtype=dtype)

    # ------------------------------------------------------------- operators
    def forward_op(self, image):
        return self.degrid(self.image_to_grid(image))

    def adjoint_op(self, values, dtype=torch.float64):
        return self.grid_to_image(self.degrid_adjoint(values), dtype=dtype)

    def __call__(self, image):
        return _Degrid.apply(image, self)


class _Degrid(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, model):
        ctx.model = model
        ctx.dtype = image.dtype
        return model.forward_op(image)

    @staticmethod
    def backward(ctx, v_bar):
        return ctx.model.adjoint_op(v_bar, dtype=ctx.dtype), None


def chi2_solve(model, vis_obs, weight=None, steps=200, x0=None, callback=None):
    """Steepest descent on chi^2 = sum w |D F C^-1 x - V|^2 with the exact line
    search of a quadratic; the gradient comes from autograd (the adjoint).
    Returns (x, history of chi^2)."""
    v_obs = K.on_device(vis_obs)
    w = None if weight is None else K.on_device(weight, torch.float32)
    x = (torch.zeros(model.image_shape, dtype=torch.float32, device=model.dev)
         if x0 is None else K.on_device(x0, torch.float32).clone())
    hist = []
    for it in range(steps):
        x.requires_grad_(True)
        r = model(x) - v_obs.to(torch.complex64)
        chi2 = (r.real ** 2 + r.imag ** 2)
        if w is not None:
            chi2 = chi2 * w
        chi2 = chi2.sum()
        (g,) = torch.autograd.grad(chi2, x)
        with torch.no_grad():
            ag = model.forward_op(g)
            num = float((g.double() ** 2).sum())
            den_t = (ag.real ** 2 + ag.imag ** 2)
            if w is not None:
                den_t = den_t * w
            den = 2.0 * float(den_t.double().sum())
            alpha = num / den if den > 0 else 0.0
            x = (x.detach() - alpha * g).contiguous()
        c2 = float(chi2.detach())
        hist.append(c2)
        if callback is not None:
            callback(it, c2)
    return x.detach(), hist
