"""PSWF gridding kernel (reference: src/astroviper/core/imaging/imaging_utils/
gcf_prolate_spheroidal.py).  The rational approximation is evaluated by the
av_pswf* kernels in FP64."""
import numpy as np

from .... import _host as H
from .... import _kernels as K


def create_prolate_spheroidal_kernel(oversampling, support, n_uv):
    """Returns (kernel, kernel_image): the (n_os, n_os, support, support)
    oversampled kernel (gcf_prolate_spheroidal.py:28-67) and the grid
    correction image (:73-79)."""
    kernel = K.pswf_kernel4d(int(oversampling), int(support)).cpu().numpy()
    kernel_image = K.corr_term(int(n_uv[0]), int(n_uv[1])).cpu().numpy()
    return kernel, kernel_image


def create_prolate_spheroidal_kernel_1D(oversampling, support):
    """The 1-D half kernel of oversampling*(support//2+1) samples
    (gcf_prolate_spheroidal.py:87-99)."""
    return K.pswf_table(int(oversampling), int(support)).cpu().numpy()


def prolate_spheroidal_function(u):
    """(grdsf, (1-u^2) grdsf) of gcf_prolate_spheroidal.py:102-158."""
    u = np.asarray(u, dtype=np.float64)
    g, k = K.pswf(u.ravel())
    return g.cpu().numpy().reshape(u.shape), k.cpu().numpy().reshape(u.shape)


def coordinates(npixel: int):
    """1D array which spans [-.5,.5[ with 0 at position npixel/2 (:161)."""
    return (np.arange(npixel) - npixel // 2) / npixel


def coordinates2(npixel: int):
    """Two dimensional grids of coordinates (:166)."""
    return (np.mgrid[0:npixel, 0:npixel] - npixel // 2) / npixel
