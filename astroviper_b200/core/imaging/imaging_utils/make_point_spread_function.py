"""make_psf (reference: src/astroviper/core/imaging/imaging_utils/
make_point_spread_function.py:1-79) on B200.

The PSF planes are the visibilities' weights gridded and imaged by
grid2image_spheroid_ms4 with dopsf=True.  Two conventions of the reference are
kept because they change the result: the planes array is
(n_freq, n_pol, image_size[1], image_size[0]), the transpose of the image
size (:45), and the l increment is negated, pixelincr = [-cell0, cell1]
(:48).  The planes become the POINT_SPREAD_FUNCTION variable of an empty sky
image over the visibilities' frequencies, polarisations and first time: an
xradio image (fk5, SIN, sky coordinates) when xradio is installed, otherwise
this package's SkyImage with the same dims and coordinates.

For non-square images the reference's xarray assignment fails (the planes'
last two axes are (ny, nx) against l / m coordinates of (nx, ny) entries);
the SkyImage accepts them, so this drop-in returns the PSF there too.
"""
import numpy as np

from ..sky_image import DIMS, make_sky_image
from .standard_grid import grid2image_spheroid_ms4


def _psf_planes(vis, im_params, grid_params, precision):
    n_freq = len(vis.coords["frequency"].values)
    n_pol = len(vis.coords["polarization"].values)
    size_x, size_y = (int(n) for n in im_params["image_size"])
    cell_x, cell_y = im_params["cell_size"]
    planes = np.zeros((n_freq, n_pol, size_y, size_x), dtype=np.float64)
    grid2image_spheroid_ms4(vis=vis, resid_array=planes, pixelincr=np.array([-cell_x, cell_y]),
                            support=grid_params["support"], sampling=grid_params["sampling"],
                            dopsf=True, chan_mode=im_params["chan_mode"], precision=precision)
    return planes


def _empty_sky_image(vis, im_params):
    coords = dict(phase_center=im_params["phase_center"], image_size=im_params["image_size"],
                  cell_size=im_params["cell_size"],
                  frequency_coords=vis.coords["frequency"].values,
                  pol_coords=vis.coords["polarization"].values,
                  time_coords=vis.coords["time"].values[0])
    try:
        from xradio.image import make_empty_sky_image
    except ImportError:
        return make_sky_image(**coords)
    return make_empty_sky_image(direction_reference="fk5", projection="SIN", do_sky_coords=True,
                                **coords)


def make_psf(vis, im_params, grid_params, *, precision=None):
    """PSF sky image of the visibilities' sampling.

    vis: an MSv4 node (VISIBILITY / UVW / WEIGHT / FLAG, frequency,
    polarization and time coordinates); im_params: image_size (nx, ny),
    cell_size (rad, rad), phase_center, chan_mode; grid_params: sampling,
    support.  Returns an image dataset whose POINT_SPREAD_FUNCTION has dims
    (time, frequency, polarization, l, m) and one time.  Like
    grid2image_spheroid_ms4, it zeroes the WEIGHT of flagged and NaN-uvw
    samples in place.  precision: "fp64" for the FP64 gridder, else the
    FP32-input tiled path (as grid2image_spheroid_ms4)."""
    planes = _psf_planes(vis, im_params, grid_params, precision)
    image = _empty_sky_image(vis, im_params)
    image["POINT_SPREAD_FUNCTION"] = (DIMS, planes[np.newaxis])
    return image
