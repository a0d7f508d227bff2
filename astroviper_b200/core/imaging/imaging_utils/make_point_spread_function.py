"""make_psf (reference: src/astroviper/core/imaging/imaging_utils/
make_point_spread_function.py:1-79) on B200.

The PSF is grid2image_spheroid_ms4(..., dopsf=True) with pixel increment
[-cell0, cell1] into an (n_freq, n_pol, ny, nx) array, as the reference.  The
reference then wraps it into an xradio sky image; when xradio is importable
the same is done here, otherwise the PSF array is returned.
"""
import numpy as np

from .standard_grid import grid2image_spheroid_ms4


def make_psf(vis, im_params, grid_params, *, precision=None):
    freq_chan = vis.coords["frequency"].values
    nfreq = len(freq_chan)
    image_size = im_params["image_size"]
    cell_size = im_params["cell_size"]
    chan_mode = im_params["chan_mode"]
    sampling = grid_params["sampling"]
    support = grid_params["support"]
    pol = vis.coords["polarization"].values
    npol = len(pol)
    psf_data = np.zeros([nfreq, npol, image_size[1], image_size[0]], dtype=float)
    grid2image_spheroid_ms4(vis=vis, resid_array=psf_data,
                            pixelincr=np.array([-cell_size[0], cell_size[1]]), support=support,
                            sampling=sampling, dopsf=True, chan_mode=chan_mode,
                            precision=precision)
    try:
        from xradio.image import make_empty_sky_image
        import xarray as xr
    except Exception:
        return psf_data
    psf_xds = make_empty_sky_image(
        phase_center=im_params["phase_center"], image_size=image_size, cell_size=cell_size,
        frequency_coords=freq_chan, pol_coords=pol, time_coords=vis.coords["time"].values[0],
        direction_reference="fk5", projection="SIN", do_sky_coords=True)
    new_dims = tuple(d for d in psf_xds.dims if d != "beam_params_label")
    coords = psf_xds.drop_vars("beam_params_label", errors="ignore").coords
    psf_xds["POINT_SPREAD_FUNCTION"] = xr.DataArray(np.expand_dims(psf_data, axis=0),
                                                    dims=new_dims, coords=coords,
                                                    name="POINT_SPREAD_FUNCTION")
    return psf_xds
