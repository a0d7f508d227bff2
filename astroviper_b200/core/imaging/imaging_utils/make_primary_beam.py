"""Primary-beam images of a single field on B200.

Drop-in for cube_single_field_primary_beam of
src/astroviper/core/imaging/imaging_utils/make_primary_beam.py (:11-122):
the same parameter validation and messages, telescope table and models.  The
beams come from this package's Airy-disk patterns (make_pb_symmetric,
av_airy_pattern), repeated over the time coordinates.  The result is a
SkyImage with a PRIMARY_BEAM variable (time, frequency, polarization, l, m)
in place of xradio's sky image, whose right ascension / declination
coordinates are not built.
"""
import numpy as np

from ..sky_image import make_sky_image
from .make_pb_symmetric import airy_disk_rorder, casa_airy_disk_rorder

# effective dish and blockage diameters in metres (make_primary_beam.py:70-78)
_TELESCOPES = {"ALMA": (10.7, 0.75), "ACA": (6.7, 0.75)}


def _validate_im_params(im_params):
    """make_primary_beam.py:11-34."""
    required_keys = ["cell_size", "image_size", "frequency_coords", "polarization",
                     "image_center", "phase_center", "time_coords"]
    for key in required_keys:
        if key not in im_params:
            raise ValueError(f"im_params must include '{key}' key")
        if key in ("cell_size", "image_size", "image_center", "phase_center"):
            if not (isinstance(im_params[key], tuple) and len(im_params[key]) == 2):
                raise ValueError(f"'{key}' must be a 2D tuple")
        if key in ("frequency_coords", "time_coords", "polarization"):
            if not isinstance(im_params[key], list):
                raise ValueError(f"'{key}' must be a list")


def cube_single_field_primary_beam(im_params, telescope, model="casa_airy_disk"):
    """make_primary_beam.py:37-122: the (time, frequency, polarization, l,
    m) primary beam of an ALMA (10.7 m dish) or ACA (6.7 m) antenna with a
    0.75 m blockage, ipower 2, from casa_airy_disk_rorder (model
    "casa_airy_disk", the default) or airy_disk_rorder (any other model),
    the same beam at every time coordinate.  ValueError for an unknown
    telescope or malformed im_params."""
    _validate_im_params(im_params)
    if telescope not in _TELESCOPES:
        raise ValueError(f"Unsupported telescope: {telescope}")
    dish_diameter, blockage_diameter = _TELESCOPES[telescope]
    pb_params = {"list_dish_diameters": [dish_diameter],
                 "list_blockage_diameters": [blockage_diameter], "ipower": 2}
    freq_chan = np.array(im_params["frequency_coords"])
    pol = im_params["polarization"]
    if model == "casa_airy_disk":
        pb = casa_airy_disk_rorder(freq_chan, pol, pb_params, im_params)
    else:
        pb = airy_disk_rorder(freq_chan, pol, pb_params, im_params)
    pb = pb[0]
    pb = np.repeat(pb[np.newaxis, :, :, :, :], len(im_params["time_coords"]), axis=0)
    image = make_sky_image(im_params["phase_center"], im_params["image_size"],
                           im_params["cell_size"], freq_chan, pol, im_params["time_coords"])
    image.attrs.update({"direction_reference": "fk5", "projection": "SIN"})
    image["PRIMARY_BEAM"] = pb
    return image
