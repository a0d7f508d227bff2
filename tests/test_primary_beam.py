"""cube_single_field_primary_beam (make_primary_beam.py:11-122).

CPU: the parameter validation and the telescope table, with the reference's
messages.  GPU: the known answers of the reference's own
test_make_primary_beam.py (shapes, coordinates, values in [0, 1], the centre
above 0.9, mirror symmetry about the centre, the beam narrowing with
frequency), and the PRIMARY_BEAM plane against make_pb_symmetric's
casa_airy_disk_rorder / airy_disk_rorder, which the mosaic tests pin to the
reference's Numba beams.
"""
import numpy as np
import pytest

PC = (5.233697011339746, 0.7109380541842404)


def _mpb():
    from astroviper_b200.core.imaging.imaging_utils import make_primary_beam as M
    return M


def _params(**kw):
    p = {"cell_size": (0.0001, 0.0001), "image_size": (64, 64), "image_center": (32, 32),
         "frequency_coords": [1e11], "polarization": ["I"], "phase_center": PC,
         "time_coords": [0.0]}
    p.update(kw)
    return p


def test_validation_follows_the_reference():
    M = _mpb()
    for key in ("cell_size", "image_size", "frequency_coords", "polarization", "image_center",
                "phase_center", "time_coords"):
        p = _params()
        del p[key]
        with pytest.raises(ValueError, match=f"im_params must include '{key}' key"):
            M.cube_single_field_primary_beam(p, "ALMA")
    for key in ("cell_size", "image_size", "image_center", "phase_center"):
        with pytest.raises(ValueError, match=f"'{key}' must be a 2D tuple"):
            M.cube_single_field_primary_beam(_params(**{key: [1, 2]}), "ALMA")
        with pytest.raises(ValueError, match=f"'{key}' must be a 2D tuple"):
            M.cube_single_field_primary_beam(_params(**{key: (1, 2, 3)}), "ALMA")
    for key in ("frequency_coords", "time_coords", "polarization"):
        with pytest.raises(ValueError, match=f"'{key}' must be a list"):
            M.cube_single_field_primary_beam(_params(**{key: (1.0,)}), "ALMA")
    with pytest.raises(ValueError, match="Unsupported telescope"):
        M.cube_single_field_primary_beam(_params(), telescope="VLA")
    # the parameters are checked before the telescope, as in the reference
    with pytest.raises(ValueError, match="'image_size' must be a 2D tuple"):
        M.cube_single_field_primary_beam(_params(image_size=[64, 64]), telescope="VLA")


@pytest.mark.gpu
def test_reference_unit_tests_known_answers():
    M = _mpb()
    pb = M.cube_single_field_primary_beam(
        _params(cell_size=(0.00001, 0.00001), image_size=(128, 128), image_center=(64, 64),
                frequency_coords=[1e11, 1.1e11]), telescope="ALMA")
    assert "PRIMARY_BEAM" in pb.data_vars
    assert pb["PRIMARY_BEAM"].dims == ("time", "frequency", "polarization", "l", "m")
    d = pb["PRIMARY_BEAM"].values
    assert d.shape == (1, 2, 1, 128, 128)
    assert pb.sizes["frequency"] == 2 and pb.sizes["polarization"] == 1
    assert np.all(d >= 0.0) and np.all(d <= 1.0) and d[0, 0, 0, 64, 64] > 0.9
    for tel, model, shape, kw in (
            ("ACA", "casa_airy_disk", (1, 2, 1, 64, 64),
             dict(cell_size=(-0.0001, 0.0001), frequency_coords=[1e11, 1.1e11])),
            ("ALMA", "airy_disk", (1, 1, 1, 64, 64), dict(cell_size=(-0.0001, 0.0001))),
            ("ALMA", "casa_airy_disk", (1, 1, 4, 64, 64),
             dict(cell_size=(-0.00001, 0.00001), polarization=["I", "Q", "U", "V"],
                  phase_center=(0.0, 0.0)))):
        d = M.cube_single_field_primary_beam(_params(**kw), telescope=tel, model=model)[
            "PRIMARY_BEAM"].values
        assert d.shape == shape and np.all(d >= 0.0) and np.all(d <= 1.0), (tel, model)
    freqs = [1.00e11, 1.01e11, 1.02e11, 1.03e11]
    pb = M.cube_single_field_primary_beam(
        _params(cell_size=(-0.00001, 0.00001), frequency_coords=freqs), telescope="ALMA")
    d = pb["PRIMARY_BEAM"].values
    assert d.shape == (1, 4, 1, 64, 64)
    assert np.array_equal(pb.coords["frequency"].values, np.array(freqs))
    assert d[0, 0, 0, 10, 32] > d[0, 3, 0, 10, 32]
    for size in [(32, 32), (64, 64), (128, 256)]:
        d = M.cube_single_field_primary_beam(
            _params(image_size=size, image_center=(size[0] // 2, size[1] // 2),
                    phase_center=(0.0, 0.0)), telescope="ALMA")["PRIMARY_BEAM"].values
        assert d.shape == (1, 1, 1, size[0], size[1])
    for cell in [(0.0001, 0.0001), (0.0005, 0.0005), (0.001, 0.001)]:
        d = M.cube_single_field_primary_beam(
            _params(cell_size=cell, polarization=[0], phase_center=(0.0, 0.0)),
            telescope="ALMA")["PRIMARY_BEAM"].values
        assert np.all(d >= 0.0) and np.all(d <= 1.0)
    d = M.cube_single_field_primary_beam(
        _params(image_size=(129, 129), image_center=(64, 64)), telescope="ALMA")[
        "PRIMARY_BEAM"].values[0, 0, 0]
    np.testing.assert_array_almost_equal(d[64, :64], d[64, 65:][::-1], decimal=5)
    np.testing.assert_array_almost_equal(d[:64, 64], d[65:, 64][::-1], decimal=5)
    pb = M.cube_single_field_primary_beam(
        _params(frequency_coords=[1.0e11, 1.05e11, 1.10e11], time_coords=[0.0, 100.0],
                polarization=["I", "Q", "U", "V"]), telescope="ALMA")
    assert np.array_equal(pb.coords["frequency"].values, [1.0e11, 1.05e11, 1.10e11])
    assert np.array_equal(pb.coords["time"].values, [0.0, 100.0])
    assert np.array_equal(pb.coords["polarization"].values, ["I", "Q", "U", "V"])
    d = pb["PRIMARY_BEAM"].values
    assert d.shape == (2, 3, 4, 64, 64) and np.array_equal(d[0], d[1])


@pytest.mark.gpu
def test_beam_is_the_airy_pattern():
    from astroviper_b200.core.imaging.imaging_utils import make_pb_symmetric as PB
    M = _mpb()
    p = _params(frequency_coords=[1e11, 2e11], polarization=["XX", "YY"])
    for model, fn, block in (("casa_airy_disk", PB.casa_airy_disk_rorder, 0.75),
                             ("airy_disk", PB.airy_disk_rorder, 0.75)):
        for tel, dish in (("ALMA", 10.7), ("ACA", 6.7)):
            got = M.cube_single_field_primary_beam(p, tel, model)["PRIMARY_BEAM"].values
            want = fn(np.array(p["frequency_coords"]), p["polarization"],
                      {"list_dish_diameters": [dish], "list_blockage_diameters": [block],
                       "ipower": 2}, p)[0]
            assert np.array_equal(got[0], want), (model, tel)
