"""Scripted scenarios for the imager's host logic (ReturnDict,
merge_return_dicts, the ReturnDict readers and IterationController).

make_golden_imager.py runs them against the reference's own classes and
stores every result in imager_control.json; tests/test_imager_host.py runs the
same scripts against astroviper_b200's classes and compares.  `api` is a
namespace with ReturnDict, IterationController, merge_return_dicts and the
get_*_from_returndict readers.
"""
import numpy as np

READERS = ("get_peak_residual_from_returndict", "get_masksum_from_returndict",
           "get_iterations_done_from_returndict", "get_max_psf_sidelobe_from_returndict",
           "get_model_flux_from_returndict")


def _plane(iter_done, peak, masksum=4096, sidelobe=0.25, flux=0.5, gain=0.1):
    return {"iter_done": iter_done, "peakres": peak, "peakres_nomask": peak,
            "masksum": masksum, "max_psf_sidelobe": sidelobe, "model_flux": flux,
            "start_peakres": 2 * peak, "start_model_flux": 0.0, "loop_gain": gain,
            "niter": 100, "threshold": 0.0, "stop_code": None}


def _first(peak, ny=64, nx=64, gain=0.1):
    return {"peakres": peak, "peakres_nomask": peak, "masksum": ny * nx, "iter_done": 0,
            "max_psf_sidelobe": 0.2, "loop_gain": gain}


SCENARIOS = {
    "threshold_stop": {
        "init": {"niter": 100, "nmajor": 3, "threshold": 0.05, "cyclefactor": 1.5},
        "ops": [
            ["new", "rd0"], ["add", "rd0", _first(1.0), 0, 0, 0],
            ["cycle_controls", "rd0"],
            ["new", "rd1"], ["add", "rd1", _plane(40, -0.4, sidelobe=0.3), 0, 0, 0],
            ["add", "rd1", _plane(35, 0.2, sidelobe=0.3), 0, 1, 0],
            ["update_counts", "rd1"], ["merge", "comb", ["comb", "rd1"], "update"],
            ["check", "rd1"], ["cycle_controls", "comb"], ["state"],
            ["new", "rd2"], ["add", "rd2", _plane(30, 0.04, flux=0.7), 0, 0, 0],
            ["add", "rd2", _plane(12, -0.03, flux=0.1), 0, 1, 0],
            ["update_counts", "rd2"], ["merge", "comb", ["comb", "rd2"], "update"],
            ["check", "rd2"], ["update_counts", "rd2"], ["state"], ["dump", "comb"],
            ["dump", "rd1"],
        ]},
    "iteration_limit": {
        "init": {"niter": 50},
        "ops": [
            ["new", "rd"], ["add", "rd", _plane(60, 0.5), 0, 0, 0], ["cycle_controls", "rd"],
            ["update_counts", "rd"], ["check", "rd"], ["state"], ["reset"], ["state"],
        ]},
    "major_limit": {
        "init": {"niter": 1000, "nmajor": 1, "threshold": 0.0},
        "ops": [
            ["new", "rd"], ["add", "rd", _plane(10, 0.5), 0, 0, 0], ["update_counts", "rd"],
            ["check", "rd"], ["state"], ["reset_stopcode"], ["state"],
        ]},
    "zero_mask": {
        "init": {"niter": 1000, "threshold": 1.0},
        "ops": [
            ["new", "rd"], ["add", "rd", _plane(10, 0.5, masksum=0), 0, 0, 0],
            ["check", "rd"], ["cycle_controls", "rd"], ["state"],
        ]},
    "cycle_fractions": {
        "init": {"niter": 500, "cycleniter": 10, "cyclefactor": 2.0, "minpsffraction": 0.1,
                 "maxpsffraction": 0.6, "threshold": 0.01},
        "ops": [
            ["new", "a"], ["add", "a", _plane(0, 2.0, sidelobe=0.01), 0, 0, 0],
            ["cycle_controls", "a"],
            ["new", "b"], ["add", "b", _plane(0, 2.0, sidelobe=0.9), 0, 0, 0],
            ["cycle_controls", "b"],
            ["new", "c"], ["add", "c", _plane(0, 0.001, sidelobe=0.2), 0, 0, 0],
            ["cycle_controls", "c"],
            ["new", "d"], ["cycle_controls", "d"],
            ["add", "a", _plane(5, 1.5, masksum=0), 0, 1, 0], ["cycle_controls", "a"],
            ["cycle_controls_sel", "a", None, 1, None],
        ]},
    "merges": {
        "init": {},
        "ops": [
            ["new", "x"], ["add", "x", _plane(1, 0.5), 0, 0, 0], ["add", "x", _plane(2, 0.4), 0, 0, 1],
            ["new", "y"], ["add", "y", _plane(3, 0.3), 0, 0, 0], ["add", "y", _plane(4, 0.2), 0, 1, 0],
            ["set_field", "y", [0, 0, 0], "iter_done", 7],
            ["merge", "u", ["x", "y"], "update"], ["dump", "u"], ["dump", "x"],
            ["merge", "l", ["x", "y"], "latest"], ["dump", "l"],
            ["merge", "e", ["x", "y"], "error"],
            ["merge", "q", ["x", "y"], "bogus"],
            ["new", "z"], ["add", "z", _plane(9, 0.1), 1, 0, 0],
            ["merge", "q2", ["x", "z"], "bogus"], ["dump", "q2"],
            ["merge", "empty", [], "update"], ["dump", "empty"],
        ]},
    "readers": {
        "init": {},
        "ops": [
            ["new", "r"], ["add", "r", _plane(10, -0.8, sidelobe=0.3, flux=1.5), 0, 0, 0],
            ["add", "r", _plane(20, 0.3, masksum=0, sidelobe=0.5, flux=0.25), 0, 1, 0],
            ["add", "r", _plane(5, 0.6, sidelobe=0.1, flux=2.0), 0, 0, 0],
            ["add", "r", {"peakres": 0.9}, 0, 0, 1],
            ["read", "get_peak_residual_from_returndict", "r", {}],
            ["read", "get_peak_residual_from_returndict", "r", {"use_mask": False}],
            ["read", "get_peak_residual_from_returndict", "r", {"pol": 1, "use_mask": False}],
            ["read", "get_peak_residual_from_returndict", "r", {"chan": 1}],
            ["read", "get_masksum_from_returndict", "r", {}],
            ["read", "get_iterations_done_from_returndict", "r", {}],
            ["read", "get_iterations_done_from_returndict", "r", {"pol": 0, "chan": 0}],
            ["read", "get_max_psf_sidelobe_from_returndict", "r", {}],
            ["read", "get_max_psf_sidelobe_from_returndict", "r", {"chan": 1}],
            ["read", "get_model_flux_from_returndict", "r", {}],
            ["read", "get_model_flux_from_returndict", "r", {"time": 3}],
            ["new", "n"],
            ["read", "get_peak_residual_from_returndict", "n", {"pol": 0}],
            ["read", "get_masksum_from_returndict", "n", {}],
            ["read", "get_max_psf_sidelobe_from_returndict", "n", {}],
            ["sel", "r", {"pol": 0}], ["sel", "r", {"pol": 1}], ["sel", "r", {"time": 9}],
            ["dump", "r"],
        ]},
    "keyerror_listing": {
        "init": {},
        "ops": [["new", "k"]] + [["add", "k", {"peakres": 0.1 * i, "iter_done": i}, 0, i, 0]
                                 for i in range(12)] + [
            ["read", "get_masksum_from_returndict", "k", {"chan": 5}],
            ["new", "k2"], ["add", "k2", {"peakres": 0.1}, 0, 0, 0],
            ["read", "get_masksum_from_returndict", "k2", {"time": 1, "pol": 2}],
        ]},
    "update_parameters": {
        "init": {"niter": 100, "threshold": 0.1, "cyclefactor": 1.0},
        "ops": [
            ["update_parameters", {"niter": 200, "cycleniter": 20, "nmajor": 4}], ["state"],
            ["update_parameters", {"niter": -2}], ["update_parameters", {"niter": "abc"}],
            ["update_parameters", {"nmajor": 2.7, "cycleniter": "x"}], ["state"],
            ["update_parameters", {"threshold": "10mJy"}], ["state"],
            ["update_parameters", {"threshold": " 5uJy "}], ["state"],
            ["update_parameters", {"threshold": "2Jy"}], ["state"],
            ["update_parameters", {"threshold": "1kHz"}],
            ["update_parameters", {"threshold": "-3mJy"}],
            ["update_parameters", {"threshold": -1.0}],
            ["update_parameters", {"threshold": None, "cyclefactor": 0}],
            ["update_parameters", {"cyclefactor": "x"}],
            ["update_parameters", {"cyclefactor": "2.5"}], ["state"],
        ]},
}


def _py(v):
    """JSON-friendly copy of a result."""
    if isinstance(v, dict):
        return {str(k): _py(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_py(x) for x in v]
    if isinstance(v, np.ndarray):
        return _py(v.tolist())
    if isinstance(v, np.generic):
        return v.item()
    return v


def _dump(rd):
    return [[list(k), _py(v)] for k, v in rd.data.items()]


def run(name, api):
    """Results of scenario `name` as a list of JSON-friendly values."""
    sc = SCENARIOS[name]
    ctl = api.IterationController(**sc["init"])
    rds = {"comb": api.ReturnDict()}
    out = []
    for op in sc["ops"]:
        kind = op[0]
        try:
            if kind == "new":
                rds[op[1]] = api.ReturnDict()
                res = None
            elif kind == "add":
                rds[op[1]].add(dict(op[2]), op[3], op[4], op[5])
                res = None
            elif kind == "set_field":
                key = [k for k in rds[op[1]].data if list(k) == op[2]][0]
                rds[op[1]].data[key][op[3]] = op[4]
                res = None
            elif kind == "cycle_controls":
                res = list(ctl.calculate_cycle_controls(rds[op[1]]))
            elif kind == "cycle_controls_sel":
                res = list(ctl.calculate_cycle_controls(rds[op[1]], time=op[2], pol=op[3],
                                                        chan=op[4]))
            elif kind == "update_counts":
                ctl.update_counts(rds[op[1]])
                res = None
            elif kind == "check":
                code, desc = ctl.check_convergence(rds[op[1]])
                res = [code.major, code.minor, desc]
            elif kind == "merge":
                rds[op[1]] = api.merge_return_dicts([rds[n] for n in op[2]], op[3])
                res = None
            elif kind == "dump":
                res = _dump(rds[op[1]])
            elif kind == "read":
                res = getattr(api, op[1])(rds[op[2]], **op[3])
            elif kind == "sel":
                got = rds[op[1]].sel(**op[2])
                res = got if got is None or isinstance(got, dict) else list(got)
            elif kind == "state":
                res = ctl.get_state()
            elif kind == "reset":
                ctl.reset()
                res = None
            elif kind == "reset_stopcode":
                ctl.reset_stopcode()
                res = None
            elif kind == "update_parameters":
                res = list(ctl.update_parameters(**op[1]))
            else:
                raise AssertionError(kind)
        except (KeyError, ValueError) as e:
            res = {"error": type(e).__name__, "msg": str(e).strip("'\"")}
        out.append(_py(res))
    return out


# ----------------------------------------------------------------------------
# Imaging-loop cases (imager.py:108-351): the inputs and parameters of the
# loops that make_golden_imager.py runs through the oracle's loop with the
# reference's own IterationController, merge_return_dicts and ReturnDict
# (imager_loop.json), and that tests/test_imager_gpu.py runs through
# astroviper_b200's run_imaging_loop.
LOOP_CASES = ("default", "linear4", "circular2", "initial_model_threshold")


def loop_inputs(n_time=16, n_chan=2, pol_scale=(1.0, 0.8)):
    """64 antennas, n_time steps x 2016 baselines x n_chan channels
    (1.3-1.5 GHz), point sources at half the small workload's offsets,
    correlations scaled by pol_scale; a flagged stretch and a NaN uvw row."""
    from astroviper_b200 import synthetic as S
    W = S.workload_small(n_time=n_time)
    uvw = W["uvw"].copy()
    freq = np.linspace(1.3e9, 1.5e9, n_chan)
    rng = np.random.default_rng(11)
    flux, dx, dy = W["sources"]
    l, m = S.source_lm(dx / 2, dy / 2, W["pixelincr"])
    vis = S.point_source_vis(uvw, freq, len(pol_scale), flux, l, m, 0.01, rng)
    # distinct correlations (e.g. YY fainter than XX), so Q (V) is not zero
    vis = vis * np.asarray(pol_scale)
    weight = np.ones(vis.shape)
    flag = np.zeros(vis.shape, dtype=bool)
    flag[3, 10:20] = True
    uvw[5, 7, 0] = np.nan
    return vis, uvw, weight, flag, freq, W["pixelincr"]


def loop_params(cell):
    return {"image_size": (128, 128), "cell_size": (abs(cell[0]), abs(cell[1])), "niter": 300,
            "nmajor": 4, "cyclefactor": 1.5, "gain": 0.1, "threshold": 0.0,
            "chan_mode": "cube"}


def loop_case(name):
    """(vis, uvw, weight, flag, freq, pols, params, initial_model) of a case."""
    if name == "default":
        vis, uvw, weight, flag, freq, cell = loop_inputs()
        return vis, uvw, weight, flag, freq, ["XX", "YY"], loop_params(cell), None
    scale = {"linear4": (1.0, 0.1, 0.05, 0.8), "circular2": (1.0, 0.7),
             "initial_model_threshold": (1.0, 0.8)}[name]
    pols = {"linear4": ["XX", "XY", "YX", "YY"], "circular2": ["RR", "LL"],
            "initial_model_threshold": ["XX", "YY"]}[name]
    vis, uvw, weight, flag, freq, cell = loop_inputs(n_time=12, pol_scale=scale)
    params = loop_params(cell)
    params.update(niter=120, nmajor=3)
    init = None
    if name == "circular2":
        params["corr_type"] = "circular"
    if name == "initial_model_threshold":
        params.update(threshold=0.05, nmajor=6, niter=2000)
        init = np.zeros((2, 2, 128, 128))
        init[0, 0, 60, 64] = 0.3
    return vis, uvw, weight, flag, freq, pols, params, init


def loop_decisions(out):
    """What a loop's controller decided (from the oracle loop's output dict):
    its final state, the cycle niter and threshold of every major cycle, and
    the merged ReturnDict (per plane, the per-cycle iterations, peaks and
    fluxes the controller read)."""
    ctl = out["controller"]
    return {"state": _py(ctl.get_state()),
            "cycles": [{"niter": int(c["niter"]), "threshold": float(c["threshold"])}
                       for c in out["cycles"]],
            "combined": _dump(out["combined"])}
