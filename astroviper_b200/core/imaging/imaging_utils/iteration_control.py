"""Major/minor-cycle iteration control.

Drop-in for src/astroviper/core/imaging/imaging_utils/iteration_control.py
(:1-1056): the stop codes, merge_return_dicts, the ReturnDict readers and
IterationController, with the reference's rules, defaults and messages
(callers and tests read the stop codes and the descriptions).  This is host
logic: it runs between device launches and reads a handful of numbers per
plane.  The convergence plots (:1057-1381) need matplotlib and are not part
of this module.
"""
from collections import namedtuple
from typing import Any, Dict, List, Optional, Tuple

from .return_dict import FIELD_ACCUM, FIELD_SINGLE_VALUE, Key, ReturnDict  # noqa: F401

HAVE_RETURNDICT = True

StopCode = namedtuple("StopCode", ["major", "minor"])

# major-cycle (global) stop codes, CASA's numbering
MAJOR_CONTINUE = 0
MAJOR_ITER_LIMIT = 1
MAJOR_THRESHOLD = 2
MAJOR_ZERO_MASK = 7
MAJOR_CYCLE_LIMIT = 9

# minor-cycle stop codes
MINOR_CONTINUE = 0
MINOR_ITER_LIMIT = 1
MINOR_THRESHOLD = 2
MINOR_DIVERGENCE = 4
MINOR_ZERO_MASK = 7

MAJOR_STOPCODE_DESCRIPTIONS = {
    MAJOR_CONTINUE: "Continue iterations",
    MAJOR_ITER_LIMIT: "Reached the iteration limit",
    MAJOR_THRESHOLD: "Reached global stopping threshold (within mask)",
    MAJOR_ZERO_MASK: "Zero mask",
    MAJOR_CYCLE_LIMIT: "Reached the major cycle limit (nmajor)",
}

MINOR_STOPCODE_DESCRIPTIONS = {
    MINOR_CONTINUE: "Continue minor cycle",
    MINOR_ITER_LIMIT: "Reached cycle iteration limit",
    MINOR_THRESHOLD: "Reached cycle threshold",
    MINOR_DIVERGENCE: "Possible divergence detected",
    MINOR_ZERO_MASK: "Zero mask",
}


# ------------------------------------------------------- ReturnDict readers --
def _validate_returndict_selection(return_dict, selected, time=None, pol=None, chan=None):
    """KeyError when an explicit time / pol / chan filter matched nothing
    (iteration_control.py:72-129); wildcard queries never raise."""
    filters = [(n, v) for n, v in (("time", time), ("pol", pol), ("chan", chan))
               if v is not None]
    if not filters:
        return
    if selected is not None and not (isinstance(selected, list) and not selected):
        return
    what = ", ".join(f"{n}={v}" for n, v in filters)
    keys = list(return_dict.data.keys())
    if not keys:
        avail = "ReturnDict is empty"
    elif len(keys) <= 10:
        avail = f"Available keys: {keys}"
    else:
        avail = f"Available keys (first 10 of {len(keys)}): {keys[:10]}"
    raise KeyError(f"No entries found for {what}. {avail}")


def _selected(return_dict, time, pol, chan):
    got = return_dict.sel(time=time, pol=pol, chan=chan)
    _validate_returndict_selection(return_dict, got, time, pol, chan)
    if got is None:
        return []
    return got if isinstance(got, list) else [got]


_EMPTY = object()


def _latest(value):
    """Last entry of a history list (_EMPTY for an empty one), or the value."""
    if isinstance(value, list):
        return value[-1] if value else _EMPTY
    return value


def merge_return_dicts(return_dicts: List[ReturnDict], merge_strategy: str = "update"):
    """One ReturnDict from several (iteration_control.py:132-244).  A key seen
    once keeps the very entry object of its source.  On a repeated key:
    "update" concatenates the history fields and replaces the others,
    "latest" keeps the last entry, "error" raises ValueError; any other
    strategy raises ValueError when a key repeats."""
    merged = ReturnDict()
    for rd in return_dicts or []:
        for key, value in rd.data.items():
            if key not in merged.data:
                merged.data[key] = value
                continue
            if merge_strategy == "latest":
                merged.data[key] = value
            elif merge_strategy == "error":
                raise ValueError(
                    f"Conflicting key found during merge: {key}. "
                    f"Use merge_strategy='latest' or 'update' to handle conflicts.")
            elif merge_strategy == "update":
                cur = merged.data[key]
                if not (isinstance(cur, dict) and isinstance(value, dict)):
                    merged.data[key] = value
                    continue
                for field, fv in value.items():
                    if field not in FIELD_ACCUM:
                        cur[field] = fv
                        continue
                    new = fv if isinstance(fv, list) else [fv]
                    if field in cur:
                        old = cur[field] if isinstance(cur[field], list) else [cur[field]]
                        cur[field] = old + new
                    else:
                        cur[field] = new
            else:
                raise ValueError(f"Unknown merge_strategy: {merge_strategy}")
    return merged


def get_peak_residual_from_returndict(return_dict, use_mask=True, time=None, pol=None,
                                      chan=None) -> float:
    """Largest |latest peakres| (or peakres_nomask) over the selected planes;
    with use_mask, planes whose latest masksum is 0 are left out
    (iteration_control.py:247-312)."""
    field = "peakres" if use_mask else "peakres_nomask"
    peak = 0.0
    for entry in _selected(return_dict, time, pol, chan):
        if entry is None or field not in entry:
            continue
        v = _latest(entry[field])
        if v is _EMPTY:
            continue
        if use_mask and "masksum" in entry:
            ms = _latest(entry["masksum"])
            if ms is _EMPTY or ms == 0:
                continue
        peak = max(peak, abs(v))
    return peak


def get_masksum_from_returndict(return_dict, time=None, pol=None, chan=None) -> float:
    """Sum of the latest masksum of the selected planes (:315-362)."""
    total = 0.0
    for entry in _selected(return_dict, time, pol, chan):
        if entry is None or "masksum" not in entry:
            continue
        v = _latest(entry["masksum"])
        if v is not _EMPTY:
            total += v
    return total


def get_iterations_done_from_returndict(return_dict, time=None, pol=None, chan=None) -> int:
    """Iterations over the whole history of the selected planes (:365-411)."""
    total = 0
    for entry in _selected(return_dict, time, pol, chan):
        if entry is None or "iter_done" not in entry:
            continue
        v = entry["iter_done"]
        total += sum(v) if isinstance(v, list) else v
    return total


def get_max_psf_sidelobe_from_returndict(return_dict, time=None, pol=None,
                                         chan=None) -> float:
    """Largest max_psf_sidelobe of the selected planes, 0.2 when none has
    one (:414-464)."""
    found = [entry["max_psf_sidelobe"] for entry in _selected(return_dict, time, pol, chan)
             if entry is not None and "max_psf_sidelobe" in entry]
    if not found:
        return 0.2
    best = 0.0
    for v in found:
        best = max(best, v)
    return best


def get_model_flux_from_returndict(return_dict, time=None, pol=None, chan=None) -> float:
    """Sum of the latest model_flux of the selected planes (:467-537)."""
    total = 0.0
    for entry in _selected(return_dict, time, pol, chan):
        if entry is None or "model_flux" not in entry:
            continue
        v = _latest(entry["model_flux"])
        if v is not _EMPTY:
            total += v
    return total


# -------------------------------------------------------------- controller --
class IterationController:
    """Global iteration budget and stopping rules of the major cycle
    (iteration_control.py:540-1055): niter and nmajor count down, each minor
    cycle gets min(cycleniter, niter) iterations and a cycle threshold of
    clamp(max_psf_sidelobe x cyclefactor, minpsffraction, maxpsffraction) x
    peak residual (at least threshold), and the loop stops on a zero mask,
    the iteration limit, the global threshold or the major-cycle limit, in
    that order."""

    def __init__(self, niter: int = 1000, nmajor: int = -1, threshold: float = 0.0,
                 gain: float = 0.1, cyclefactor: float = 1.0, minpsffraction: float = 0.05,
                 maxpsffraction: float = 0.8, cycleniter: int = -1, nsigma: float = 0.0):
        self._initial_niter = niter
        self.niter = niter
        self.nmajor = nmajor
        self.threshold = threshold
        self.nsigma = nsigma
        self.gain = gain
        self.cyclefactor = cyclefactor
        self.minpsffraction = minpsffraction
        self.maxpsffraction = maxpsffraction
        self.cycleniter = cycleniter
        self.major_done = 0
        self.total_iter_done = 0
        self.reset_stopcode()

    def calculate_cycle_controls(self, return_dict, time=None, pol=None,
                                 chan=None) -> Tuple[int, float]:
        """(iterations, threshold) of the next minor cycle (:653-727)."""
        sidelobe = get_max_psf_sidelobe_from_returndict(return_dict, time=time, pol=pol,
                                                        chan=chan)
        peak = get_peak_residual_from_returndict(return_dict, use_mask=True, time=time, pol=pol,
                                                 chan=chan)
        n = self.niter if self.cycleniter < 0 else min(self.cycleniter, self.niter)
        frac = min(max(sidelobe * self.cyclefactor, self.minpsffraction), self.maxpsffraction)
        return int(n), max(frac * peak, self.threshold)

    def check_convergence(self, return_dict, time=None, pol=None,
                          chan=None) -> Tuple[StopCode, str]:
        """Major-cycle stop code from the latest statistics (:730-831)."""
        peak = get_peak_residual_from_returndict(return_dict, use_mask=True, time=time, pol=pol,
                                                 chan=chan)
        masksum = get_masksum_from_returndict(return_dict, time=time, pol=pol, chan=chan)
        if masksum == 0:
            code = MAJOR_ZERO_MASK
        elif self.niter <= 0:
            code = MAJOR_ITER_LIMIT
        elif self.threshold > 0 and peak <= self.threshold:
            code = MAJOR_THRESHOLD
        elif self.nmajor != -1 and self.nmajor <= 0:
            code = MAJOR_CYCLE_LIMIT
        else:
            code = MAJOR_CONTINUE
        self.stopdescription = MAJOR_STOPCODE_DESCRIPTIONS[code]
        self.stopcode = StopCode(major=code, minor=MINOR_CONTINUE)
        return self.stopcode, self.stopdescription

    def update_counts(self, return_dict, time=None, pol=None, chan=None) -> None:
        """Charge a finished major cycle to the budgets (:834-899); nothing
        changes once a stop code is set."""
        if self.stopcode.major != MAJOR_CONTINUE or self.stopcode.minor != MINOR_CONTINUE:
            return
        done = get_iterations_done_from_returndict(return_dict, time=time, pol=pol, chan=chan)
        if self.nmajor != -1:
            self.nmajor = max(self.nmajor - 1, 0)
        self.niter = max(self.niter - done, 0)
        self.major_done += 1
        self.total_iter_done += done

    def update_parameters(self, niter=None, cycleniter=None, nmajor=None, threshold=None,
                          cyclefactor=None) -> Tuple[int, str]:
        """Validated interactive update (:902-999): (0, "") or (-1, reason).
        Parameters are applied in the order niter, cycleniter, nmajor,
        threshold, cyclefactor; a rejected one leaves the later ones as they
        were."""
        for name, value in (("niter", niter), ("cycleniter", cycleniter), ("nmajor", nmajor)):
            if value is None:
                continue
            try:
                v = int(value)
            except (ValueError, TypeError):
                return -1, f"{name} must be an integer"
            if v < -1:
                return -1, f"{name} must be >= -1"
            setattr(self, name, v)
        if threshold is not None:
            try:
                if isinstance(threshold, str):
                    t = self._parse_threshold_string(threshold)
                else:
                    t = float(threshold)
            except (ValueError, TypeError):
                return -1, "threshold must be a number, or a number with units (Jy/mJy/uJy)"
            if t < 0:
                return -1, "threshold must be >= 0"
            self.threshold = t
        if cyclefactor is not None:
            try:
                cf = float(cyclefactor)
            except (ValueError, TypeError):
                return -1, "cyclefactor must be a number"
            if cf <= 0:
                return -1, "cyclefactor must be > 0"
            self.cyclefactor = cf
        return 0, ""

    def _parse_threshold_string(self, threshold_str: str) -> float:
        """'12mJy' -> 0.012 (Jy, mJy, uJy)."""
        s = threshold_str.strip()
        for unit, scale in (("uJy", 1e6), ("mJy", 1e3)):
            if unit in s:
                return float(s.replace(unit, "")) / scale
        if "Jy" in s:
            return float(s.replace("Jy", ""))
        raise ValueError(f"Unknown units in threshold string: {threshold_str}")

    def reset(self) -> None:
        self.niter = self._initial_niter
        self.major_done = 0
        self.total_iter_done = 0
        self.reset_stopcode()

    def reset_stopcode(self) -> None:
        self.stopcode = StopCode(major=MAJOR_CONTINUE, minor=MINOR_CONTINUE)
        self.stopdescription = MAJOR_STOPCODE_DESCRIPTIONS[MAJOR_CONTINUE]

    def get_state(self) -> Dict[str, Any]:
        return {
            "niter": self.niter,
            "nmajor": self.nmajor,
            "initial_niter": self._initial_niter,
            "threshold": self.threshold,
            "nsigma": self.nsigma,
            "gain": self.gain,
            "cyclefactor": self.cyclefactor,
            "minpsffraction": self.minpsffraction,
            "maxpsffraction": self.maxpsffraction,
            "cycleniter": self.cycleniter,
            "major_done": self.major_done,
            "total_iter_done": self.total_iter_done,
            "stopcode": {"major": self.stopcode.major, "minor": self.stopcode.minor},
            "stopdescription": self.stopdescription,
        }
