"""ReturnDict: per-(time, pol, chan) deconvolution statistics with history.

Drop-in for src/astroviper/core/imaging/imaging_utils/return_dict.py.  Keys
are Key(time, pol, chan) named tuples; each holds a plain dict of fields.
Fields named in FIELD_ACCUM keep one entry per add() (a history list, used by
the major-cycle controller); every other field keeps its latest value.  The
two field sets are the reference's own (return_dict.py:22-40), since callers
and the controller depend on which fields carry history.
"""
from collections import OrderedDict, namedtuple

Key = namedtuple("Key", ["time", "pol", "chan"])

# fields with one entry per cycle (lists)
FIELD_ACCUM = frozenset({
    "peakres",
    "peakres_nomask",
    "iter_done",
    "masksum",
    "model_flux",
    "start_peakres",
    "start_peakres_nomask",
    "start_model_flux",
})

# fields that hold one value (parameters and PSF properties)
FIELD_SINGLE_VALUE = frozenset({
    "max_psf_sidelobe",
    "loop_gain",
    "niter",
    "threshold",
})


class ReturnDict:
    """Ordered mapping Key -> {field: value or history list}."""

    def __init__(self):
        self._data = OrderedDict()

    @property
    def data(self):
        return self._data

    @data.setter
    def data(self, value):
        self._data = value

    def add(self, value, time, pol, chan):
        """Record value (a dict of fields) for plane (time, pol, chan):
        history fields are appended, the others replaced
        (return_dict.py:54-104)."""
        key = Key(time, pol, chan)
        entry = self._data.get(key)
        fresh = entry is None
        if fresh:
            entry = {}
            self._data[key] = entry
        for field, v in value.items():
            if field not in FIELD_ACCUM:
                entry[field] = v
            elif fresh or field not in entry:
                entry[field] = [v]
            else:
                cur = entry[field]
                if not isinstance(cur, list):  # a value stored without history
                    cur = [cur]
                    entry[field] = cur
                cur.append(v)

    def sel(self, time=None, pol=None, chan=None):
        """The entries of the matching keys (None matches anything): one
        entry alone, a list of several, or None when nothing matches."""
        hits = [v for k, v in self._data.items()
                if (time is None or k.time == time) and (pol is None or k.pol == pol)
                and (chan is None or k.chan == chan)]
        if not hits:
            return None
        return hits[0] if len(hits) == 1 else hits

    def to_dict(self):
        return self._data

    def __repr__(self):
        return "\n".join(f"  {k}: {v}" for k, v in self._data.items())
