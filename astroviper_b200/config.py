"""Package-wide settings."""


class _Config:
    def __init__(self):
        # "fp32": tiled FP32 gridder / degridder (FP64 index math and weights
        # sums); "fp64": plain FP64 kernels in the reference's arithmetic.
        self.precision = "fp32"


config = _Config()


def resolve_precision(precision):
    p = config.precision if precision is None else precision
    if p not in ("fp32", "fp64"):
        raise ValueError(f"precision must be 'fp32' or 'fp64', got {p!r}")
    return p
