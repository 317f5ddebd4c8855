"""trench_b200: B200-native (sm_100a) backend of the trench01 per-batch charging step.

Host side: Python/PyTorch (device memory, streams).  Compute: hand-written CUDA
kernels in libtrench_b200.so behind the C ABI of include/trench_b200.h.

    from trench_b200 import B200Tracer          # reference tracer interface
"""
from .params import Params, is_tapered  # noqa: F401

__all__ = ["Params", "is_tapered", "B200Tracer"]


def __getattr__(name):
    if name == "B200Tracer":
        from .tracer import B200Tracer
        return B200Tracer
    raise AttributeError(name)
