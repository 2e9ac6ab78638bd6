"""sidon_b200 -- B200-native engine for the discretised autoconvolution ratio

    F(a) = 2 n max_k (a*a)_k / (sum_i a_i)^2,   a >= 0,

the objective of the memetic search in nanegate-dev/sidon-autocorrelation-bound.
The compute lives in ``libsidon_b200.so`` (hand-written sm_100a CUDA behind
the C ABI of ``include/sidon_b200.h``); this package is the host-side mirror
of the reference operator surface (``kernels``), the reference's vector and
certificate formats (``formats``) and the seeded workload generators
(``synth``).
"""
from . import _lib  # noqa: F401
from ._lib import SidonError, load  # noqa: F401

__all__ = ["SidonError", "load", "kernels", "formats", "synth"]


def __getattr__(name):
    if name in ("kernels", "formats", "synth"):
        import importlib
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
