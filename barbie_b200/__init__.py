"""barbie_b200: B200-native BEAM redshift-space bispectrum estimator hot path.

The product is libbeam_gpu.so (C ABI, include/beam_gpu.h) and the `barbie`
host drop-in built beside it; ``barbie_b200.beam`` binds the library from
Python and ``barbie_b200.synth`` makes seeded input fields.
"""
from . import synth  # noqa: F401

__all__ = ["synth", "beam"]
