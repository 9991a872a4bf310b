"""B200-native point pair feature (PPF) registration engine.

The registration path of nicolasavru/ppf-registration-spatial-hashing
(PPF compute + quantise + hash -> sorted hash array -> voting -> threshold ->
poses -> spatial-hash pose clustering -> best pose) as hand-written sm_100a
CUDA behind the C ABI in include/ppf_b200.h.  This package holds the kernels
(csrc/), their build (build.py), the ctypes binding (_capi.py), the
reference-shaped Python API (api.py) and the seeded synthetic workloads
(synthetic.py).
"""
from . import synthetic  # noqa: F401
from ._capi import header_symbols, load  # noqa: F401
from .api import (  # noqa: F401
    Context,
    Model,
    PPFError,
    Scene,
    Server,
    cloud_extent,
    cluster_poses,
    ht_dist,
    load_ply,
    load_xf,
    save_ply,
    validate,
    model_d_dist,
    preprocess,
    voxel_downsample,
    default_context,
    lookup_batch,
    pair_keys,
    ppf_registration,
)
