"""ctypes declarations of the C ABI in include/ppf_b200.h."""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "ppf_b200.h"
LIBPATH = PKG / "libppf_b200.so"

PPF_OK = 0
STATUS_NAMES = {
    0: "PPF_OK",
    1: "PPF_ERR_INVALID_ARGUMENT",
    2: "PPF_ERR_CUDA",
    3: "PPF_ERR_OUT_OF_MEMORY",
    4: "PPF_ERR_NO_VOTES",
    5: "PPF_ERR_TIMEOUT",
    6: "PPF_ERR_INTERNAL",
}


class ppf_stats(C.Structure):
    _fields_ = [
        ("n_votes", C.c_uint64),
        ("n_matched_pairs", C.c_uint64),
        ("max_vote_count", C.c_uint32),
        ("min_votecount", C.c_float),
        ("n_kept", C.c_uint64),
        ("max_idx", C.c_uint64),
        ("best_score", C.c_float),
        ("n_candidates", C.c_uint64),
        ("n_exact_bins", C.c_uint64),
        ("vote_ms", C.c_float),
        ("total_ms", C.c_float),
        ("gpu_launches", C.c_uint32),
        ("n_redo_items", C.c_uint32),
        ("cluster_path", C.c_uint32),
        ("vote_segment", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)

SIGNATURES = {
    "ppf_last_error": (C.c_char_p, []),
    "ppf_abi_version": (C.c_int, []),
    "ppf_context_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "ppf_context_destroy": (C.c_int, [_vp]),
    "ppf_context_synchronize": (C.c_int, [_vp]),
    "ppf_context_stream": (_vp, [_vp]),
    "ppf_context_kernel_launches": (C.c_uint64, [_vp]),
    "ppf_context_device": (C.c_int, [_vp]),
    "ppf_model_create": (
        C.c_int,
        [_vp, _vp, _vp, C.c_uint64, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)],
    ),
    "ppf_model_set_point_vote_weights": (C.c_int, [_vp, _vp, C.c_uint64]),
    "ppf_model_destroy": (C.c_int, [_vp]),
    "ppf_model_num_points": (C.c_uint64, [_vp]),
    "ppf_model_num_keys": (C.c_uint64, [_vp]),
    "ppf_model_num_chunks": (C.c_uint64, [_vp]),
    "ppf_scene_create": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_float, C.c_uint32, C.POINTER(_vp)]),
    "ppf_scene_destroy": (C.c_int, [_vp]),
    "ppf_model_lookup": (C.c_int, [_vp, _vp, _vp, C.POINTER(ppf_stats)]),
    "ppf_registration": (
        C.c_int,
        [
            _vp, C.c_uint64, C.POINTER(_vp), C.POINTER(_vp), _u64p,
            C.c_uint64, C.POINTER(_vp), C.POINTER(_vp), _u64p, _fp,
            C.c_uint32, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, _fp, _vp,
            C.POINTER(ppf_stats),
        ],
    ),
    "ppf_model_get_votes": (C.c_int, [_vp, _u64p, _u32p, C.c_uint64, _u64p]),
    "ppf_model_get_transformations": (C.c_int, [_vp, _fp, C.c_uint64, _u64p]),
    "ppf_model_get_cluster_state": (C.c_int, [_vp, _fp, _fp, _fp, C.c_uint64, _u64p]),
    "ppf_model_get_hash_array": (
        C.c_int,
        [_vp, _u32p, _u32p, _u32p, C.c_uint64, _u32p, C.c_uint64, _u64p, _u64p],
    ),
    "ppf_pair_keys": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_float, C.c_uint32, _vp]),
    "ppf_model_all_votes": (C.c_int, [_vp, _vp, _u64p, _u32p, C.c_uint64, _u64p]),
    "ppf_model_pair_vote_counts": (C.c_int, [_vp, _vp, _vp]),
    "ppf_lookup_batch": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp, _vp]),
    "ppf_cluster_poses": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_float, C.c_float, _vp, _vp, _vp]),
    "ppf_ply_read": (C.c_int, [C.c_char_p, _vp, _vp, C.c_uint64, _u64p]),
    "ppf_ply_write": (C.c_int, [C.c_char_p, _vp, _vp, C.c_uint64]),
    "ppf_cloud_extent": (C.c_int, [_vp, _vp, C.c_uint64, _vp, _vp]),
    "ppf_voxel_downsample": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_float, _vp, _vp, C.c_uint64, _u64p]),
    "ppf_server_create": (C.c_int, [C.c_int, C.c_uint64, _vp, C.c_uint64, C.c_uint32, C.c_uint32, _vp]),
    "ppf_server_submit": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_uint32, C.c_uint64, _vp, _vp]),
    "ppf_server_wait": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp]),
    "ppf_server_destroy": (C.c_int, [_vp]),
    "ppf_model_vote_cells_noalloc": (
        C.c_int,
        [_vp, _vp, _vp, C.c_uint64, C.c_uint32, C.c_float, _vp, _vp, C.c_uint64, _u64p, _u32p],
    ),
}


def header_symbols(path: Path = HEADER):
    """Function names declared in the public header."""
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ppf_[a-z0-9_]+)\s*\(", text)) - {"ppf_status"})


_lib = None


def load(path: Path | str | None = None):
    """Loads libppf_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else Path(os.environ.get("PPF_B200_LIB", LIBPATH))
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(the engine has no CPU fallback)"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib
