"""Python face of the engine, mirroring the reference's C++ API.

``Model``, ``Scene`` and ``ppf_registration`` keep the reference's names,
argument order and meaning (include/model.h:17-35, include/scene.h:15-16,
include/ppf.h:9-15); results come back as numpy arrays.  Every call goes
through libppf_b200.so; there is no CPU fallback.

A cloud is anything with ``points`` and ``normals`` attributes, or a
``(points, normals)`` pair, each ``(n, 3)`` float32: numpy arrays (host) or
contiguous CUDA tensors (device, passed by pointer).
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _capi


class PPFError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_capi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _lib():
    return _capi.load()


def _check(status: int):
    if status != _capi.PPF_OK:
        msg = _lib().ppf_last_error()
        raise PPFError(status, msg.decode() if msg else "")


def _split_cloud(cloud):
    if isinstance(cloud, (tuple, list)) and len(cloud) == 2:
        return cloud[0], cloud[1]
    return cloud.points, cloud.normals


class _Buf:
    """Pointer + length of a (n, 3) float32 array, host or device."""

    def __init__(self, a, name):
        if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
            if a.dtype.__repr__() != "torch.float32" or not a.is_contiguous() or a.dim() != 2 or a.shape[1] != 3:
                raise ValueError(f"{name}: expected a contiguous (n, 3) float32 tensor")
            self.keep = a
            self.ptr = C.c_void_p(a.data_ptr())
            self.n = int(a.shape[0])
        else:
            arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
            if arr.ndim != 2 or arr.shape[1] != 3:
                raise ValueError(f"{name}: expected an (n, 3) array")
            self.keep = arr
            self.ptr = C.c_void_p(arr.ctypes.data)
            self.n = int(arr.shape[0])


class Context:
    """A device, a stream and a workspace (device index as devUse, src/cuda/ppf.cu:37-49)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(_lib().ppf_context_create(int(device), C.byref(h)))
        self.handle = h

    def synchronize(self):
        _check(_lib().ppf_context_synchronize(self.handle))

    @property
    def kernel_launches(self) -> int:
        return int(_lib().ppf_context_kernel_launches(self.handle))

    @property
    def stream(self) -> int:
        return int(_lib().ppf_context_stream(self.handle) or 0)

    @property
    def device(self) -> int:
        """The CUDA device index the context runs on."""
        return int(_lib().ppf_context_device(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            _lib().ppf_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Scene:
    """Scene(cloud, d_dist, ref_point_downsample_factor=1) (include/scene.h:15-16)."""

    def __init__(self, cloud, d_dist: float, ref_point_downsample_factor: int = 1, context=None):
        self.ctx = context or default_context()
        p, q = _split_cloud(cloud)
        bp, bq = _Buf(p, "points"), _Buf(q, "normals")
        if bp.n != bq.n:
            raise ValueError("points and normals differ in length")
        h = C.c_void_p()
        _check(
            _lib().ppf_scene_create(
                self.ctx.handle, bp.ptr, bq.ptr, bp.n, float(d_dist), int(ref_point_downsample_factor), C.byref(h)
            )
        )
        self.handle = h
        self.n = bp.n
        self.d_dist = float(d_dist)
        self.ref_point_downsample_factor = int(ref_point_downsample_factor)

    def numPoints(self) -> int:
        return self.n

    def close(self):
        if getattr(self, "handle", None):
            _lib().ppf_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Model:
    """Model(cloud, d_dist, vote_count_threshold, cpu_clustering, use_l1_norm,
    use_averaged_clusters) (include/model.h:17-19)."""

    def __init__(self, cloud, d_dist: float, vote_count_threshold: float = 0.4, cpu_clustering: bool = False,
                 use_l1_norm: bool = False, use_averaged_clusters: bool = False, context=None):
        self.ctx = context or default_context()
        p, q = _split_cloud(cloud)
        bp, bq = _Buf(p, "points"), _Buf(q, "normals")
        if bp.n != bq.n:
            raise ValueError("points and normals differ in length")
        h = C.c_void_p()
        _check(
            _lib().ppf_model_create(
                self.ctx.handle, bp.ptr, bq.ptr, bp.n, float(d_dist), float(vote_count_threshold),
                int(bool(cpu_clustering)), int(bool(use_l1_norm)), int(bool(use_averaged_clusters)), C.byref(h),
            )
        )
        self.handle = h
        self.n = bp.n
        self.d_dist = float(d_dist)
        self.vote_count_threshold = float(vote_count_threshold)
        self.cpu_clustering = bool(cpu_clustering)
        self.use_l1_norm = bool(use_l1_norm)
        self.use_averaged_clusters = bool(use_averaged_clusters)
        self.stats = None
        self.pose = None

    # Model::SetModelPointVoteWeights (src/cuda/model.cu:91-93)
    def SetModelPointVoteWeights(self, weights):
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float32))
        _check(_lib().ppf_model_set_point_vote_weights(self.handle, C.c_void_p(w.ctypes.data), w.size))

    # Model::ppf_lookup (src/cuda/model.cu:269-306) + pose extraction (src/cuda/ppf.cu:74-93)
    def ppf_lookup(self, scene: Scene, raise_on_no_votes: bool = True) -> np.ndarray:
        pose = np.zeros(16, np.float32)
        st = _capi.ppf_stats()
        status = _lib().ppf_model_lookup(self.handle, scene.handle, C.c_void_p(pose.ctypes.data), C.byref(st))
        self.stats = st.as_dict()
        self.pose = pose.reshape(4, 4)
        if status == 4 and not raise_on_no_votes:
            return self.pose
        _check(status)
        return self.pose

    @property
    def num_chunks(self) -> int:
        """Chunks of model reference points per scene reference point in the vote pass."""
        return int(_lib().ppf_model_num_chunks(self.handle))

    @property
    def max_idx(self) -> int:
        return int(self.stats["max_idx"]) if self.stats else 0

    def _count(self, fn, *args):
        n = C.c_uint64()
        _check(fn(self.handle, *args, 0, C.byref(n)))
        return int(n.value)

    def get_votes(self):
        """(codes uint64, counts uint32) of the kept votes in the reference's order."""
        L = _lib()
        n = self._count(L.ppf_model_get_votes, None, None)
        codes = np.zeros(n, np.uint64)
        counts = np.zeros(n, np.uint32)
        m = C.c_uint64()
        _check(L.ppf_model_get_votes(self.handle, codes.ctypes.data_as(_capi._u64p),
                                     counts.ctypes.data_as(_capi._u32p), n, C.byref(m)))
        return codes, counts

    @property
    def votes(self):
        return self.get_votes()[0]

    @property
    def voteCounts(self):
        return self.get_votes()[1]

    def getTransformations(self) -> np.ndarray:
        L = _lib()
        n = self._count(L.ppf_model_get_transformations, None)
        T = np.zeros((n, 16), np.float32)
        m = C.c_uint64()
        _check(L.ppf_model_get_transformations(self.handle, T.ctypes.data_as(_capi._fp), n, C.byref(m)))
        return T

    def get_cluster_state(self):
        """(transformation_trans (U,3), transformation_rots (U,4), vote_counts_out (U,))."""
        L = _lib()
        n = self._count(L.ppf_model_get_cluster_state, None, None, None)
        t = np.zeros((n, 3), np.float32)
        q = np.zeros((n, 4), np.float32)
        s = np.zeros(n, np.float32)
        m = C.c_uint64()
        _check(L.ppf_model_get_cluster_state(self.handle, t.ctypes.data_as(_capi._fp), q.ctypes.data_as(_capi._fp),
                                             s.ctypes.data_as(_capi._fp), n, C.byref(m)))
        return t, q, s

    def hash_array(self):
        """The model's ParallelHashArray: dict(keys, counts, first, map)."""
        L = _lib()
        K, P = C.c_uint64(), C.c_uint64()
        _check(L.ppf_model_get_hash_array(self.handle, None, None, None, 0, None, 0, C.byref(K), C.byref(P)))
        k = np.zeros(K.value, np.uint32)
        c = np.zeros(K.value, np.uint32)
        f = np.zeros(K.value, np.uint32)
        mp = np.zeros(P.value, np.uint32)
        _check(L.ppf_model_get_hash_array(
            self.handle, k.ctypes.data_as(_capi._u32p), c.ctypes.data_as(_capi._u32p), f.ctypes.data_as(_capi._u32p),
            K.value, mp.ctypes.data_as(_capi._u32p), P.value, C.byref(K), C.byref(P)))
        return {"keys": k, "counts": c, "first": f, "map": mp}

    def all_votes(self, scene: Scene):
        """Every nonzero vote cell (code asc) with its count, before the threshold."""
        L = _lib()
        n = C.c_uint64()
        _check(L.ppf_model_all_votes(self.handle, scene.handle, None, None, 0, C.byref(n)))
        codes = np.zeros(n.value, np.uint64)
        counts = np.zeros(n.value, np.uint32)
        _check(L.ppf_model_all_votes(self.handle, scene.handle, codes.ctypes.data_as(_capi._u64p),
                                     counts.ctypes.data_as(_capi._u32p), n.value, C.byref(n)))
        return codes, counts

    def vote_cells_noalloc(self, scene_xyz, scene_nxyz, ref_point_df: int, vote_floor: float,
                           codes_out, counts_out):
        """Allocation-free vote pass (ppf_model_vote_cells_noalloc; no reference counterpart).

        For callers that may not allocate device memory while they run.  All
        four arrays are the caller's CUDA tensors and are passed by pointer
        with no copy or conversion: scene_xyz / scene_nxyz contiguous (n, 3)
        float32, codes_out int64 / uint64 and counts_out int32 / uint32 of equal
        length.  Writes the vote cells to the front of the outputs in no
        particular order and returns (n_cells, max_count).  An output that is
        too small raises PPFError (PPF_ERR_OUT_OF_MEMORY) whose ``needed``
        attribute is the number of cells the call needed.  Calls on one device
        share the library's static scratch array and must not overlap.
        """
        for name, t, dt in (("scene_xyz", scene_xyz, ("torch.float32",)),
                            ("scene_nxyz", scene_nxyz, ("torch.float32",)),
                            ("codes_out", codes_out, ("torch.int64", "torch.uint64")),
                            ("counts_out", counts_out, ("torch.int32", "torch.uint32"))):
            if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous() and repr(t.dtype) in dt):
                raise ValueError(f"{name}: expected a contiguous CUDA tensor of {' or '.join(dt)}")
            if t.device.index != self.ctx.device:
                raise ValueError(f"{name}: tensor on cuda:{t.device.index}, model's context on "
                                 f"cuda:{self.ctx.device}")
        if scene_xyz.shape != scene_nxyz.shape or scene_xyz.dim() != 2 or scene_xyz.shape[1] != 3:
            raise ValueError("scene_xyz / scene_nxyz: expected two (n, 3) tensors")
        if codes_out.numel() != counts_out.numel():
            raise ValueError("codes_out and counts_out must have the same length")
        n = C.c_uint64()
        mx = C.c_uint32()
        status = _lib().ppf_model_vote_cells_noalloc(
            self.handle, C.c_void_p(scene_xyz.data_ptr()), C.c_void_p(scene_nxyz.data_ptr()),
            int(scene_xyz.shape[0]), int(ref_point_df), float(vote_floor),
            C.c_void_p(codes_out.data_ptr()), C.c_void_p(counts_out.data_ptr()),
            int(codes_out.numel()), C.byref(n), C.byref(mx))
        if status != _capi.PPF_OK:
            msg = _lib().ppf_last_error()
            err = PPFError(status, msg.decode() if msg else "")
            err.needed = int(n.value)
            raise err
        return int(n.value), int(mx.value)

    def pair_vote_counts(self, scene: Scene) -> np.ndarray:
        out = np.zeros(scene.n * scene.n, np.uint64)
        _check(_lib().ppf_model_pair_vote_counts(self.handle, scene.handle, C.c_void_p(out.ctypes.data)))
        return out.reshape(scene.n, scene.n)

    def close(self):
        if getattr(self, "handle", None):
            _lib().ppf_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pair_keys(cloud, d_dist: float, ref_point_downsample_factor: int = 1, context=None) -> np.ndarray:
    """Keys of all ordered pairs, (n, n) uint32 (Scene::initPPFs + ppf_hash_kernel)."""
    ctx = context or default_context()
    p, q = _split_cloud(cloud)
    bp, bq = _Buf(p, "points"), _Buf(q, "normals")
    out = np.zeros(bp.n * bp.n, np.uint32)
    _check(_lib().ppf_pair_keys(ctx.handle, bp.ptr, bq.ptr, bp.n, float(d_dist), int(ref_point_downsample_factor),
                                C.c_void_p(out.ctypes.data)))
    return out.reshape(bp.n, bp.n)


def cluster_poses(transforms, votes, trans_thresh: float, rot_thresh: float, context=None):
    """clusterPoses (src/transformation_clustering.cpp:62-123) on the device:
    (poses (k, 4, 4), vote totals (k,)) of the k <= 3 best greedy clusters."""
    ctx = context or default_context()
    T = np.ascontiguousarray(np.asarray(transforms, np.float32).reshape(-1, 16))
    v = np.ascontiguousarray(np.asarray(votes, np.uint32))
    if len(T) != len(v):
        raise ValueError("one vote count per pose is required")
    out = np.zeros((3, 16), np.float32)
    ov = np.zeros(3, np.uint32)
    nc = C.c_uint32()
    _check(_lib().ppf_cluster_poses(ctx.handle, C.c_void_p(T.ctypes.data), C.c_void_p(v.ctypes.data), len(v),
                                    float(trans_thresh), float(rot_thresh), C.c_void_p(out.ctypes.data),
                                    C.c_void_p(ov.ctypes.data), C.byref(nc)))
    return out[: nc.value].reshape(-1, 4, 4), ov[: nc.value]


def load_ply(path):
    """pcl::io::loadPLYFile<PointNormal> as the alignment driver uses it
    (src/alignment.cpp:212,241): (points, normals) float32 (n, 3)."""
    L = _lib()
    p = str(path).encode()
    n = C.c_uint64()
    _check(L.ppf_ply_read(p, None, None, 0, C.byref(n)))
    xyz = np.zeros((max(n.value, 1), 3), np.float32)
    nrm = np.zeros((max(n.value, 1), 3), np.float32)
    _check(L.ppf_ply_read(p, C.c_void_p(xyz.ctypes.data), C.c_void_p(nrm.ctypes.data), n.value, C.byref(n)))
    return xyz[: n.value], nrm[: n.value]


def save_ply(path, cloud):
    """Writes a binary little-endian PLY of float x y z nx ny nz."""
    p, q = _split_cloud(cloud)
    p = np.ascontiguousarray(np.asarray(p, np.float32))
    q = np.ascontiguousarray(np.asarray(q, np.float32))
    _check(_lib().ppf_ply_write(str(path).encode(), C.c_void_p(p.ctypes.data), C.c_void_p(q.ctypes.data), len(p)))


def load_xf(path) -> np.ndarray:
    """A ground-truth pose file (.xf) as the driver reads it into an
    Eigen::Matrix4f (src/alignment.cpp:306-307): 16 numbers, row-major."""
    vals = np.array(open(path).read().split(), dtype=np.float64)
    if vals.size < 16:
        raise ValueError(f"{path}: expected 16 numbers")
    return vals[:16].reshape(4, 4).astype(np.float32)


def _quat(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix (largest-component branch)."""
    R = np.asarray(R, np.float64)
    t = np.trace(R)
    if t > 0:
        s = np.sqrt(t + 1.0) * 2
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k]) * 2
        q = [0.0, 0.0, 0.0, 0.0]
        q[0] = (R[k, j] - R[j, k]) / s
        q[1 + i] = 0.25 * s
        q[1 + j] = (R[j, i] + R[i, j]) / s
        q[1 + k] = (R[k, i] + R[i, k]) / s
    q = np.array(q)
    return q / np.linalg.norm(q)


def ht_dist(a, b):
    """ht_dist (src/cuda/linalg.cu:9-20): (|t_a - t_b|, rotation angle of
    R_a^-1 R_b in [0, pi]) of two 4x4 poses.  The reference takes the angle
    from Eigen's AngleAxis of the quaternion product, 2 atan2(|v|, |w|);
    Eigen is not installed here, so the same quantity is restated in float64
    (the translation distance is taken in float32, as the reference does)."""
    a = np.asarray(a, np.float32).reshape(4, 4)
    b = np.asarray(b, np.float32).reshape(4, 4)
    d = a[:3, 3] - b[:3, 3]
    td = float(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))
    qa, qb = _quat(a[:3, :3]), _quat(b[:3, :3])
    w = qa[0] * qb[0] + np.dot(qa[1:], qb[1:])  # (qa^-1 qb).w
    v = qa[0] * qb[1:] - qb[0] * qa[1:] - np.cross(qa[1:], qb[1:])
    return td, float(abs(2.0 * np.arctan2(np.linalg.norm(v), abs(w))))


def validate(pose, truth, model_diameter: float, translation_threshold: float = 0.1,
             rotation_threshold_deg: float = 12.0):
    """The driver's validation (src/alignment.cpp:300-335): a pose matches when
    its translation is within translation_threshold * model_diameter of the
    ground truth and its rotation within rotation_threshold_deg.  Returns
    (match, (translation distance, rotation angle))."""
    td, rd = ht_dist(pose, truth)
    ok = td < translation_threshold * model_diameter and rd < np.deg2rad(rotation_threshold_deg)
    return bool(ok), (td, rd)


def cloud_extent(cloud, context=None):
    """pcl::getMinMax3D of a cloud's points (finite ones): (min[3], max[3])."""
    ctx = context or default_context()
    p, _ = _split_cloud(cloud) if isinstance(cloud, (tuple, list)) or hasattr(cloud, "points") else (cloud, None)
    bp = _Buf(p, "points")
    lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
    _check(_lib().ppf_cloud_extent(ctx.handle, bp.ptr, bp.n, C.c_void_p(lo.ctypes.data), C.c_void_p(hi.ctypes.data)))
    return lo, hi


def model_d_dist(cloud, tau_d: float, context=None) -> float:
    """The alignment driver's d_dist of a model: tau_d times its largest
    axis-aligned extent, in float32 (src/alignment.cpp:246-253)."""
    lo, hi = cloud_extent(cloud, context)
    return float(np.float32(tau_d) * np.max(hi - lo))


def voxel_downsample(cloud, leaf: float, context=None):
    """voxelGridDownsample (src/alignment.cpp:79-87, pcl::VoxelGrid with a
    cubic leaf): (points, normals) of the voxel means, as float32 numpy."""
    ctx = context or default_context()
    p, q = _split_cloud(cloud)
    bp, bq = _Buf(p, "points"), _Buf(q, "normals")
    if bp.n != bq.n:
        raise ValueError("points and normals differ in length")
    ox = np.zeros((max(bp.n, 1), 3), np.float32)
    on = np.zeros((max(bp.n, 1), 3), np.float32)
    k = C.c_uint64()
    _check(_lib().ppf_voxel_downsample(ctx.handle, bp.ptr, bq.ptr, bp.n, float(leaf), C.c_void_p(ox.ctypes.data),
                                       C.c_void_p(on.ctypes.data), bp.n, C.byref(k)))
    return ox[: k.value].copy(), on[: k.value].copy()


def preprocess(scene_clouds, model_clouds, tau_d, scene_leaf_size: float, context=None):
    """The alignment driver's preparation (src/alignment.cpp:203-288): each
    model's d_dist from its extent and tau_d, scenes downsampled with
    scene_leaf_size, each model with its own d_dist.  Returns (scenes,
    models, model_d_dists) with clouds as (points, normals) pairs."""
    if len(tau_d) != len(model_clouds):
        raise ValueError("each model must have an associated tau_d")
    d_dists = [model_d_dist(m, t, context) for m, t in zip(model_clouds, tau_d)]
    scenes = [voxel_downsample(s, scene_leaf_size, context) for s in scene_clouds]
    models = [voxel_downsample(m, d, context) for m, d in zip(model_clouds, d_dists)]
    return scenes, models, d_dists


class Server:
    """Request loop over a resident model library (ppf_server_*).

    ``models`` are Model objects kept alive by the server.  ``submit`` queues a
    scene (host arrays, copied before it returns) against library models by
    index and returns a ticket; ``wait`` blocks for it and returns (poses
    (k, 4, 4), stats, latency_ms).  Each pose equals Model.ppf_lookup of the
    same (model, scene).  Submissions and waits may come from several threads.
    """

    def __init__(self, models, memory_budget: int = 40 << 30, workers: int = 4, max_batch: int = 16,
                 device: int = 0):
        self.models = list(models)
        arr = (C.c_void_p * len(self.models))(*[m.handle for m in self.models])
        h = C.c_void_p()
        _check(_lib().ppf_server_create(int(device), len(self.models), arr, int(memory_budget), int(workers),
                                        int(max_batch), C.byref(h)))
        self.handle = h
        # ticket -> number of target models: wait() sizes the pose buffer
        # that the library fills from it
        self._targets = {}
        self._lock = threading.Lock()

    def submit(self, cloud, model_ids, ref_point_downsample_factor: int = 1) -> int:
        p, q = _split_cloud(cloud)
        bp, bq = _Buf(p, "points"), _Buf(q, "normals")
        if bp.n != bq.n:
            raise ValueError("points and normals differ in length")
        ids = np.ascontiguousarray(np.atleast_1d(model_ids), np.uint32)
        t = C.c_uint64()
        _check(_lib().ppf_server_submit(self.handle, bp.ptr, bq.ptr, bp.n, int(ref_point_downsample_factor),
                                        ids.size, C.c_void_p(ids.ctypes.data), C.byref(t)))
        with self._lock:
            self._targets[t.value] = ids.size
        return t.value

    def wait(self, ticket: int, raise_on_no_votes: bool = True):
        with self._lock:
            k = self._targets.pop(int(ticket), None)
        if k is None:  # the library's own answer for a ticket it does not hold
            raise PPFError(1, f"unknown or already collected ticket {ticket}")
        poses = np.zeros((k, 16), np.float32)
        stats = (_capi.ppf_stats * k)()
        lat = C.c_double()
        status = _lib().ppf_server_wait(self.handle, int(ticket), C.c_void_p(poses.ctypes.data), stats,
                                        C.byref(lat))
        if not (status == 4 and not raise_on_no_votes):
            _check(status)
        return poses.reshape(k, 4, 4), [stats[i].as_dict() for i in range(k)], float(lat.value)

    def close(self):
        if getattr(self, "handle", None):
            _lib().ppf_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lookup_batch(models, scenes, context=None, return_stats: bool = False, raise_on_no_votes: bool = True):
    """Lookups of (models[i], scenes[i]) with one batched vote pass.

    Each pose equals Model.ppf_lookup(scene) for the same pair; returns an
    (n, 4, 4) array (and the per-request stats dicts with return_stats).
    """
    models, scenes = list(models), list(scenes)
    if len(models) != len(scenes):
        raise ValueError("models and scenes must have the same length")
    ctx = context or (models[0].ctx if models else default_context())
    n = len(models)
    mh = (C.c_void_p * max(n, 1))(*[m.handle for m in models])
    sh = (C.c_void_p * max(n, 1))(*[s.handle for s in scenes])
    poses = np.zeros((max(n, 1), 16), np.float32)
    stats = (_capi.ppf_stats * max(n, 1))()
    status = _lib().ppf_lookup_batch(ctx.handle, n, mh, sh, C.c_void_p(poses.ctypes.data), stats)
    if not (status == 4 and not raise_on_no_votes):
        _check(status)
    out = poses[:n].reshape(n, 4, 4)
    if return_stats:
        return out, [stats[i].as_dict() for i in range(n)]
    return out


def ppf_registration(scene_clouds, model_clouds, model_d_dists, ref_point_downsample_factor=1,
                     vote_count_threshold=0.4, cpu_clustering=False, use_l1_norm=False,
                     use_averaged_clusters=False, devUse=0, model_weights=None, context=None,
                     return_stats=False):
    """ppf_registration (include/ppf.h:9-15): poses[i][j] of model j in scene i (4x4 float32)."""
    L = _lib()
    scenes = [tuple(_Buf(a, "scene") for a in _split_cloud(c)) for c in scene_clouds]
    models = [tuple(_Buf(a, "model") for a in _split_cloud(c)) for c in model_clouds]
    ns, nm = len(scenes), len(models)
    sx = (C.c_void_p * max(ns, 1))(*[s[0].ptr for s in scenes])
    sn = (C.c_void_p * max(ns, 1))(*[s[1].ptr for s in scenes])
    sc = (C.c_uint64 * max(ns, 1))(*[s[0].n for s in scenes])
    mx = (C.c_void_p * max(nm, 1))(*[m[0].ptr for m in models])
    mn = (C.c_void_p * max(nm, 1))(*[m[1].ptr for m in models])
    mc = (C.c_uint64 * max(nm, 1))(*[m[0].n for m in models])
    dd = np.ascontiguousarray(np.asarray(model_d_dists, np.float32))
    if dd.size != nm:
        raise ValueError("one d_dist per model is required")
    poses = np.zeros((max(ns, 1), max(nm, 1), 16), np.float32)
    stats = (_capi.ppf_stats * max(ns * nm, 1))()
    ctx_h = context.handle if context is not None else None
    status = L.ppf_registration(
        ctx_h, ns, sx, sn, sc, nm, mx, mn, mc, dd.ctypes.data_as(_capi._fp),
        int(ref_point_downsample_factor), float(vote_count_threshold), int(bool(cpu_clustering)),
        int(bool(use_l1_norm)), int(bool(use_averaged_clusters)), int(devUse), None,
        C.c_void_p(poses.ctypes.data), stats,
    )
    if status not in (0, 4):
        _check(status)
    out = [[poses[i, j].reshape(4, 4).copy() for j in range(nm)] for i in range(ns)]
    if return_stats:
        return out, [[stats[i * nm + j].as_dict() for j in range(nm)] for i in range(ns)]
    return out
