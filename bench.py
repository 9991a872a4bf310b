"""Benchmark: PPF registrations/s on the multi-model scene workload.

Workload (one "step"): one 60k-point scene holding four 30%-occluded models
(superellipsoid, torus, 3-capsule union, spheres on a slab; 3k-6k points
each) registered against all four models with ref_point_df=5 and
tau_d = 0.03/0.035/0.03/0.05 of each model's diameter: four registrations.
Each step rebuilds the four model hash arrays and runs the four lookups, the
work the reference's ppf_registration does for one scene.

value : registrations/s with the clouds already in device memory
        (ppf_registration on device pointers), device time over K steps.
e2e   : the same through the C ABI with host buffers in pinned memory; the
        host->device copies of the clouds and the device->host read of the
        poses are inside the timed region.
clocks: nvidia-smi samples the SM clock and throttle reasons every 2.5 s inside
        the timed region (denser sampling stretched the host-synchronised part
        of a step by up to 10% on B200).
L2    : a 256 MB buffer is written on the engine's stream after every timed
        step (inside the timed region), and each step's model tables (about
        1 GB for the four models) exceed the 126 MB L2 anyway.
--profile-case: one lookup of the first model against the scene at
        ref_point_df=50 (same model tables, 10x fewer scene reference points),
        a short vote launch for ncu captures; prints the lookup's stats.
roofline: the vote kernel (dominant), algorithmic bytes 4 B per vote
        (one 32-bit run entry streamed per vote) + 32 B per scene pair
        evaluated, over its CUDA-event time, against MEASURED_PEAKS.json.
cpu_baseline: the CPU oracle (C++/OpenMP restatement of the reference path)
        on a bounded sample of scene reference points, scaled.
served: (1 GPU) the small library preset of --serve on its first 24 requests:
        plain ppf_registration per request, one batched lookup, and the request
        loop under Poisson arrivals (p50/p99 latency), with the served poses
        compared to plain; host wall clock, after the timed region.

Multi-GPU: replicas (each rank registers its own copy of the scene; no
collective on the data path), weak scaling; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402

METRIC = "registrations/s"
TAU_D = (0.03, 0.035, 0.03, 0.05)
REF_DF = 5
THR = 0.3
# DRAM bytes (read + write) per vote of the vote kernel for each of the
# workload's four models, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on each model's profile case (--profile-all: the same
# model tables against the scene at ref_point_df=50).  A model's entries are
# re-read by concurrent work items while still in L2, so its DRAM bytes scale
# with its votes; the 3047-point model's tables fit L2 entirely.
DRAM_BYTES_PER_VOTE = (0.04995, 0.03125, 0.04418, 0.001337)
# Shared-memory bank wavefronts per warp-wide atomic of the vote kernel, from
# ncu on the first model's profile case
# (l1tex__data_pipe_lsu_wavefronts_mem_shared_op_atom.sum over
# smsp__inst_executed_op_shared_atom.sum).
VOTE_WAVEFRONTS_PER_ATOMIC = 1.94


def shared_atomic_peaks(device):
    """Warp-wide shared atomics one SM completes per cycle, measured by the
    probe library (peaks/shared_atomic_peak.cu) for its three address
    patterns: one wavefront, two wavefronts, and one word for all lanes.
    Best of three launches each; None when the probe is not built."""
    import ctypes

    lib_path = ROOT / "ppf-registration-spatial-hashing_b200" / "libppf_peaks.so"
    if not lib_path.exists():
        return None
    lib = ctypes.CDLL(str(lib_path))
    f = lib.ppf_peak_shared_atomics
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double),
                  ctypes.POINTER(ctypes.c_double)]
    out = {}
    for pattern, name in ((0, "1_wavefront"), (1, "2_wavefronts"), (2, "one_word")):
        best = 0.0
        for _ in range(3):
            rate, ms = ctypes.c_double(), ctypes.c_double()
            rc = f(device, pattern, 20000, ctypes.byref(rate), ctypes.byref(ms))
            if rc != 0:
                raise RuntimeError(f"shared atomic probe failed: CUDA error {rc}")
            best = max(best, rate.value)
        out[name] = best
    return out


def atomic_roofline(peaks, votes, vote_s, sm_mhz, n_sm):
    """The vote kernel's warp-wide shared atomics per SM-cycle against the
    probe's rate.  Every vote is one lane of a warp-wide atomic; the unrolled
    passes keep all 32 lanes busy and the masked remainder of a segment holds
    about 1% of the votes, so the kernel issues about votes / 32 of them.  The
    ceiling at the kernel's own conflict level interpolates the probe's cycles
    per atomic linearly between one and two wavefronts."""
    if not peaks or vote_s <= 0 or not sm_mhz:
        return None
    achieved = votes / 32.0 / (vote_s * sm_mhz * 1e6 * n_sm)
    c1, c2 = 1.0 / peaks["1_wavefront"], 1.0 / peaks["2_wavefronts"]
    ceiling = 1.0 / (c1 + (VOTE_WAVEFRONTS_PER_ATOMIC - 1.0) * (c2 - c1))
    return {"unit": "warp-wide shared atomics per SM cycle", "achieved": achieved,
            "peak_measured": peaks, "wavefronts_per_atomic": VOTE_WAVEFRONTS_PER_ATOMIC,
            "ceiling_at_kernel_conflicts": ceiling, "frac": achieved / ceiling,
            "frac_of_conflict_free": achieved / peaks["1_wavefront"], "sm_mhz": sm_mhz, "sms": n_sm}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_group(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist

    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(dist, value, device=None):
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=2500, out_dir=None):
        import tempfile

        self.gpu = gpu_index
        self.interval_ms = int(interval_ms)
        self.proc = None
        self.path = Path(out_dir or tempfile.gettempdir()) / f"clocks_rank{gpu_index}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval_ms)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [ln.split(",") for ln in self.path.read_text().splitlines() if ln.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows)}


def workload(seed=1001):
    pkg = ge.load_package()
    spec = pkg.synthetic.config_multi_model(seed=seed)
    return pkg, spec


def workload_name(spec, avg):
    """The bench workload as named in both arms' JSON lines."""
    return ("multi-model scene: 4 models (superellipsoid/torus/capsules/spheres-on-slab, "
            f"{'/'.join(str(len(m)) for m in spec.models)} pts), {len(spec.scene)}-pt scene, "
            "ref_point_df=5, tau_d=0.03/0.035/0.03/0.05, vote_count_threshold=0.3, GPU clustering, "
            f"use_averaged_clusters={'on' if avg else 'off'}")


def recall_of(spec, poses):
    """Pose errors against the ground truth and recall at two bounds: the
    north star's (translation <= 1% of the model diameter, rotation <= 2 deg)
    and the reference driver's validation (0.1 diameter, 12 deg;
    src/alignment.cpp:300-335)."""
    pkg = ge.load_package()
    families = spec.extra.get("families", [None] * len(spec.models))
    errs, errs_sym = [], []
    for inst in spec.instances:
        P = poses[inst.model_index]
        G = inst.pose
        terr = float(np.linalg.norm(P[:3, 3] - G[:3, 3])) / spec.diameters[inst.model_index]
        errs.append((terr, pkg.synthetic.rotation_error_deg(P[:3, :3], G[:3, :3])))
        errs_sym.append((terr, pkg.synthetic.rotation_error_deg(P[:3, :3], G[:3, :3], families[inst.model_index])))

    def count(e, t_max, a_max):
        return f"{sum(t <= t_max and a <= a_max for t, a in e)}/{len(e)}"

    return {"terr_over_diam_and_deg": errs, "at_1pct_2deg": count(errs, 0.01, 2.0),
            "at_reference_bounds_0.1diam_12deg": count(errs, 0.1, 12.0),
            "modulo_shape_symmetry": {"terr_over_diam_and_deg": errs_sym, "at_1pct_2deg": count(errs_sym, 0.01, 2.0),
                                      "at_reference_bounds_0.1diam_12deg": count(errs_sym, 0.1, 12.0)}}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_sample(orc, O, spec, refs_per_model, offset, threads):
    """One bounded sample of the workload on the CPU oracle: per model, its
    hash array in full and `refs_per_model` scene reference points evenly
    spaced from `offset` (a multiple of ref_point_df).  Returns the measured
    seconds, the projected seconds of the full step (vote time scaled by
    reference points, builds as timed) and the reference points done."""
    sc = spec.scene
    n_ref = (len(sc) + REF_DF - 1) // REF_DF
    stride = max(1, n_ref // refs_per_model)
    t0 = time.perf_counter()
    proj = 0.0
    done = 0
    for m, d in zip(spec.models, spec.d_dists):
        r = O.register((m.points, m.normals), (sc.points, sc.normals), d, REF_DF, THR, n_threads=threads,
                       sr_range=(offset, len(sc)), sr_step=stride * REF_DF)
        proj += r["t_build"] + r["t_vote"] / max(r["n_refs"], 1) * n_ref
        done += r["n_refs"]
    return time.perf_counter() - t0, proj, done


def cpu_baseline(spec, sample_refs=2, threads=None, offset=0):
    """The oracle (C++/OpenMP restatement of the reference path) on a bounded
    sample of the workload: every model's hash array in full plus
    `sample_refs` scene reference points per model; the registration rate is
    projected by scaling the vote time to all reference points."""
    orc = ge.load_oracle()
    O = orc.Oracle()
    threads = threads or orc.n_cores()
    n_ref = (len(spec.scene) + REF_DF - 1) // REF_DF
    secs, proj, done = cpu_sample(orc, O, spec, sample_refs, offset, threads)
    return {"value": len(spec.models) / proj, "unit": METRIC, "cores": threads, "kind": "port",
            "projected": True,
            "sample": f"{done} scene reference points (about {sample_refs} per model, evenly spaced) of {n_ref} "
                      f"per model, all model hash arrays built; {secs:.1f} s measured, vote time scaled by "
                      f"reference points to a full step of {proj:.0f} s"}


def run_reference_arm(args):
    """The reference's algorithm on the host cores (the oracle restatement).
    Each timed step is a bounded sample: all four model hash arrays plus
    --cpu-refs scene reference points per model, a different evenly spaced set
    per step (offsets step * stride / steps).  ms_per_step is the measured
    time of one such sample step; value is the registration rate projected to
    full steps (vote time scaled by reference points), and the line says so."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    orc = ge.load_oracle()
    O = orc.Oracle()
    threads = orc.n_cores()
    _, spec = workload()
    n_ref = (len(spec.scene) + REF_DF - 1) // REF_DF
    stride = max(1, n_ref // args.cpu_refs)
    steps = max(1, args.steps)
    for w in range(args.warmup):
        # warm-up samples: page in the oracle and the clouds (a few reference points)
        cpu_sample(orc, O, spec, 1, REF_DF * ((w * 7919) % n_ref), threads)
    meas, projs, done = [], [], 0
    for k in range(steps):
        offset = REF_DF * ((k * stride) // steps)
        secs, proj, n = cpu_sample(orc, O, spec, args.cpu_refs, offset, threads)
        meas.append(secs)
        projs.append(proj)
        done += n
    value = len(spec.models) / statistics.median(projs)
    per_step = [len(spec.models) / p for p in projs]
    cb = {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "projected": True,
          "sample": f"{steps} steps, each all four model hash arrays and about {args.cpu_refs} scene reference "
                    f"points per model ({done} distinct points of {n_ref} per model in all, a different evenly "
                    "spaced set per step); value = median over steps of the projected registration rate"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
            "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * statistics.mean(meas), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(spec, args.avg), "parallelism": f"host threads ({threads})"},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "projected": {"value_is_projected": True,
                          "ms_per_step_is": "measured wall time of one sample step",
                          "projected_ms_per_full_step": 1000.0 * statistics.median(projs),
                          "per_step_projected_value_min_median_max": [min(per_step), statistics.median(per_step),
                                                                      max(per_step)]},
            "note": "the reference runs this path only on the GPU and cannot at this size (int pair indexing "
                    "beyond 46340 points, every vote materialised); the timed arm is the oracle restatement of "
                    "its algorithm on the host cores"}
    print(json.dumps(line), flush=True)


def run_cpu_config1(args):
    """BASELINE config 1 (2000-point model, 10000-point scene, ref_point_df 5,
    tau_d 0.05) registered in full by the CPU oracle on all host cores, and a
    1-core run over every 10th scene reference point, projected (with
    --cpu-one-core-full: the 1-core run registers in full as well)."""
    orc = ge.load_oracle()
    O = orc.Oracle()
    pkg = ge.load_package()
    spec = pkg.synthetic.config_plain(seed=1000)
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    threads = orc.n_cores()
    t0 = time.perf_counter()
    r = O.register((m.points, m.normals), (s.points, s.normals), d, 5, 0.3, n_threads=threads)
    full = time.perf_counter() - t0
    line = {"mode": "cpu_config1", "workload": "config 1: 2000-pt superellipsoid, 10000-pt scene, "
            "ref_point_df 5, tau_d 0.05, threshold 0.3, GPU-style clustering",
            "n_votes": r["n_votes"], "all_cores": threads, "all_cores_s": full,
            "all_cores_registrations_per_s": 1.0 / full}
    t0 = time.perf_counter()
    if args.cpu_one_core_full:
        r1 = O.register((m.points, m.normals), (s.points, s.normals), d, 5, 0.3, n_threads=1)
        one = time.perf_counter() - t0
        line.update({"one_core_s": one, "one_core_registrations_per_s": 1.0 / one,
                     "one_core_pose_equals_all_cores": bool(np.array_equal(r1["pose"], r["pose"]))})
    else:
        r1 = O.register((m.points, m.normals), (s.points, s.normals), d, 5, 0.3, n_threads=1, sr_step=50)
        one = time.perf_counter() - t0
        n_ref = (len(s) + 4) // 5
        one_proj = r1["t_build"] + r1["t_vote"] / max(r1["n_refs"], 1) * n_ref
        line.update({"one_core_sample_s": one, "one_core_sample_refs": r1["n_refs"],
                     "one_core_projected_s": one_proj, "one_core_registrations_per_s_projected": 1.0 / one_proj})
    print(json.dumps(line), flush=True)


SERVE_PRESETS = {
    # name: (models, model point range, scene point range, scenes, workers, seed)
    "small": (8, (2000, 6000), (5000, 40000), 64, 4, 1003),
    # 16 models of 2k-20k points, scenes of 5k-200k points
    # (the first --serve-scenes of its 256 scenes)
    "config3": (16, (2000, 20000), (5000, 200000), 24, 2, 1002),
    # 64 models of 2k-20k points, scenes of 5k-300k points
    "config4": (64, (2000, 20000), (5000, 300000), 16, 2, 1005),
}


def run_serve(args):
    """Library workload: --serve-preset small (8 models of 2k-6k points,
    scenes of 5k-40k points), config3 or config4 (BASELINE's library sizes,
    on the first --serve-scenes scenes); tau_d = 0.04, each scene holds 1-4
    library models and a request registers it against them (ref_point_df=5,
    threshold 0.3).

    plain  : one ppf_registration per request, rebuilding its models (the
             reference's per-call behaviour), requests one after another.
    batched: resident library; all requests in one ppf_lookup_batch.
    served : resident library behind the request loop (2 workers); requests
             arrive as a seeded Poisson process, at 70% of the batched rate
             (latency under load) and at 150% (capacity: the queue stays full).
    Every served pose is compared with the plain pose of the same pair."""
    import threading

    pkg = ge.load_package()
    n_models, model_range, scene_range, n_scenes, workers, seed = SERVE_PRESETS[args.serve_preset]
    n_scenes = args.serve_scenes or n_scenes
    workers = args.serve_workers or workers
    models, d_dists, scenes = pkg.synthetic.config_library(
        seed=seed, n_models=n_models, n_scenes=n_scenes, model_range=model_range, scene_range=scene_range)
    ctx = pkg.Context(0)
    reqs = [(sc, sorted({i.model_index for i in inst})) for sc, inst in scenes]
    n_reg = sum(len(ids) for _, ids in reqs)

    def plain_all(subset=None):
        out = []
        for sc, ids in (reqs if subset is None else subset):
            p = pkg.ppf_registration([sc], [models[j] for j in ids], [d_dists[j] for j in ids], REF_DF, THR,
                                     context=ctx)
            out.append(np.asarray(p[0]))
        return out

    # warm-up (pool, tuner, candidate hints): every request for the small
    # preset, the first one for the library configs
    plain_all(None if args.serve_preset == "small" else reqs[:1])
    ctx.synchronize()
    t0 = time.perf_counter()
    plain = plain_all()
    ctx.synchronize()
    t_plain = time.perf_counter() - t0

    lib = [pkg.Model(m, d, THR, context=ctx) for m, d in zip(models, d_dists)]

    def batched_all(subset=None):
        ms, ss = [], []
        for sc, ids in (reqs if subset is None else subset):
            for j in ids:
                ms.append(lib[j])
                ss.append(pkg.Scene(sc, d_dists[j], REF_DF, context=ctx))
        return pkg.lookup_batch(ms, ss, context=ctx, raise_on_no_votes=False)

    batched_all(None if args.serve_preset == "small" else reqs[:2])
    ctx.synchronize()
    t0 = time.perf_counter()
    batched_all()
    ctx.synchronize()
    t_batch = time.perf_counter() - t0

    srv = pkg.Server(lib, workers=workers, max_batch=args.serve_max_batch)
    for t in [srv.submit(sc, ids, REF_DF) for sc, ids in reqs[:4]]:
        srv.wait(t, raise_on_no_votes=False)

    def serve_at(load, seed):
        rate = load * len(reqs) / t_batch  # requests/s offered
        arrivals = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, len(reqs)))
        tickets = [None] * len(reqs)

        def submitter():
            start = time.perf_counter()
            for i, (sc, ids) in enumerate(reqs):
                d = start + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(sc, ids, REF_DF)

        t0 = time.perf_counter()
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        res = [srv.wait(t, raise_on_no_votes=False) for t in tickets]
        t_serve = time.perf_counter() - t0
        lat = np.array([r[2] for r in res])
        same = sum(int(np.array_equal(r[0], plain[i])) for i, r in enumerate(res))
        return {"offered_requests_per_s": rate, "registrations_per_s": n_reg / t_serve,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "identical_poses_vs_plain": f"{same}/{len(reqs)}"}

    light = serve_at(0.7, 7)
    heavy = serve_at(1.5, 8)
    nominal = serve_at(50.0 * t_batch / len(reqs), 9) if args.serve_preset == "config4" else None
    srv.close()
    line = {"mode": "serve", "metric": METRIC, "unit": METRIC, "higher_is_better": True, "n_gpus": 1,
            "plain": n_reg / t_plain, "batched": n_reg / t_batch, "served": heavy["registrations_per_s"],
            "batched_over_plain": t_plain / t_batch,
            "served_over_plain": heavy["registrations_per_s"] / (n_reg / t_plain),
            "served_at_70pct": light, "served_at_150pct": heavy,
            "requests": len(reqs), "registrations": n_reg, "data": "synthetic", "dtype": "f32",
            "scene_points_total": int(sum(len(sc) for sc, _ in reqs)),
            "config": {"preset": args.serve_preset,
                       "workload": f"library of {n_models} models ({model_range[0]}-{model_range[1]} pts, "
                                   f"tau_d=0.04), {len(reqs)} scenes of {scene_range[0]}-{scene_range[1]} pts "
                                   "holding 1-4 models each, ref_point_df=5, threshold 0.3",
                       "served": f"{workers} workers, max_batch {args.serve_max_batch}, Poisson arrivals at 70% "
                                 "and 150% of the batched rate"}}
    if nominal:
        line["served_at_50_requests_per_s"] = nominal
    return line


def run_large(args):
    """BASELINE config 5, the large stress case: a 40000-point model (dense
    superellipsoid + torus union, 1.6e9 ordered pairs in its hash array)
    against a 1M-point scene holding 10 instances (40% occlusion, plane and box
    clutter, sigma 1 mm), tau_d 0.025, threshold 0.3.  The model is built in
    full and timed.  The lookup runs at --large-ref-df (default 1000: 1000 of
    the 200000 scene reference points that ref_point_df 5 gives); its votes
    and vote time are reported as measured and, scaled by reference points,
    projected to ref_point_df 5."""
    import torch

    pkg = ge.load_package()
    spec = pkg.synthetic.config_large()
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    ctx = pkg.Context(0)
    dev = torch.device("cuda", 0)
    free0, total = torch.cuda.mem_get_info(dev)
    md = (torch.from_numpy(m.points).to(dev), torch.from_numpy(m.normals).to(dev))
    sd = (torch.from_numpy(s.points).to(dev), torch.from_numpy(s.normals).to(dev))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    model = pkg.Model(md, d, THR, context=ctx)
    ctx.synchronize()
    build_s = time.perf_counter() - t0
    free_build = torch.cuda.mem_get_info(dev)[0]
    scene = pkg.Scene(sd, d, args.large_ref_df, context=ctx)
    t0 = time.perf_counter()
    pose = model.ppf_lookup(scene, raise_on_no_votes=False)
    ctx.synchronize()
    lookup_s = time.perf_counter() - t0
    st = dict(model.stats)
    free_lookup = torch.cuda.mem_get_info(dev)[0]
    n_ref = (len(s) + args.large_ref_df - 1) // args.large_ref_df
    n_ref5 = (len(s) + 4) // 5
    scale = n_ref5 / n_ref
    best = min(((float(np.linalg.norm(pose[:3, 3] - i.pose[:3, 3])) / spec.diameters[0],
                 float(np.degrees(np.arccos(np.clip((np.trace(pose[:3, :3].T @ i.pose[:3, :3]) - 1) / 2, -1, 1)))))
                for i in spec.instances), key=lambda e: e[0])
    # the model build's two radix sorts: 4 passes of 32-bit keys + 32-bit
    # values and 8 passes of 64-bit keys + 32-bit values, each pass reading
    # and writing every element once
    P = len(m) ** 2
    sort_bytes = P * (4 * 2 * (4 + 4) + 8 * 2 * (8 + 4))
    print(json.dumps({
        "mode": "large", "workload": f"config 5: {len(m)}-pt model ({P:.3g} pairs), {len(s)}-pt scene with "
                                     f"{len(spec.instances)} instances, tau_d 0.025, threshold 0.3",
        "model_build_s": build_s, "model_keys": int(pkg.api._lib().ppf_model_num_keys(model.handle)),
        "num_chunks": model.num_chunks, "sort_algorithmic_bytes": sort_bytes,
        "ref_point_df": args.large_ref_df, "scene_ref_points": n_ref, "lookup_s": lookup_s,
        "n_votes": st["n_votes"], "vote_ms": st["vote_ms"], "total_ms": st["total_ms"],
        "votes_per_s": st["n_votes"] / (st["vote_ms"] / 1000.0) if st["vote_ms"] else None,
        "n_kept": st["n_kept"], "n_candidates": st["n_candidates"], "max_vote_count": st["max_vote_count"],
        "projected_ref_point_df5": {"scene_ref_points": n_ref5, "n_votes": st["n_votes"] * scale,
                                    "vote_s": st["vote_ms"] / 1000.0 * scale},
        "device_memory_used_gb": {"after_build": (free0 - free_build) / 1e9,
                                  "after_lookup": (free0 - free_lookup) / 1e9, "total": total / 1e9},
        "nearest_instance_err_terr_over_diam_deg": best}), flush=True)


def run_profile_case(args):
    """Lookups of the workload's models at ref_point_df=50 (same model tables,
    10x fewer scene reference points): --profile-model K (default 0), or all
    four with --profile-all.  Each model runs warmup + steps lookups, then the
    next model; one JSON line per model with its last lookup's stats."""
    pkg, spec = workload()
    ctx = pkg.Context(0)
    ks = range(len(spec.models)) if args.profile_all else [args.profile_model]
    models = [(k, pkg.Model(spec.models[k], spec.d_dists[k], THR, context=ctx),
               pkg.Scene(spec.scene, spec.d_dists[k], 50, context=ctx)) for k in ks]
    reps = max(1, args.warmup) + max(1, args.steps)
    # warm-up lookups of every model first, then the measured ones, so that
    # an ncu capture can skip the first len(models) * warmup vote launches
    for r in range(reps):
        for k, model, scene in models:
            model.ppf_lookup(scene, raise_on_no_votes=False)
            if r == reps - 1:
                st = model.stats
                n_ref = (len(spec.scene) + 49) // 50
                print(json.dumps({"profile_case": f"model {k} ({len(spec.models[k])} pts) x {len(spec.scene)}-pt "
                                                  "scene, ref_point_df=50",
                                  "n_votes": st["n_votes"], "vote_ms": st["vote_ms"], "total_ms": st["total_ms"],
                                  "alg_bytes": 4.0 * st["n_votes"] + 32.0 * n_ref * len(spec.scene),
                                  "model_entries_bytes": 4 * len(spec.models[k]) ** 2}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--avg", action="store_true", help="use_averaged_clusters on")
    ap.add_argument("--cpu-refs", type=int, default=2,
                    help="scene reference points per model in each CPU sample step")
    ap.add_argument("--cpu-one-core-full", action="store_true",
                    help="with --cpu-config1: register config 1 in full on one core too (minutes)")
    ap.add_argument("--cpu-config1", action="store_true",
                    help="config 1 registered in full by the CPU oracle (all cores) and a projected 1-core run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--clocks-dir", default=None, help="where the clock samples are written (default: temp dir)")
    ap.add_argument("--clock-interval-ms", type=int, default=2500,
                    help="nvidia-smi sampling interval during the timed region (each query stalls the "
                         "engine's CUDA calls briefly)")
    ap.add_argument("--serve", action="store_true",
                    help="library workload: plain per-request registration vs batched lookups vs the "
                         "request loop under Poisson arrivals (p50/p99 latency)")
    ap.add_argument("--serve-preset", default="small", choices=sorted(SERVE_PRESETS))
    ap.add_argument("--serve-scenes", type=int, default=0, help="scenes (requests); 0: the preset's")
    ap.add_argument("--serve-workers", type=int, default=0, help="request-loop workers; 0: the preset's")
    ap.add_argument("--serve-max-batch", type=int, default=16)
    ap.add_argument("--no-serve", action="store_true",
                    help="leave the served-mode summary out of the default bench line")
    ap.add_argument("--bench-serve-scenes", type=int, default=24,
                    help="requests of the served-mode summary in the default bench line (small library preset)")
    ap.add_argument("--profile-case", action="store_true",
                    help="one lookup of one model at ref_point_df=50 (short vote launch for ncu)")
    ap.add_argument("--profile-model", type=int, default=0)
    ap.add_argument("--profile-all", action="store_true", help="the profile case of each of the four models")
    ap.add_argument("--large", action="store_true", help="config 5 (40k-point model, 1M-point scene), sampled lookup")
    ap.add_argument("--large-ref-df", type=int, default=1000)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.cpu_config1:
        return run_cpu_config1(args)
    if args.profile_case or args.profile_all:
        return run_profile_case(args)
    if args.serve:
        print(json.dumps(run_serve(args)), flush=True)
        return
    if args.large:
        return run_large(args)

    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_group(world, "nccl")
    pkg, spec = workload()
    ctx = pkg.Context(local)
    dev = torch.device("cuda", local)
    models_d = [(torch.from_numpy(m.points).to(dev), torch.from_numpy(m.normals).to(dev)) for m in spec.models]
    scene_d = (torch.from_numpy(spec.scene.points).to(dev), torch.from_numpy(spec.scene.normals).to(dev))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def step(models, scene):
        return pkg.ppf_registration([scene], models, spec.d_dists, REF_DF, THR, False, False, args.avg,
                                    local, None, context=ctx, return_stats=True)

    # vote chunks of each model (queried once, outside the timed region)
    chunks = [pkg.Model(m, d, THR, context=ctx).num_chunks for m, d in zip(models_d, spec.d_dists)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.fill_(1)

    for _ in range(max(1, args.warmup)):  # at least one, for the correctness guard below
        poses, stats = step(models_d, scene_d)
        flush_l2()
    warm_poses = [p.copy() for p in poses[0]]
    recall = recall_of(spec, poses[0])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    vote_ms = 0.0
    votes = 0
    traffic = 0.0
    pairs = 0
    with ClockSampler(local, args.clock_interval_ms, args.clocks_dir) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            poses, stats = step(models_d, scene_d)
            flush_l2()
            for k, s in enumerate(stats[0]):
                vote_ms += s["vote_ms"]
                votes += s["n_votes"]
                traffic += s["n_votes"] * DRAM_BYTES_PER_VOTE[k]
        ev1.record(stream)
        ev1.synchronize()
        if dist:
            dist.barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.kernel_launches - launches0
    # the engine is deterministic: every timed step must give the warm-up poses bit for bit
    changed = [k for k, (a, b) in enumerate(zip(warm_poses, poses[0])) if not np.array_equal(a, b)]
    if changed:
        sys.stderr.write(f"bench: poses of models {changed} changed between warm-up and timed steps\n")
        sys.exit(3)
    n_ref = (len(spec.scene) + REF_DF - 1) // REF_DF
    # every (scene reference point, chunk) work item walks the whole scene, so
    # a model of C chunks evaluates each scene pair C times
    pairs = n_ref * len(spec.scene) * sum(chunks) * args.steps
    ms_max = reduce_max(dist, ms, dev)
    regs = world * len(spec.models) * args.steps
    value = regs / (ms_max / 1000.0)

    # e2e: host buffers through the C ABI
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()

        host_models = [(pinned(m.points), pinned(m.normals)) for m in spec.models]
        host_scene = (pinned(spec.scene.points), pinned(spec.scene.normals))
        step(host_models, host_scene)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev0.record(stream)
        k = max(1, min(args.steps, 3))
        for _ in range(k):
            step(host_models, host_scene)
            flush_l2()
        ev1.record(stream)
        ev1.synchronize()
        wall = time.perf_counter() - t0
        e_ms = reduce_max(dist, max(ev0.elapsed_time(ev1), wall * 1000.0), dev)
        h2d = sum(m[0].nbytes + m[1].nbytes for m in host_models) + host_scene[0].nbytes + host_scene[1].nbytes
        e2e = {"value": world * len(spec.models) * k / (e_ms / 1000.0), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(len(spec.models) * 64)}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    clocks = clk.summary()
    atomics = atomic_roofline(shared_atomic_peaks(local), votes, vote_ms / 1000.0, clocks.get("sm_mhz"),
                              torch.cuda.get_device_properties(dev).multi_processor_count)
    alg_bytes = 4.0 * votes + 32.0 * pairs
    vote_s = vote_ms / 1000.0
    achieved = alg_bytes / vote_s / 1e9 if vote_s > 0 else 0.0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": workload_name(spec, args.avg),
            "parallelism": f"replicas x{world}",
            "l2": "256 MB L2 flush after every timed step; per-step model tables (~1 GB) exceed L2",
        },
        "votes_per_s": world * votes / (ms_max / 1000.0),
        "votes_per_step": votes // args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": "vote_batch_kernel (one launch per step: the four lookups' vote passes)",
                     "traffic": traffic / args.steps,
                     "traffic_note": "DRAM bytes per launch: measured bytes per vote of each model's profile "
                                     "case times its votes; the entries are served from L2 (about 0.5% of the "
                                     "algorithmic bytes reach DRAM); the kernel is latency-bound on its L2 entry "
                                     "loads, with the l1tex data pipe (shared atomics + loads) at 69% of peak on the "
                                     "profile case",
                     "alg_bytes_per_launch": alg_bytes / args.steps,
                     "alg_bytes_rule": "4 B per vote + 32 B per scene pair evaluated (pairs x vote chunks of the model)",
                     "vote_chunks": chunks,
                     "vote_ms_per_launch": vote_ms / args.steps,
                     "shared_atomics": atomics},
        "gpu_launches": int(launches),
        "vote_segments_tuned": [int(s["vote_segment"]) for s in stats[0]],
        "recall": recall,
        "clocks": clocks,
    }
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(spec, sample_refs=args.cpu_refs)
    if world == 1 and not args.no_serve:
        # plain / batched / served on the small library preset, after the
        # timed region (host wall clock; see run_serve)
        sv = argparse.Namespace(**vars(args))
        sv.serve_preset, sv.serve_scenes, sv.serve_workers = "small", args.bench_serve_scenes, 0
        try:
            line["served"] = {k: v for k, v in run_serve(sv).items()
                              if k not in ("mode", "metric", "unit", "higher_is_better", "n_gpus", "data", "dtype")}
        except Exception as e:  # the summary is an addition; its failure must not cost the bench line
            line["served"] = {"error": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
