"""Autotuner of launch shapes (no reference counterpart: the reference's launch shapes are constants).

For one kernel and one workload shape on one device, every candidate launch shape is run and timed on the device
(CUDA events on the launching stream, one untimed run first, the median of `repeats` timed runs), and the fastest is
kept in a JSON cache keyed by device and shape, so the search runs once per (device, shape):

    tuner = Tuner()                                        # cache: $XCB200_CACHE_DIR/tune_v1.json (~/.cache/xclean_b200)
    best = tune_front(gf, left_ptr, right_ptr, F, budget, half, dlo, dhi, stream, tuner)   # applied to gf
    best = tune_mapmatch(mm, args, stream, tuner)          # applied to mm

A cache entry: {"best": {knob: value}, "ms": [median ms per candidate], "candidates": [{knob: value}, ...],
"repeats": n}.  Selection is deterministic: the smallest median, ties to the earlier candidate; a cached entry is
reused only when it was made for the same candidate list.  Results never depend on the launch shape (the kernels'
outputs are bit-identical across the candidates), only the time does.
"""
from __future__ import annotations

import json
import os
import statistics

from . import _lib

CACHE_FILE = "tune_v1.json"

# knob name -> C-ABI knob id
STEREO_WARPS = "stereo_warps"
STEREO_GROUP = "stereo_group"
MM_LANES = "mm_lanes"
KNOB_IDS = {STEREO_WARPS: _lib.XCB_TUNE_STEREO_WARPS, STEREO_GROUP: _lib.XCB_TUNE_STEREO_GROUP,
            MM_LANES: _lib.XCB_TUNE_MM_LANES}


def cache_dir():
    d = os.environ.get("XCB200_CACHE_DIR") or os.path.join(os.path.expanduser("~"), ".cache", "xclean_b200")
    os.makedirs(d, exist_ok=True)
    return d


def device_key(device=None):
    """Name and SM count of the CUDA device (the tuning is valid for that part only)."""
    import torch
    p = torch.cuda.get_device_properties(device if device is not None else torch.cuda.current_device())
    return "%s|sm%d%d|%dSM" % (p.name, p.major, p.minor, p.multi_processor_count)


def shape_key(kernel, shape):
    return kernel + "|" + "|".join("%s=%s" % (k, shape[k]) for k in sorted(shape))


def gpu_timer(run, repeats, stream=None):
    """Median device time (ms) of `run()` over `repeats` runs after one untimed run."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    run()
    torch.cuda.synchronize()
    ms = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        run()
        e1.record(s)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(statistics.median(ms))


class Tuner:
    """The search and its cache.  timer(run, repeats) -> ms (default: gpu_timer); device: the device key (default:
    the current CUDA device's)."""

    def __init__(self, path=None, repeats=5, timer=None, device=None):
        self.path = path or os.path.join(cache_dir(), CACHE_FILE)
        self.repeats = int(repeats)
        self.timer = timer or gpu_timer
        self._device = device
        self.cache = self._load()

    def device(self):
        if self._device is None:
            self._device = device_key()
        return self._device

    def _load(self):
        try:
            with open(self.path) as fh:
                c = json.load(fh)
            return c if isinstance(c, dict) else {}
        except (OSError, ValueError):
            return {}

    def _save(self):
        tmp = "%s.%d" % (self.path, os.getpid())
        with open(tmp, "w") as fh:
            json.dump(self.cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def key(self, kernel, shape):
        return self.device() + "|" + shape_key(kernel, shape)

    def choose(self, kernel, shape, candidates, apply, run, force=False):
        """-> (best candidate, cache entry).  apply(candidate) sets the launch shape; run() launches the workload."""
        cands = [dict(c) for c in candidates]
        if not cands:
            raise ValueError("Tuner.choose: no candidates")
        k = self.key(kernel, shape)
        ent = self.cache.get(k)
        if not force and ent and ent.get("candidates") == cands and ent.get("best") in cands:
            apply(ent["best"])
            return dict(ent["best"]), ent
        ms = []
        for c in cands:
            apply(c)
            ms.append(float(self.timer(run, self.repeats)))
        i = min(range(len(cands)), key=lambda j: (ms[j], j))
        ent = {"best": cands[i], "ms": ms, "candidates": cands, "repeats": self.repeats}
        self.cache[k] = ent
        self._save()
        apply(cands[i])
        return dict(cands[i]), ent


def _front_apply(gf):
    def apply(c):
        for name, v in c.items():
            gf.set_tuning(KNOB_IDS[name], int(v))
    return apply


def stereo_candidates(half):
    wmax = 6 if int(half) >= 5 else 8
    return [{STEREO_WARPS: w, STEREO_GROUP: g} for w in (4, 6, 8) if w <= wmax for g in (8, 16, 32)]


def tune_front(gf, left_ptr, right_ptr, F, budget, half, dlo, dhi, stream, tuner=None, force=False):
    """Tune the stereo launch shape of GpuFront `gf` on the batched pipeline of F frames already on the device (the
    whole graph is timed; only its stereo stage depends on the knobs).  -> (best, cache entry)."""
    tuner = tuner or Tuner()
    shape = {"W": gf.W, "H": gf.H, "cap": gf.cap, "frames": int(F), "budget": int(budget), "half": int(half),
             "dlo": int(dlo), "dhi": int(dhi)}
    sptr = stream.cuda_stream

    def run():
        gf.pipeline_dev(left_ptr, right_ptr, int(F), int(budget), int(half), int(dlo), int(dhi), match_prev=False,
                        stream=sptr)

    import torch
    timer = tuner.timer
    tuner_timer = (lambda r, n: timer(r, n, stream)) if timer is gpu_timer else timer
    saved, tuner.timer = tuner.timer, tuner_timer
    try:
        return tuner.choose("front_stereo", shape, stereo_candidates(half), _front_apply(gf), run, force)
    finally:
        tuner.timer = saved
        torch.cuda.synchronize()


def tune_mapmatch(mm, match_args, stream, tuner=None, force=False):
    """Tune the gate kernel's lanes per landmark of MapMatcher `mm` on one batched device call (match_args: the
    keyword arguments of mm.match_dev).  -> (best, cache entry)."""
    tuner = tuner or Tuner()
    F, L = int(match_args["uv"].shape[0]), int(match_args["uv"].shape[1])
    shape = {"W": mm.W, "H": mm.H, "frames": F, "landmarks": L, "keypoints": int(match_args["kp"].shape[1])}

    def apply(c):
        mm.set_tuning(KNOB_IDS[MM_LANES], int(c[MM_LANES]))

    def run():
        mm.match_dev(**match_args, stream=stream.cuda_stream)

    timer = tuner.timer
    saved = tuner.timer
    tuner.timer = (lambda r, n: timer(r, n, stream)) if timer is gpu_timer else timer
    try:
        return tuner.choose("mapmatch_gate", shape, [{MM_LANES: v} for v in (1, 2, 4, 8)], apply, run, force)
    finally:
        tuner.timer = saved
