"""The autotuner's search and cache (xclean_b200.tune) on the host: deterministic choice, the cache file's format, reuse
of a cached choice, and keys that separate devices and shapes.  A fake timer stands in for the device."""
import json

import pytest

from xclean_b200 import tune as T


def _tuner(tmp_path, times, device="FakeGPU|sm100|148SM"):
    calls = []

    def timer(run, repeats):
        run()
        return times[len(calls) - 1] if calls else 0.0

    class Rec:
        def __init__(self):
            self.current = None

        def apply(self, c):
            self.current = dict(c)
            calls.append(dict(c))

        def run(self):
            pass

    return T.Tuner(path=str(tmp_path / "tune.json"), repeats=3, timer=timer, device=device), Rec(), calls


def test_choice_is_the_fastest_and_ties_go_to_the_earlier_candidate(tmp_path):
    cands = [{"stereo_warps": w, "stereo_group": g} for w in (4, 8) for g in (16, 32)]
    tuner, rec, calls = _tuner(tmp_path, [3.0, 1.0, 1.0, 2.0])
    best, ent = tuner.choose("front_stereo", {"W": 1241, "H": 376, "half": 4}, cands, rec.apply, rec.run)
    assert best == cands[1] and rec.current == cands[1]
    assert ent["ms"] == [3.0, 1.0, 1.0, 2.0] and ent["candidates"] == cands and ent["repeats"] == 3
    # the file: one entry under the device + kernel + shape key, readable JSON
    data = json.load(open(tmp_path / "tune.json"))
    (key,) = data
    assert key == "FakeGPU|sm100|148SM|front_stereo|H=376|W=1241|half=4"
    assert data[key]["best"] == cands[1]


def test_cached_choice_is_reused_and_invalidated_by_other_candidates(tmp_path):
    cands = [{"mm_lanes": v} for v in (1, 2, 4, 8)]
    tuner, rec, calls = _tuner(tmp_path, [4.0, 3.0, 1.0, 2.0])
    tuner.choose("mapmatch_gate", {"frames": 100}, cands, rec.apply, rec.run)
    n = len(calls)
    t2 = T.Tuner(path=str(tmp_path / "tune.json"), repeats=3, timer=lambda r, k: pytest.fail("re-timed"),
                 device="FakeGPU|sm100|148SM")
    best, _ = t2.choose("mapmatch_gate", {"frames": 100}, cands, rec.apply, rec.run)
    assert best == {"mm_lanes": 4} and rec.current == {"mm_lanes": 4} and len(calls) == n + 1
    # another shape, another device, or another candidate list: searched again
    assert t2.key("mapmatch_gate", {"frames": 200}) != t2.key("mapmatch_gate", {"frames": 100})
    t3 = T.Tuner(path=str(tmp_path / "tune.json"), repeats=3, timer=lambda r, k: 1.0, device="Other|sm90|132SM")
    assert t3.key("mapmatch_gate", {"frames": 100}) != t2.key("mapmatch_gate", {"frames": 100})
    best, ent = t2.__class__(path=str(tmp_path / "tune.json"), repeats=3, timer=lambda r, k: 1.0,
                             device="FakeGPU|sm100|148SM").choose("mapmatch_gate", {"frames": 100}, cands[:2],
                                                                   rec.apply, rec.run)
    assert best == cands[0] and ent["candidates"] == cands[:2]


def test_stereo_candidates_respect_the_window_limit():
    assert all(c["stereo_warps"] <= 6 for c in T.stereo_candidates(5))
    assert {c["stereo_warps"] for c in T.stereo_candidates(4)} == {4, 6, 8}
    assert {c["stereo_group"] for c in T.stereo_candidates(3)} == {8, 16, 32}
