"""Loading helpers for the golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py)."""
import hashlib
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("calib160", "small752", "kitti1241")


def png_decode(buf):
    import cv2
    return cv2.imdecode(np.asarray(buf, np.uint8), cv2.IMREAD_UNCHANGED)


def load_case(name):
    z = np.load(os.path.join(GOLDEN, "front_%s.npz" % name))
    d = {k: z[k] for k in z.files}
    for k in ("left0", "right0", "left1"):
        d[k] = png_decode(d[k])
    return d


def meta():
    z = np.load(os.path.join(GOLDEN, "front_meta.npz"))
    return {k: z[k] for k in z.files}


def calib_of(case):
    m = meta()
    return dict(dy_vend=int(case["dy_vend"]), dx_vend=int(case["dx_vend"]), blur_vr=int(case["blur_vr"]),
                blur_vc=int(case["blur_vc"]), kf=np.asarray(m["kf"], np.float32), q99=float(m["q99"]))


def pattern():
    """The ORB test pairs probed from this machine's cv2, checked against the fixture's hash."""
    from xclean_b200.front.gpu_front import probe_orb_pattern
    pat = probe_orb_pattern()
    h = hashlib.sha256(pat.astype(np.int64).tobytes()).hexdigest()
    if h != str(meta()["pattern_sha256"]):
        import pytest
        pytest.skip("the cv2 build here has a different ORB pattern than the fixtures' (%s)" % h[:12])
    return pat


def stereo_variants(case):
    out = []
    for k in sorted(case):
        if k.startswith("st_") and k.endswith("_args"):
            tag = k[3:-5]
            dlo, dhi, band, dy = case[k]
            out.append((tag, None if dlo < 0 else int(dlo), None if dhi < 0 else int(dhi), float(dy), int(band)))
    return out


def same_bits(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float64 or b.dtype == np.float64:
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return np.array_equal(a, b)


def mapmatch_cases():
    """The gated map matcher fixture (tests/golden/make_golden_mapmatch.py): name -> dict of inputs and outputs."""
    z = np.load(os.path.join(GOLDEN, "mapmatch_golden.npz"))
    out = {}
    for n in z["names"]:
        n = str(n)
        out[n] = {k.split("__", 1)[1]: z[k] for k in z.files if k.startswith(n + "__")}
    return out


def same_outputs(got, want):
    """(kp index, distance, d2) triples equal bit for bit (NaN payloads included)."""
    return (np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
            and np.array_equal(np.asarray(got[2], np.float64).view(np.uint64),
                               np.asarray(want[2], np.float64).view(np.uint64)))


def predict_cases():
    """The gating-prediction fixture (predict_golden.npz, made by tests/golden/make_golden_mapmatch.py)."""
    z = np.load(os.path.join(GOLDEN, "predict_golden.npz"))
    out = {}
    for n in z["names"]:
        n = str(n)
        out[n] = {k.split("__", 1)[1]: z[k] for k in z.files if k.startswith(n + "__")}
    return out


PREDICT_ARGS = ("Rwb_t", "pwb_t", "Rbc", "pbc", "Rwc_h", "pwc_h", "lmp", "Spose", "Sl", "sig_px", "fx", "fy", "cx",
                "cy", "W", "H")


def predict_args(c):
    """The positional inputs of predict_projection from a fixture case (scalars as Python floats)."""
    return [float(c[k]) if np.ndim(c[k]) == 0 else c[k] for k in PREDICT_ARGS]
