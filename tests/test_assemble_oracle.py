"""The Problem-assembly oracle (oracle/assemble_oracle.py) against the reference's own P1Engine._problem outputs
(tests/golden/assemble_golden.npz, made by tests/golden/make_golden_assemble.py).  Bit-exact: gathers, a stable sort
and the float64 weights in the reference's operation order."""
import os

import numpy as np
import pytest

from oracle import assemble_oracle as AO

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "assemble_golden.npz")
CASES = (0, 1, 2)


def case_inputs(z, c):
    p = "c%d_" % c
    kappa_d, fB, sig_px = (float(x) for x in z[p + "consts"])
    return dict(slot_n=z[p + "slot_n"], sids=z[p + "sids"], lid=z[p + "slot_lid"], uv=z[p + "slot_uv"],
                cam=z[p + "slot_cam"], valid=z[p + "slot_valid"], sig=z[p + "slot_sig"], lm_alive=z[p + "lm_alive"],
                n_lm=int(z[p + "n_lm"][0]), lm_host=z[p + "lm_host"], lm_p=z[p + "lm_p"],
                lm_rho_meas=z[p + "lm_rho_meas"], lm_sig_lk=z[p + "lm_sig_lk"], lm_span=z[p + "lm_span"],
                prior_mode=bool(z[p + "mode"][0]), kappa_d=kappa_d, fB=fB, sig_px=sig_px,
                select=z[p + "select"] if (p + "select") in z.files else None)


@pytest.fixture(scope="module")
def z():
    return np.load(GOLD)


@pytest.mark.parametrize("c", CASES)
def test_oracle_is_bit_exact(z, c):
    got = AO.assemble(**case_inputs(z, c))
    p = "c%d_" % c
    assert np.array_equal(got["alive"], z[p + "alive"])
    assert np.array_equal(got["src"], z[p + "src"])
    for k in ("lmp", "lm_host", "lm_mask", "rho_meas", "rho_isig", "ob_start", "ob_pose", "ob_cam", "ob_z", "ob_isig",
              "ob_valid"):
        a, b = np.asarray(got[k]), np.asarray(z[p + "pb_" + k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), np.ascontiguousarray(b).view(np.uint8)) if a.dtype == b.dtype \
            else np.array_equal(a, b), k
