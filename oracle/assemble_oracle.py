"""CPU restatement of the window Problem assembly (test infrastructure only: the checker of the device assembly).

The reference's P1Engine._problem (src/xclean/vio/engine_live.py:407-530), visual part: the alive landmarks (in id
order, optionally filtered by a selection), the slots' observations of them sorted stably by landmark, each
landmark's host slot, the inverse-depth prior of the "prior" stereo mode (sigma = max(kappa_d x LK sigma, span) / fB,
weight 1 / sigma where finite and positive and the measurement positive; zero in the "ur" mode) and the per-row
whitening (1 / sigma_px on left rows, 1 / max(kappa_d x the row's sigma, 1e-9) on right rows).  No marginal prior,
no IMU, no pose-free split (the batched solve carries pose-free landmarks as ordinary ones).

Inputs are the engine state in flat form: the slots' observation lists concatenated in slot order (lid, uv, cam,
valid, sig, with slot_n observations per slot), the slots' sids, and the landmark arrays indexed by landmark id.
"""
from __future__ import annotations

import numpy as np


def assemble(slot_n, sids, lid, uv, cam, valid, sig, lm_alive, n_lm, lm_host, lm_p, lm_rho_meas, lm_sig_lk, lm_span,
             prior_mode, kappa_d, fB, sig_px, select=None):
    """-> dict(alive, lmp, lm_host, lm_mask, rho_meas, rho_isig, ob_start, ob_pose, ob_cam, ob_z, ob_isig, ob_valid,
    src): the Problem's visual arrays and the (slot, index) of every observation."""
    slot_n = np.asarray(slot_n, np.int64)
    P = len(slot_n)
    alive = np.nonzero(np.asarray(lm_alive)[:n_lm])[0]
    if select is not None:
        alive = alive[np.asarray(select)[alive]]
    L = len(alive)
    loc = np.full(n_lm, -1, np.int64)
    loc[alive] = np.arange(L)
    pose = np.repeat(np.arange(P, dtype=np.int64), slot_n)
    within = np.concatenate([np.arange(n, dtype=np.int64) for n in slot_n]) if P else np.zeros(0, np.int64)
    lid = np.asarray(lid, np.int64)
    local = loc[lid] if len(lid) else np.zeros(0, np.int64)
    keep = local >= 0
    order = np.argsort(local[keep], kind="stable")
    idx = np.nonzero(keep)[0][order]
    local = local[idx]
    ob_start = np.zeros(L + 1, np.int64)
    if L:
        np.cumsum(np.bincount(local, minlength=L), out=ob_start[1:])
    sid2i = {int(s): i for i, s in enumerate(sids)}
    host = np.array([sid2i[int(h)] for h in np.asarray(lm_host)[alive]], np.int64)
    if prior_mode:
        rm = np.asarray(lm_rho_meas, np.float64)[alive]
        sg = np.maximum(kappa_d * np.asarray(lm_sig_lk, np.float64)[alive], np.asarray(lm_span, np.float64)[alive]) / fB
        ris = np.where(np.isfinite(sg) & (sg > 0) & (rm > 0), 1.0 / np.where(sg > 0, sg, 1.0), 0.0)
    else:
        rm = np.zeros(L)
        ris = np.zeros(L)
    cam = np.asarray(cam, np.int64)[idx]
    sg_ob = np.asarray(sig, np.float64)[idx]
    return dict(alive=alive, lmp=np.asarray(lm_p, np.float64)[alive], lm_host=host, lm_mask=np.ones(L, np.bool_),
                rho_meas=rm, rho_isig=ris, ob_start=ob_start, ob_pose=pose[idx], ob_cam=cam,
                ob_z=np.asarray(uv, np.float64).reshape(-1, 2)[idx],
                ob_isig=np.where(cam == 0, 1.0 / sig_px, 1.0 / np.maximum(kappa_d * sg_ob, 1e-9)),
                ob_valid=np.asarray(valid, np.bool_)[idx], src=np.stack([pose[idx], within[idx]], axis=1))
