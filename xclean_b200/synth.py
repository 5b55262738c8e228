"""Seeded synthetic stereo scenes (stand-ins for the datasets the reference is run on, which are not available here).

Textured planes rendered by ray-plane intersection (no graphics API: plain tensor arithmetic on the CPU or the GPU),
rectified pinhole stereo, Gaussian sensor noise, uint8 output.

  scene_planes(seed, ...)           N random planes at depths [z0, z1] plus a background plane (the small-frame case)
  scene_road(seed, length)          a driving corridor: road, two facades, roadside boards, a far backdrop
  render_pair(scene, cam, pose)     -> (left, right) uint8 (H, W)
  sequence(...)                     a forward-driving sequence of stereo pairs, [F, H, W] uint8 tensors
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class Camera:
    W: int
    H: int
    fx: float
    fy: float
    cx: float
    cy: float
    baseline: float


CAM_SMALL = Camera(752, 480, 458.0, 458.0, 367.0, 248.0, 0.11)        # 752x480, disparities 0-64 at 2 m +
CAM_KITTI = Camera(1241, 376, 718.0, 718.0, 607.0, 185.0, 0.54)       # 1241x376, disparities 0-96
CAM_HD = Camera(1280, 720, 640.0, 640.0, 640.0, 360.0, 0.075)         # 1280x720, disparities 0-128


def fractal_texture(seed, n=1024, beta=1.0):
    """1/f^beta noise (FFT-shaped), normalised to [0, 1]."""
    rng = np.random.default_rng(seed)
    fy = np.fft.fftfreq(n)[:, None]
    fx = np.fft.rfftfreq(n)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    spec = (rng.normal(size=f.shape) + 1j * rng.normal(size=f.shape)) / f ** beta
    spec[0, 0] = 0.0
    t = np.fft.irfftn(spec, s=(n, n), axes=(0, 1))
    t = (t - t.min()) / max(t.max() - t.min(), 1e-12)
    return t.astype(np.float32)


@dataclass
class Scene:
    centers: np.ndarray          # (P, 3)
    axes_u: np.ndarray           # (P, 3)
    axes_v: np.ndarray           # (P, 3)
    half: np.ndarray             # (P, 2) half extents (m)
    tex_id: np.ndarray           # (P,)
    tex_scale: np.ndarray        # (P,) texels per metre
    tex_off: np.ndarray          # (P, 2)
    gain: np.ndarray             # (P,) brightness
    textures: np.ndarray = field(repr=False)   # (K, n, n)


def _rot(ax, ay, az):
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def scene_planes(seed, cam, n_planes=6, z0=2.0, z1=15.0, n_tex=4):
    """n_planes - 1 random tilted planes at depths U(z0, z1) in the view, and a background plane behind them."""
    rng = np.random.default_rng(seed)
    tex = np.stack([fractal_texture(seed * 131 + k) for k in range(n_tex)])
    C, U, V, Hx, T, S, O, G = [], [], [], [], [], [], [], []
    C.append([0.0, 0.0, z1 + 1.0]); U.append([1.0, 0, 0]); V.append([0, 1.0, 0]); Hx.append([1e3, 1e3])
    for _ in range(n_planes - 1):
        z = rng.uniform(z0, z1)
        x = rng.uniform(-0.4, 0.4) * z * cam.W / cam.fx
        y = rng.uniform(-0.4, 0.4) * z * cam.H / cam.fy
        R = _rot(rng.uniform(-0.5, 0.5), rng.uniform(-0.5, 0.5), rng.uniform(-0.3, 0.3))
        C.append([x, y, z]); U.append(R[:, 0]); V.append(R[:, 1])
        Hx.append([rng.uniform(0.15, 0.45) * z * cam.W / cam.fx, rng.uniform(0.15, 0.45) * z * cam.H / cam.fy])
    P = len(C)
    for _ in range(P):
        T.append(rng.integers(0, n_tex)); S.append(rng.uniform(60.0, 200.0)); O.append(rng.uniform(0, 1024, 2))
        G.append(rng.uniform(0.55, 1.0))
    return Scene(np.array(C, float), np.array(U, float), np.array(V, float), np.array(Hx, float), np.array(T),
                 np.array(S), np.array(O), np.array(G), tex)


def scene_road(seed, length=600.0, n_tex=6):
    """A driving corridor along +z: road (y = 1.65), facades at x = -7.5 and +8.5, boards every ~12 m, backdrop."""
    rng = np.random.default_rng(seed)
    tex = np.stack([fractal_texture(seed * 131 + k) for k in range(n_tex)])
    C, U, V, Hx = [], [], [], []
    ex, ey, ez = np.array([1.0, 0, 0]), np.array([0, 1.0, 0]), np.array([0, 0, 1.0])
    C.append([0, 1.65, length / 2]); U.append(ex); V.append(ez); Hx.append([20.0, length])          # road
    C.append([-7.5, -2.0, length / 2]); U.append(ez); V.append(ey); Hx.append([length, 6.0])       # left facade
    C.append([8.5, -2.0, length / 2]); U.append(ez); V.append(ey); Hx.append([length, 6.0])        # right facade
    C.append([0, -3.0, length + 50]); U.append(ex); V.append(ey); Hx.append([1e3, 1e3])           # backdrop
    z = 6.0
    while z < length:
        side = rng.choice([-1.0, 1.0])
        x = side * rng.uniform(2.5, 6.0)
        R = _rot(0.0, rng.uniform(-0.6, 0.6), 0.0)
        C.append([x, rng.uniform(-1.0, 0.8), z]); U.append(R[:, 0]); V.append(R[:, 1])
        Hx.append([rng.uniform(0.6, 1.8), rng.uniform(0.6, 1.6)])
        z += rng.uniform(6.0, 18.0)
    P = len(C)
    T = rng.integers(0, n_tex, P)
    S = rng.uniform(40.0, 160.0, P)
    O = rng.uniform(0, 1024, (P, 2))
    G = rng.uniform(0.55, 1.0, P)
    return Scene(np.array(C, float), np.array(U, float), np.array(V, float), np.array(Hx, float), T, S, O, G, tex)


class Renderer:
    """Holds a scene on a device and renders grey images for camera poses (R_wc, t_wc) of the LEFT camera."""

    def __init__(self, scene, cam, device="cpu"):
        self.cam = cam
        self.dev = torch.device(device)
        d = dict(dtype=torch.float32, device=self.dev)
        self.C = torch.tensor(scene.centers, **d)
        self.U = torch.tensor(scene.axes_u, **d)
        self.V = torch.tensor(scene.axes_v, **d)
        self.N = torch.cross(self.U, self.V, dim=1)
        self.half = torch.tensor(scene.half, **d)
        self.tid = torch.tensor(scene.tex_id, dtype=torch.long, device=self.dev)
        self.tscale = torch.tensor(scene.tex_scale, **d)
        self.toff = torch.tensor(scene.tex_off, **d)
        self.gain = torch.tensor(scene.gain, **d)
        self.tex = torch.tensor(scene.textures, **d)
        v, u = torch.meshgrid(torch.arange(cam.H, **d), torch.arange(cam.W, **d), indexing="ij")
        self.rays = torch.stack([(u - cam.cx) / cam.fx, (v - cam.cy) / cam.fy, torch.ones_like(u)], -1).reshape(-1, 3)

    def _visible(self, R, t, max_depth=250.0):
        """planes not entirely behind the camera nor (small ones) beyond max_depth"""
        Cn = self.C.cpu().numpy()
        rad = np.linalg.norm(self.half.cpu().numpy(), axis=1)
        fwd = R[:, 2].cpu().numpy()
        dz = (Cn - t.cpu().numpy()) @ fwd
        return [p for p in range(len(Cn)) if dz[p] + rad[p] > 0.2 and (dz[p] - rad[p] < max_depth or rad[p] > 100)]

    def _render(self, R, t, gen, noise):
        d = (self.rays @ R.T)                                     # world directions (z-depth parametrised)
        best = torch.full((d.shape[0],), float("inf"), device=self.dev)
        val = torch.zeros(d.shape[0], device=self.dev)
        n_tex = self.tex.shape[-1]
        for p in self._visible(R, t):
            n = self.N[p]
            den = d @ n
            tt = ((self.C[p] - t) @ n) / torch.where(den.abs() < 1e-9, torch.full_like(den, 1e-9), den)
            hit = t + tt[:, None] * d
            rel = hit - self.C[p]
            s1, s2 = rel @ self.U[p], rel @ self.V[p]
            ok = (tt > 0.2) & (s1.abs() <= self.half[p, 0]) & (s2.abs() <= self.half[p, 1]) & (tt < best)
            if not bool(ok.any()):
                continue
            tx = torch.remainder(s1 * self.tscale[p] + self.toff[p, 0], n_tex - 1)
            ty = torch.remainder(s2 * self.tscale[p] + self.toff[p, 1], n_tex - 1)
            x0, y0 = tx.floor().long().clamp(0, n_tex - 2), ty.floor().long().clamp(0, n_tex - 2)
            ax, ay = tx - x0, ty - y0
            T = self.tex[self.tid[p]]
            a = T[y0, x0]; b = T[y0, x0 + 1]; c = T[y0 + 1, x0]; e = T[y0 + 1, x0 + 1]
            g = (a + ax * (b - a)) * (1 - ay) + (c + ax * (e - c)) * ay
            g = 20.0 + 215.0 * g * self.gain[p]
            best = torch.where(ok, tt, best)
            val = torch.where(ok, g, val)
        if noise > 0:
            val = val + noise * torch.randn(val.shape, generator=gen, device=self.dev)
        img = torch.clamp(torch.round(val), 0, 255).to(torch.uint8).reshape(self.cam.H, self.cam.W)
        return img

    def pair(self, R_wc, t_wc, seed=0, noise=2.0):
        """-> (left, right) uint8 tensors for the left camera pose (R_wc (3,3), t_wc (3,))."""
        R = torch.as_tensor(np.asarray(R_wc), dtype=torch.float32, device=self.dev)
        t = torch.as_tensor(np.asarray(t_wc), dtype=torch.float32, device=self.dev)
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(int(seed))
        left = self._render(R, t, gen, noise)
        right = self._render(R, t + R[:, 0] * self.cam.baseline, gen, noise)
        return left, right


def yaw(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def sequence(cam, n_frames, seed=0, device="cpu", step=1.0, yaw_sigma_deg=0.5, noise=2.0, scene=None):
    """A forward-driving stereo sequence (step metres per frame, yaw noise): -> (left [F,H,W], right [F,H,W])."""
    scene = scene if scene is not None else scene_road(seed, length=step * n_frames + 120.0)
    rd = Renderer(scene, cam, device)
    rng = np.random.default_rng(seed + 7)
    L = torch.empty((n_frames, cam.H, cam.W), dtype=torch.uint8, device=rd.dev)
    R = torch.empty_like(L)
    for k in range(n_frames):
        Rw = yaw(math.radians(rng.normal(0.0, yaw_sigma_deg)))
        l, r = rd.pair(Rw, np.array([0.0, 0.0, step * k]), seed=seed * 100003 + k, noise=noise)
        L[k] = l
        R[k] = r
    return L, R


def map_landmarks(kp, counts, desc, m0, m1, nmatch, n_lm=1500, D=3, seed=0):
    """Map-matching inputs for a frame sequence (the frontend's per-frame outputs): frame f's landmarks are the first
    n_lm keypoints of frame f-1 (frame 0 takes the last frame's), predicted where frame f's matches put them (+0.7 px
    noise) or, unmatched, at their old position shifted by the median flow (+3 px noise); innovation covariances with
    sigmas in [0.8, 4] px and correlation in [-0.5, 0.5]; D descriptor slots (the keypoint's own, a copy with ~4 % of
    the bits flipped, a random one) of which 1..D are valid.
    -> uv (F,n_lm,2) float64, S (F,n_lm,2,2) float64, lm_desc (F,n_lm,D,32) uint8, lm_ndesc (F,n_lm) int64,
    nlm (F,) int32."""
    F = len(counts)
    rng = np.random.default_rng(seed)
    uv = np.zeros((F, n_lm, 2))
    S = np.zeros((F, n_lm, 2, 2))
    lmd = np.zeros((F, n_lm, D, 32), np.uint8)
    lnd = np.zeros((F, n_lm), np.int64)
    nlm = np.zeros(F, np.int32)
    for f in range(F):
        p = (f - 1) % F
        L = min(int(counts[p]), n_lm)
        nlm[f] = L
        q, t = m0[f, :int(nmatch[f])], m1[f, :int(nmatch[f])]
        keep = q < L
        q, t = q[keep], t[keep]
        base = kp[p, :L].astype(np.float64)
        flow = np.median(kp[f, t].astype(np.float64) - base[q], axis=0) if len(q) else np.zeros(2)
        u = base + flow + rng.normal(0, 3.0, (L, 2))
        u[q] = kp[f, t].astype(np.float64) + rng.normal(0, 0.7, (len(q), 2))
        uv[f, :L] = u
        sx, sy, rho = rng.uniform(0.8, 4.0, L), rng.uniform(0.8, 4.0, L), rng.uniform(-0.5, 0.5, L)
        S[f, :L, 0, 0] = sx * sx
        S[f, :L, 1, 1] = sy * sy
        S[f, :L, 0, 1] = S[f, :L, 1, 0] = rho * sx * sy
        lmd[f, :L, 0] = desc[p, :L]
        if D > 1:
            flips = np.packbits(rng.random((L, 256)) < 0.04, axis=1)
            lmd[f, :L, 1] = desc[p, :L] ^ flips
        if D > 2:
            lmd[f, :L, 2:] = rng.integers(0, 256, (L, D - 2, 32), dtype=np.uint8)
        lnd[f, :L] = rng.integers(1, D + 1, L)
    return uv, S, lmd, lnd, nlm


def tracking_window(seed, n_lm=2000, cam=None, n_clutter=400):
    """One tracking step's inputs: a window of n_lm inverse-depth landmarks hosted by 8 keyframes along a forward
    path (camera z = body x), the predicted body pose one metre ahead of the newest keyframe, pose and landmark
    covariances, and the frame's keypoints (the in-view projections with 1 px noise, 70 % of them, plus clutter)
    with descriptors (the landmark's own with ~5 % of the bits flipped).
    -> dict(pose=[Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, sig_px, fx, fy, cx, cy], W, H, kp, desc,
    lm_desc, lm_ndesc); kp are placed from this module's own float64 projection."""
    cam = cam or CAM_KITTI
    rng = np.random.default_rng(seed)
    Rbc = np.array([[0.0, 0.0, 1.0], [-1.0, 0.0, 0.0], [0.0, -1.0, 0.0]])
    pbc = np.array([0.3, -0.1, 0.05])
    nh = 8
    def rz(a):                                          # body yaw (z up)
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])

    yaw_h = [rz(rng.normal(0, 0.01)) for _ in range(nh)]
    pwb_h = [np.array([1.0 * i, rng.normal(0, 0.05), 0.0]) for i in range(nh)]
    host = rng.integers(0, nh, n_lm)
    Rwc_h = np.stack([yaw_h[h] @ Rbc for h in host])
    pwc_h = np.stack([pwb_h[h] + yaw_h[h] @ pbc for h in host])
    lmp = np.stack([rng.uniform(-0.6, 0.6, n_lm), rng.uniform(-0.2, 0.2, n_lm), rng.uniform(0.03, 0.3, n_lm)], 1)
    Rwb_t = yaw_h[-1]
    pwb_t = pwb_h[-1] + np.array([1.0, 0.0, 0.0])
    A = rng.normal(0, 0.002, (6, 6))
    Spose = A @ A.T
    B = rng.normal(0, 0.002, (n_lm, 3, 3))
    Sl = np.einsum("lij,lkj->lik", B, B)
    fx, fy, cx, cy = cam.fx, cam.fy, cam.cx, cam.cy
    # in-view projections (plain float64 pinhole; the exact values come from predict_projection itself)
    Rwc_t = Rwb_t @ Rbc
    pwc_t = pwb_t + Rwb_t @ pbc
    m = np.stack([lmp[:, 0], lmp[:, 1], np.ones(n_lm)], 1)
    Pw = pwc_h + np.einsum("nij,nj->ni", Rwc_h, m) / lmp[:, 2:3]
    Xc = (Pw - pwc_t) @ Rwc_t
    with np.errstate(all="ignore"):
        u = fx * Xc[:, 0] / Xc[:, 2] + cx
        v = fy * Xc[:, 1] / Xc[:, 2] + cy
    vis = np.nonzero((Xc[:, 2] > 0.1) & (u >= 0) & (u < cam.W) & (v >= 0) & (v < cam.H))[0]
    seen = vis[rng.random(len(vis)) < 0.7]
    lm_desc = rng.integers(0, 256, (n_lm, 3, 32), dtype=np.uint8)
    lm_ndesc = rng.integers(1, 4, n_lm).astype(np.int64)
    kp = np.concatenate([np.stack([u[seen], v[seen]], 1) + rng.normal(0, 1.0, (len(seen), 2)),
                         np.stack([rng.uniform(0, cam.W, n_clutter), rng.uniform(0, cam.H, n_clutter)], 1)])
    flips = np.packbits(rng.random((len(seen), 256)) < 0.05, axis=1)
    desc = np.concatenate([lm_desc[seen, 0] ^ flips, rng.integers(0, 256, (n_clutter, 32), dtype=np.uint8)])
    perm = rng.permutation(len(kp))
    return dict(pose=[Rwb_t, pwb_t, Rbc, pbc, Rwc_h, pwc_h, lmp, Spose, Sl, 1.0, float(fx), float(fy), float(cx),
                      float(cy)], W=cam.W, H=cam.H, kp=kp[perm].astype(np.float32), desc=desc[perm],
                lm_desc=lm_desc, lm_ndesc=lm_ndesc)
