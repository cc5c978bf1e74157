"""Reprojection inputs that sit on the rounding boundaries of the success mask.

The reprojection mask depends on float expressions whose last bit decides
it: the rounded previous position (screen-border test), the normal distance
ratio against 4, and the bilinear weight sum against 0.01
(ops/reproject.cu.cc:38-47, 97, 158).  A GPU compiler may evaluate some of
them with fused multiply-adds.  Each builder below draws candidates near one
boundary, runs the CPU oracle under every rounding hypothesis and keeps the
pixels whose mask differs between hypotheses, so that the reference kernel's
own output on these inputs pins which hypothesis it follows.

Builders return a dict of NHWC float32 numpy arrays named like the Reproject
op arguments plus ``inputs`` (the reprojected list).
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as orc


def _base(B, H, W, rng):
    # flat depth and one normal everywhere: depth and normal tests pass for
    # every tap, so only the boundary under study decides the mask
    z = np.full((B, H, W, 1), 10.0, np.float32)
    lin = np.concatenate([z, np.full_like(z, 0.5), np.zeros_like(z)], -1)
    n = np.broadcast_to(np.array([0.0, 0.6, 0.8], np.float32), (B, H, W, 3)).copy()
    d = dict(
        mvec=np.zeros((B, H, W, 3), np.float32),
        linear_z=lin, prev_linear_z=lin.copy(),
        normal=n.astype(np.float32), prev_normal=n.astype(np.float32).copy(),
        pn_fwidth=np.zeros((B, H, W, 3), np.float32),
        opacity=np.ones((B, H, W, 1), np.float32),
        prev_opacity=np.ones((B, H, W, 1), np.float32),
        inputs=[rng.uniform(0, 1, (B, H, W, 3)).astype(np.float32),
                rng.uniform(0, 1, (B, H, W, 3)).astype(np.float32),
                rng.uniform(0, 1, (B, H, W, 2)).astype(np.float32)],
    )
    return d


def _run(d, mode):
    s, _ = orc.reproject(d["mvec"], d["inputs"], d["linear_z"], d["prev_linear_z"], d["normal"],
                         d["prev_normal"], d["pn_fwidth"], d["opacity"], d["prev_opacity"], mode=mode)
    return s


def _keep_disagreeing(d, modes, propose, rounds=40):
    """Redraw per-pixel proposals until the mask differs between `modes`."""
    B, H, W, _ = d["mvec"].shape
    done = np.zeros((B, H, W), bool)
    for _ in range(rounds):
        propose(d, ~done)
        masks = [_run(d, m)[..., 0] for m in modes]
        differ = np.zeros_like(done)
        for m in masks[1:]:
            differ |= m != masks[0]
        done |= differ
    return d, done


def border_case(seed=0, H=80, W=96, rounds=60):
    """Rounded previous positions int(pos + mvec*dim + 0.5)
    (ops/reproject.cu.cc:97) within an ulp of a half-pixel boundary.

    Previous opacity is 1 only on columns c = 2 (mod 4) and every pixel is
    sent near x = k + 0.5 with k = 0 (mod 4): the bilinear taps k, k+1 are
    invalid, so the 3x3 fallback decides, and its box contains the valid
    column k+2 only when the rounded position is k+1.  The mask therefore
    reads the rounding of pos + mvec*dim directly.  W = 96 makes mvec*dim
    inexact (x3)."""
    rng = np.random.default_rng(seed)
    d = _base(1, H, W, rng)
    d["prev_opacity"][:] = 0.0
    d["prev_opacity"][:, :, 2::4] = 1.0
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float32)

    def propose(d, todo):
        k = 4 * rng.integers(1, W // 4 - 2, (H, W))
        ty = rng.integers(2, H - 3, (H, W)) + 0.25
        mx = ((k + 0.5 - xs) / W).astype(np.float32)
        steps = rng.integers(-3, 4, (H, W))
        for st in range(3):
            mx = np.where(steps > st, np.nextafter(mx, np.float32(np.inf)), mx)
            mx = np.where(steps < -st, np.nextafter(mx, np.float32(-np.inf)), mx)
        my = ((ty - ys) / H).astype(np.float32)
        sel = todo[0]
        d["mvec"][0, ..., 0][sel] = mx[sel]
        d["mvec"][0, ..., 1][sel] = my[sel]

    base = orc.RP_MODE
    return _keep_disagreeing(d, [base, base ^ orc.RP_FMA_IPOS], propose, rounds=rounds)


def normal_case(seed=1, H=48, W=48):
    """Normal distances whose ratio to (fwidth + 1e-2) sits on 4 within an ulp
    (ops/reproject.cu.cc:46), for every contraction of the dot product."""
    rng = np.random.default_rng(seed)
    d = _base(1, H, W, rng)
    npv = np.array([0.3, -0.5, 0.81], np.float32)
    npv /= np.linalg.norm(npv)
    d["prev_normal"][:] = npv

    def propose(d, todo):
        v = rng.normal(size=(H, W, 3)).astype(np.float32)
        v /= np.linalg.norm(v, axis=-1, keepdims=True)
        mag = rng.uniform(0.05, 1.5, (H, W, 1)).astype(np.float32)
        n = (npv + v * mag).astype(np.float32)
        dvec = (n - npv).astype(np.float32)
        dist = np.sqrt(np.sum(dvec.astype(np.float64) ** 2, -1))
        fw = (dist / 4.0 - 1e-2).astype(np.float32)
        steps = rng.integers(-3, 4, (H, W))
        for k in range(3):
            fw = np.where(steps > k, np.nextafter(fw, np.float32(np.inf)), fw)
            fw = np.where(steps < -k, np.nextafter(fw, np.float32(-np.inf)), fw)
        fw = np.maximum(fw, 0).astype(np.float32)
        sel = todo[0]
        d["normal"][0][sel] = n[sel]
        d["pn_fwidth"][0, ..., 1][sel] = fw[sel]

    base = orc.RP_MODE & ~(3 << orc.RP_DOT_SHIFT)
    modes = [base | (m << orc.RP_DOT_SHIFT) for m in range(4)]
    return _keep_disagreeing(d, modes, propose)


def weightsum_case(seed=2, H=64, W=64, rounds=30, candidates=512):
    """Bilinear weight sums on the 0.01 threshold (ops/reproject.cu.cc:158).

    Batch 1 carries the test.  Its previous opacity is 0 on pixels with both
    coordinates even; every pixel is sent to (lx + x, ly + y) with (lx, ly)
    an even-even pixel next to it, so the top-left tap is invalid and the
    other three taps weigh x(1-y) + (1-x)y + xy = x + y - xy.  x and y are
    chosen on the float32 grid of the previous position so that this sum,
    evaluated exactly, lies within a few 1e-9 of 0.01f.  W = H = 64 keeps
    mvec * dim exact, so only the weight-sum rounding differs between
    hypotheses.  Batch 0's previous opacity is all 0; the reference's 3x3
    fallback reads previous opacity without the batch offset
    (ops/reproject.cu.cc:191), so in batch 1 the fallback never succeeds and
    the mask is exactly (sum >= 0.01)."""
    rng = np.random.default_rng(seed)
    d = _base(2, H, W, rng)
    d["prev_opacity"][0] = 0.0
    d["prev_opacity"][1, 0::2, 0::2] = 0.0
    ys, xs = np.mgrid[0:H, 0:W]
    lx = np.clip(xs - xs % 2, 2, W - 4).astype(np.float64)
    ly = np.clip(ys - ys % 2, 2, H - 4).astype(np.float64)
    qx = np.spacing((lx + 0.5).astype(np.float32)).astype(np.float64)[..., None]
    qy = np.spacing((ly + 0.5).astype(np.float32)).astype(np.float64)[..., None]
    target = float(np.float32(0.01))

    def propose(d, todo):
        x = qx * rng.integers(1, np.maximum(2, (0.009 / qx).astype(np.int64)),
                              (H, W, candidates))
        y = np.round((target - x) / (1.0 - x) / qy) * qy
        resid = np.abs(x + y - x * y - target)
        best = resid.argmin(-1)[..., None]
        xb = np.take_along_axis(x, best, -1)[..., 0]
        yb = np.take_along_axis(y, best, -1)[..., 0]
        mx = ((lx + xb - xs) / W).astype(np.float32)
        my = ((ly + yb - ys) / H).astype(np.float32)
        sel = todo[1]
        d["mvec"][1, ..., 0][sel] = mx[sel]
        d["mvec"][1, ..., 1][sel] = my[sel]

    base = orc.RP_MODE
    return _keep_disagreeing(d, [base, base ^ orc.RP_FMA_SUMW], propose, rounds=rounds)
