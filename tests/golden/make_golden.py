"""Generate the golden fixtures of tests/golden from the reference's own CUDA
kernels (compiled from the reference sources by oracle/Makefile into
oracle/_ref).  Needs a CUDA GPU; run from the repository root:

    python tests/golden/make_golden.py --out tests/golden

Each fixture is an .npz holding the op inputs (in_*), the attributes (attr_*)
and the reference outputs (ref_*), small enough to commit.  Inputs come from
the seeded synthetic generator and from tests/adversarial.py (reprojection
inputs on the mask's rounding boundaries).
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import __graft_entry__ as ge  # noqa: E402
from oracle import reference as ref  # noqa: E402
import adversarial  # noqa: E402

pkg = ge.load_package()
dev = torch.device("cuda:0")


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def N(t):
    return t.detach().cpu().numpy()


def frames(H, W, seed, motion):
    seq = pkg.synth.make_sequence(H, W, seed=seed, object_motion=motion)
    f0, f1 = seq.frame(4), seq.frame(5)
    return {k: v.numpy() for k, v in f0.items()}, {k: v.numpy() for k, v in f1.items()}


def save(out, name, **arrays):
    path = os.path.join(out, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


def reproject_fixture(out, name, d):
    succ, outs = ref.reproject(T(d["mvec"]), [T(x) for x in d["inputs"]], T(d["linear_z"]),
                               T(d["prev_linear_z"]), T(d["normal"]), T(d["prev_normal"]),
                               T(d["pn_fwidth"]), T(d["opacity"]), T(d["prev_opacity"]))
    torch.cuda.synchronize()
    arrays = {f"in_{k}": v for k, v in d.items() if k != "inputs"}
    for i, x in enumerate(d["inputs"]):
        arrays[f"in_list{i}"] = x
        arrays[f"ref_out{i}"] = N(outs[i])
    arrays["ref_success"] = N(succ)
    save(out, name, **arrays)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if not ref.available():
        raise SystemExit("reference kernels not built (make -C oracle ref)")

    # --- reprojection: rounding-boundary cases and a moving sequence -------
    for name, builder in (("reproject_border", adversarial.border_case),
                          ("reproject_normal", adversarial.normal_case),
                          ("reproject_weightsum", adversarial.weightsum_case)):
        d, _ = builder()
        reproject_fixture(args.out, name, d)
    f0, f1 = frames(48, 64, seed=11, motion=2.0)
    d = dict(mvec=f1["mvec"], linear_z=f1["linearZ"], prev_linear_z=f0["linearZ"],
             normal=f1["normal"], prev_normal=f0["normal"], pn_fwidth=f1["pnFwidth"],
             opacity=f1["opacity"], prev_opacity=f0["opacity"],
             inputs=[np.log1p(f0["color"]), np.log1p(f0["color2"]), f0["albedo"][..., :2].copy()])
    d["opacity"][0, 5:9, 10:20] = 0.0          # exercise the opacity rejections
    d["prev_opacity"][0, 20:24, 30:34] = 0.0
    reproject_fixture(args.out, "reproject_sequence", d)

    # --- temporal screening on the sequence's reprojection -----------------
    succ, outs = ref.reproject(T(d["mvec"]), [T(np.log1p(f0["color"])), T(np.log1p(f0["color2"])),
                                              T(np.log1p(f0["color"]) * 0.5)],
                               T(d["linear_z"]), T(d["prev_linear_z"]), T(d["normal"]),
                               T(d["prev_normal"]), T(d["pn_fwidth"]), T(d["opacity"]),
                               T(d["prev_opacity"]))
    eroded = ref.erode3x3(succ)
    c1, c2 = T(np.log1p(f1["color"])), T(np.log1p(f1["color2"]))
    for wc, wp in ((7, 1), (5, 3)):
        o = ref.temporal_screening(c1, c2, outs[0], outs[1], outs[2], eroded, wc, wp)
        torch.cuda.synchronize()
        save(args.out, f"temporal_w{wc}_{wp}", in_current1=N(c1), in_current2=N(c2),
             in_prev=N(outs[0]), in_prev1=N(outs[1]), in_prev2=N(outs[2]),
             in_reproj_mask=N(succ), in_reproj_success=N(eroded), attr_win_curr=wc, attr_win_prev=wp,
             ref_output=N(o[0]), ref_output1=N(o[1]), ref_output2=N(o[2]), ref_success=N(o[3]))

    # --- cross regression ---------------------------------------------------
    y1, y2 = np.log1p(f1["color"]), np.log1p(f1["color2"])
    for win, sp, rs in ((15, 4, 1), (17, 4, 2), (11, 2, 1)):
        o = ref.cross_regression(T(y1), T(y2), T(f1["albedo"]), T(f1["normal"]), win, sp, rs)
        torch.cuda.synchronize()
        save(args.out, f"regression_w{win}_s{sp}_r{rs}", in_imga=y1, in_imgb=y2,
             in_albedo=f1["albedo"], in_normal=f1["normal"], attr_win_size=win, attr_sparsity=sp,
             attr_recon_scale=rs, ref_outa=N(o[0]), ref_outb=N(o[1]), ref_vara=N(o[2]),
             ref_varb=N(o[3]))

    # --- spatial filter forward + reference gradient ------------------------
    g = torch.Generator().manual_seed(21)
    band = pkg.synth.random_band((1, 48, 64), g).numpy()
    rng = np.random.default_rng(22)
    ga = rng.normal(size=(1, 48, 64, 3)).astype(np.float32)
    gb = rng.normal(size=(1, 48, 64, 3)).astype(np.float32)
    gwa = rng.normal(size=(1, 48, 64, 1)).astype(np.float32)
    gwb = rng.normal(size=(1, 48, 64, 1)).astype(np.float32)
    for win in (11, 7):
        args_in = [T(y1), T(y2), T(f1["albedo"]), T(f1["normal"]), T(band)]
        o = ref.spatial_filter(*args_in, win)
        gband = ref.spatial_filter_grad(T(ga), T(gb), T(gwa), T(gwb), *args_in, win)
        torch.cuda.synchronize()
        save(args.out, f"spatial_filter_w{win}", in_imga=y1, in_imgb=y2, in_albedo=f1["albedo"],
             in_normal=f1["normal"], in_band=band, in_grad_acca=ga, in_grad_accb=gb,
             in_grad_wgtsuma=gwa, in_grad_wgtsumb=gwb, attr_win_size=win,
             ref_acca=N(o[0]), ref_accb=N(o[1]), ref_wgtsuma=N(o[2]), ref_wgtsumb=N(o[3]),
             ref_grad_band=N(gband))


if __name__ == "__main__":
    main()
