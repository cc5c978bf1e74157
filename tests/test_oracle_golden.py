"""The CPU oracle against the golden fixtures: outputs of the reference's own
CUDA kernels (compiled from the reference sources) on committed inputs,
generated by tests/golden/make_golden.py.  This pins the oracle before it is
trusted as the checker of the sm_100a kernels."""
import numpy as np
import pytest

from helpers import assert_close, assert_equal, golden, golden_names
from oracle import oracle as orc

REPROJECT = golden_names("reproject_")
TEMPORAL = golden_names("temporal_")
REGRESSION = golden_names("regression_")
FILTER = golden_names("spatial_filter_")


def test_fixtures_present():
    assert len(REPROJECT) == 4 and len(TEMPORAL) == 2 and len(REGRESSION) == 3 and len(FILTER) == 2


def _reproject(g, mode=None):
    lists = [g[k] for k in sorted(k for k in g if k.startswith("in_list"))]
    return orc.reproject(g["in_mvec"], lists, g["in_linear_z"], g["in_prev_linear_z"], g["in_normal"],
                         g["in_prev_normal"], g["in_pn_fwidth"], g["in_opacity"], g["in_prev_opacity"],
                         mode=mode)


@pytest.mark.parametrize("name", REPROJECT)
def test_reproject_matches_reference(name):
    g = golden(name)
    succ, outs = _reproject(g)
    assert_equal(succ, g["ref_success"], f"{name} success")
    for i, o in enumerate(outs):
        assert_close(o, g[f"ref_out{i}"], f"{name} out{i}", atol=1e-6)


@pytest.mark.parametrize("name,flip", [("reproject_border", orc.RP_FMA_IPOS),
                                       ("reproject_weightsum", orc.RP_FMA_SUMW),
                                       ("reproject_normal", 2 << orc.RP_DOT_SHIFT),
                                       ("reproject_normal", 3 << orc.RP_DOT_SHIFT)])
def test_reproject_fixture_pins_rounding(name, flip):
    """Each rounding-boundary fixture rejects the alternative rounding: under
    the other hypothesis the oracle's mask no longer matches the reference."""
    g = golden(name)
    alt = orc.RP_MODE ^ flip
    succ, _ = _reproject(g, mode=alt)
    assert (succ != g["ref_success"]).sum() > 50


@pytest.mark.parametrize("name", TEMPORAL)
def test_temporal_matches_reference(name):
    g = golden(name)
    ero = orc.erode3x3(g["in_reproj_mask"])
    assert_equal(ero, g["in_reproj_success"], f"{name} erosion")
    o = orc.temporal_screening(g["in_current1"], g["in_current2"], g["in_prev"], g["in_prev1"],
                               g["in_prev2"], g["in_reproj_success"], int(g["attr_win_curr"]),
                               int(g["attr_win_prev"]))
    for out, key in zip(o, ("ref_output", "ref_output1", "ref_output2", "ref_success")):
        assert_equal(out, g[key], f"{name} {key}")


@pytest.mark.parametrize("name", REGRESSION)
def test_regression_matches_reference(name):
    g = golden(name)
    o = orc.cross_regression(g["in_imga"], g["in_imgb"], g["in_albedo"], g["in_normal"],
                             int(g["attr_win_size"]), int(g["attr_sparsity"]), int(g["attr_recon_scale"]))
    assert_close(o[0], g["ref_outa"], f"{name} outa", atol=1e-5)
    assert_close(o[1], g["ref_outb"], f"{name} outb", atol=1e-5)
    assert_close(o[2], g["ref_vara"], f"{name} vara", atol=1e-6)
    assert_close(o[3], g["ref_varb"], f"{name} varb", atol=1e-6)


@pytest.mark.parametrize("name", FILTER)
def test_spatial_filter_matches_reference(name):
    g = golden(name)
    win = int(g["attr_win_size"])
    o = orc.spatial_filter(g["in_imga"], g["in_imgb"], g["in_albedo"], g["in_normal"], g["in_band"], win,
                           partials=True)
    for out, key in zip(o[:4], ("ref_acca", "ref_accb", "ref_wgtsuma", "ref_wgtsumb")):
        assert_close(out, g[key], f"{name} {key}", atol=1e-5)
    gb = orc.spatial_filter_grad_from_partials(g["in_grad_acca"], g["in_grad_accb"], g["in_grad_wgtsuma"],
                                               g["in_grad_wgtsumb"], o[4], o[5])
    scale = np.abs(g["ref_grad_band"]).max()
    assert_close(gb, g["ref_grad_band"], f"{name} grad_band", atol=1e-6 * scale)
