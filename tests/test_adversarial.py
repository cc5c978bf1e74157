"""The rounding-boundary reprojection builders produce pixels on which the
rounding hypotheses disagree (the property the golden fixtures rely on)."""
import adversarial as A


def test_builders_discriminate():
    for fn, least in ((A.border_case, 1000), (A.normal_case, 500), (A.weightsum_case, 200)):
        _, done = fn()
        assert done.sum() >= least, fn.__name__
