"""Host-side distribution set-up of libtmx.so against the reference.

These entry points run on the host (no GPU needed): orientation distribution
coefficients (random, Mishchenko, Davis-Greenstein, custom), Draine-Hensley
shape nodes/weights/limits and R_V/R_S. The fixtures come from the
unmodified reference (tests/golden/make_golden.py)."""
import math
import os

import numpy as np
import pytest

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def stages():
    return np.load(os.path.join(G, "stages.npz"))


@pytest.fixture(scope="module")
def CT():
    from costuum_b200 import build
    build.build()
    from costuum_b200 import CosTuuM
    return CosTuuM


def test_orientation_coefficients(stages, CT):
    for i, cls in ((0, lambda: CT.RandomOrientationDistribution(20)),
                   (1, lambda: CT.MishchenkoOrientationDistribution(0.6, 20)),
                   (2, lambda: CT.DavisGreensteinOrientationDistribution(2.0, 20)),
                   (3, lambda: CT.DavisGreensteinOrientationDistribution(0.5, 20))):
        assert np.array_equal(cls().coefficients, stages["od_%d" % i]), i
    # order 200: the quadratures run on several host threads
    assert np.array_equal(CT.RandomOrientationDistribution(200).coefficients,
                          stages["od_random_200"])


def test_custom_orientation(stages, CT):
    # math.cos is the C library's cosine, the one the reference's C++ calls
    # (numpy's vectorised cosine can differ by an ulp)
    od = CT.CustomOrientationDistribution(
        lambda b: 0.5 + 0.3 * math.cos(b) * math.cos(b), 40)
    assert np.array_equal(od.coefficients, stages["od_custom"])
    od2 = CT.CustomOrientationDistribution(
        lambda b, a: a[0] + a[1] * math.cos(b) * math.cos(b), 40,
        additional_arguments=(0.5, 0.3))
    assert np.array_equal(od2.coefficients, stages["od_custom"])


def test_draine_hensley(stages, CT):
    for i in range(3):
        n, cut, frac = stages["dh_%d_arg" % i]
        sd = CT.DraineHensleyShapeDistribution(int(n), cut, frac)
        ref = stages["dh_%d" % i]
        n = int(n)
        assert np.array_equal(sd.shapes, ref[:n]), i
        assert np.array_equal(sd.weights, ref[n:2 * n]), i
        assert sd.get_limits() == (ref[2 * n], ref[2 * n + 1])


def test_equal_volume_radius(stages, CT):
    for d, v in zip((0.5, 2.0, 1.0, 3.3), stages["rvrs"]):
        assert CT.get_equal_volume_radius(1.0, d) == v


def test_size_based_alignment_selection(CT):
    sb = CT.SizeBasedAlignmentDistribution(1e-7, CT.MISHCHENKO_ALIGNMENT, 10)
    assert sb.get_distribution(5e-8, 2.0) is sb.non_aligned
    assert sb.get_distribution(2e-7, 2.0) is sb.oblate
    assert sb.get_distribution(2e-7, 0.5) is sb.prolate
    assert sb.get_distribution(2e-7, 1.0) is sb.prolate  # d > 1 is oblate
    assert sb.oblate.coefficients[2] == 1.5 * 0.6 - 0.5
    with pytest.raises(ValueError):
        CT.SizeBasedAlignmentDistribution(1e-7, 7)


def test_custom_dust_properties(CT):
    dp = CT.CustomDustProperties(lambda w, s, t: complex(w, s + t))
    assert dp.get_refractive_index(2, 3.0, 1.0) == complex(1.0, 5.0)
    with pytest.raises(TypeError):
        CT.CustomDustProperties(lambda w, s, t: 1.5).get_refractive_index(0, 1, 1)
