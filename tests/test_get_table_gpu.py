"""get_table on the GPU against the reference module's own outputs
(tests/golden/tables.npz, made by the unmodified reference).

Tolerance: relative 1e-8 on every coefficient (the stated parity bound on
Q_ext/Q_abs); scattering matrices: 1e-8 relative to the largest element of
each 4x4 matrix."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-8


@pytest.fixture(scope="module")
def tab():
    return np.load(os.path.join(G, "tables.npz"))


@pytest.fixture(scope="module")
def CT():
    from costuum_b200 import CosTuuM
    return CosTuuM


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def test_one_grain_configuration(tab, CT):
    th = tab["gt1_theta"]
    res, status = CT.get_table(
        types=np.array([0]), sizes=np.array([0.2e-6]), wavelengths=np.array([1e-6]),
        thetas=th, shape_distribution=CT.SingleShapeShapeDistribution(2.0),
        alignment_distribution=CT.SizeBasedAlignmentDistribution(
            1e-5, CT.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=40),
        dust_properties=CT.CustomDustProperties(lambda w, s, t: 1.5 + 0.02j),
        maximum_order=40, do_extinction=True, return_status=True)
    ref = tab["gt1"]
    assert res.shape == ref.shape == (32, 5)
    assert np.all(status == 0)
    # Qabs, Qext (random orientation: the same number at every angle)
    for k in (0, 2):
        assert _rel(res[:, k], ref[:, k]) <= TOL
    # polarised parts are ~1e-15 (rounding) in both: absolute check
    for k in (1, 3, 4):
        assert np.max(np.abs(res[:, k] - ref[:, k])) <= TOL * np.max(np.abs(ref[:, 0]))


def test_grid_draine_hensley_mishchenko_scattering(tab, CT):
    mfun = lambda w, s, t: (1.4 + 0.3 * s / 1e-6) + 0.05j * (1e-6 / w)  # noqa: E731
    q, z = CT.get_table(
        types=np.array([0]), sizes=tab["gt2_sizes"], wavelengths=tab["gt2_lams"],
        thetas=tab["gt2_theta"], shape_distribution=CT.DraineHensleyShapeDistribution(4),
        alignment_distribution=CT.SizeBasedAlignmentDistribution(
            0.1e-6, CT.MISHCHENKO_ALIGNMENT, maximum_order=30),
        dust_properties=CT.CustomDustProperties(mfun), maximum_order=30,
        do_extinction=True, do_scattering=True)
    qref, zref = tab["gt2_qabs"], tab["gt2_z"]
    assert q.shape == qref.shape and z.shape == zref.shape
    scale = np.max(np.abs(qref[..., 0]))
    assert np.max(np.abs(q - qref)) <= TOL * scale
    zs = np.max(np.abs(zref), axis=(-1, -2), keepdims=True)
    assert np.max(np.abs(z - zref) / zs) <= TOL


def test_scattering_subtraction_davis_greenstein(tab, CT):
    res = CT.get_table(
        types=np.array([0, 2]), sizes=np.array([0.4e-6]),
        wavelengths=np.array([1e-6, 2e-6]), thetas=tab["gt3_theta"],
        shape_distribution=CT.SingleShapeShapeDistribution(1.5),
        alignment_distribution=CT.SizeBasedAlignmentDistribution(
            1e-7, CT.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=30),
        dust_properties=CT.CustomDustProperties(lambda w, s, t: (1.4 + 0.1 * t) + 0.05j),
        maximum_order=30, number_of_quadrature_angles=6, account_for_scattering=True)
    ref = tab["gt3"]
    assert res.shape == ref.shape
    assert np.max(np.abs(res - ref)) <= TOL * np.max(np.abs(ref))


def test_disabled_and_custom_alignment(tab, CT):
    kw = dict(types=np.array([0]), sizes=np.array([0.3e-6]), wavelengths=np.array([1e-6]),
              thetas=tab["gt4_theta"],
              shape_distribution=CT.SingleShapeShapeDistribution(0.7),
              dust_properties=CT.CustomDustProperties(lambda w, s, t: 1.6 + 0.2j),
              maximum_order=30, do_extinction=True)
    r4 = CT.get_table(alignment_distribution=CT.SizeBasedAlignmentDistribution(
        1e-7, CT.DISABLE_ALIGNMENT, maximum_order=30), **kw)
    assert np.max(np.abs(r4 - tab["gt4"])) <= TOL * np.max(np.abs(tab["gt4"]))
    ob = CT.MishchenkoOrientationDistribution(0.7, 60)
    pr = CT.DavisGreensteinOrientationDistribution(0.5, 60)
    r5 = CT.get_table(alignment_distribution=CT.SizeBasedAlignmentDistribution(
        1e-7, CT.CUSTOM_ALIGNMENT, 30, ob, pr), **kw)
    assert np.max(np.abs(r5 - tab["gt5"])) <= TOL * np.max(np.abs(tab["gt5"]))
