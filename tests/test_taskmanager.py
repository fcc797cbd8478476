"""The C++ TaskManager-shaped host layer (include/tmx_taskmanager.hpp).

tests/taskmanager/drive_get_table.cpp drives it as CosTuuM's Python module
drives its TaskManager in get_table (CTMModule.cpp:146-478): distributions,
TaskManager(...), add_composition/add_size/add_wavelength, generate_tasks,
QuickSched::execute_tasks, then every coefficient read back through the
ResultKey and the result objects. Its recipe is tests/taskmanager/Makefile.

* CPU: the driver compiles and links against libtmx.so (-Wall -Wextra).
* GPU: its tables equal the golden get_table outputs of the unmodified
  reference (tests/golden/tables.npz) within the get_table tolerance, and
  equal bit for bit the Python module mirror's tables, which reach the same
  tmx_get_table through ctypes.
"""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TM = os.path.join(HERE, "taskmanager")
DRIVER = os.path.join(TM, "drive_get_table")
G = os.path.join(HERE, "golden")
TOL = 1e-8


def _build():
    r = subprocess.run(["make", "-s", "-C", TM], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    assert os.path.exists(DRIVER)


def test_driver_compiles():
    _build()


@pytest.fixture(scope="module")
def driven(tmp_path_factory):
    _build()
    out = tmp_path_factory.mktemp("tm")
    r = subprocess.run([DRIVER, str(out)], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout
    return {f[:-4]: np.fromfile(os.path.join(out, f), dtype="<f8")
            for f in os.listdir(out) if f.endswith(".bin")}


@pytest.fixture(scope="module")
def tab():
    return np.load(os.path.join(G, "tables.npz"))


@pytest.mark.gpu
def test_golden_tables(driven, tab):
    gt1 = driven["gt1"].reshape(tab["gt1"].shape)
    for k in (0, 2):
        ref = tab["gt1"][:, k]
        assert np.max(np.abs(gt1[:, k] - ref) / np.abs(ref)) <= TOL
    scale = np.max(np.abs(tab["gt1"][:, 0]))
    assert np.max(np.abs(gt1 - tab["gt1"])) <= TOL * scale
    q2 = driven["gt2_q"].reshape(tab["gt2_qabs"].shape)
    z2 = driven["gt2_z"].reshape(tab["gt2_z"].shape)
    assert np.max(np.abs(q2 - tab["gt2_qabs"])) <= TOL * np.max(np.abs(tab["gt2_qabs"][..., 0]))
    zs = np.max(np.abs(tab["gt2_z"]), axis=(-1, -2), keepdims=True)
    assert np.max(np.abs(z2 - tab["gt2_z"]) / zs) <= TOL
    for name in ("gt3", "gt4", "gt5"):
        got = driven[name].reshape(tab[name].shape)
        assert np.max(np.abs(got - tab[name])) <= TOL * np.max(np.abs(tab[name])), name


@pytest.mark.gpu
def test_same_doubles_as_module_mirror(driven, tab):
    from costuum_b200 import CosTuuM as C
    th1 = driven["gt1_theta"]  # the driver's angles, bit for bit
    r1 = C.get_table(types=np.array([0]), sizes=np.array([0.2e-6]),
                     wavelengths=np.array([1e-6]), thetas=th1,
                     shape_distribution=C.SingleShapeShapeDistribution(2.0),
                     alignment_distribution=C.SizeBasedAlignmentDistribution(
                         1e-5, C.DAVIS_GREENSTEIN_ALIGNMENT, maximum_order=40),
                     dust_properties=C.CustomDustProperties(lambda w, s, t: 1.5 + 0.02j),
                     maximum_order=40, do_extinction=True)
    assert np.array_equal(driven["gt1"].reshape(r1.shape), r1)
    mfun = lambda w, s, t: (1.4 + 0.3 * s / 1e-6) + 0.05j * (1e-6 / w)  # noqa: E731
    q2, z2 = C.get_table(
        types=np.array([0]), sizes=np.array([0.05e-6, 0.3e-6]),
        wavelengths=np.array([1.5e-6, 0.8e-6]), thetas=np.array([0.3, 1.2, 2.0]),
        shape_distribution=C.DraineHensleyShapeDistribution(4),
        alignment_distribution=C.SizeBasedAlignmentDistribution(
            0.1e-6, C.MISHCHENKO_ALIGNMENT, maximum_order=30),
        dust_properties=C.CustomDustProperties(mfun), maximum_order=30,
        do_extinction=True, do_scattering=True)
    assert np.array_equal(driven["gt2_q"].reshape(q2.shape), q2)
    assert np.array_equal(driven["gt2_z"].reshape(z2.shape), z2)
