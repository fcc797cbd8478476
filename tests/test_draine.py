"""DraineDustProperties: refractive indices from the tabulated Draine (2003)
optical constants (DraineDustProperties.hpp:36-242, Table.hpp:126-260).

The tables are not part of this package; the tests read them from the
directory the reference build recorded (oracle.draine_data_directory) and
skip where it is absent. Golden values: the reference module's own
DraineDustProperties (tests/golden/draine.npz, make_golden.py draine), at
20 K and 50 K, sizes 0.01-2 um and wavelengths across and beyond the tables.
The arithmetic follows the reference's operation order; the bound is 1e-14
relative (the same doubles in practice)."""
import os

import numpy as np
import pytest

import oracle as O
from costuum_b200 import CosTuuM as C

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DATA = O.draine_data_directory()
need_data = pytest.mark.skipif(DATA is None, reason="Draine data files not available")


@need_data
@pytest.mark.parametrize("T", [20, 50])
def test_against_reference_values(T):
    z = np.load(os.path.join(G, "draine.npz"))
    D = C.DraineDustProperties(dust_temperature=float(T), data_directory=DATA)
    gold = z["m_%d" % T]
    for t in range(3):
        for i, a in enumerate(z["sizes"]):
            for j, lam in enumerate(z["wavelengths"]):
                m = D.get_refractive_index(t, a, lam)
                assert abs(m - gold[t, i, j]) <= 1e-14 * abs(gold[t, i, j]), (t, a, lam)


@need_data
def test_environment_variable_and_errors(monkeypatch):
    monkeypatch.setenv("COSTUUM_DRAINE_DATA", DATA)
    D = C.DraineDustProperties()
    assert D.get_refractive_index(C.SILICON, 1e-7, 1e-6).imag > 0
    with pytest.raises(ValueError):
        D.get_refractive_index(3, 1e-7, 1e-6)


def test_missing_tables_raise(monkeypatch, tmp_path):
    monkeypatch.delenv("COSTUUM_DRAINE_DATA", raising=False)
    with pytest.raises(FileNotFoundError):
        C.DraineDustProperties()
    with pytest.raises(FileNotFoundError):
        C.DraineDustProperties(data_directory=str(tmp_path))
