"""SKIRT .stab tables (costuum_b200/stab.py) against the byte layout of the
reference's TaskManager test (test/testTaskManager.cpp:238-298)."""
import struct

import numpy as np

from costuum_b200 import stab


def test_layout_and_round_trip(tmp_path):
    sizes = np.array([1e-7, 2e-7])
    lams = np.array([1e-6, 2e-6, 3e-6])
    th = np.array([0.1, 1.5])
    rng = np.random.default_rng(0)
    table = rng.random((2, 3, 2, 2))
    p = tmp_path / "t.stab"
    stab.write_absorption_table(p, sizes, lams, th, table)
    b = p.read_bytes()
    # header as the reference writes it
    exp = b"SKIRT X\n" + struct.pack("<Q", 0x010203040A0BFEFF) + struct.pack("<Q", 3)
    exp += b"a       lambda  theta   m       m       rad     log     log     lin     "
    exp += struct.pack("<Q", 2) + sizes.astype("<f8").tobytes()
    exp += struct.pack("<Q", 3) + lams.astype("<f8").tobytes()
    exp += struct.pack("<Q", 2) + th.astype("<f8").tobytes()
    exp += struct.pack("<Q", 2) + b"Qabs    Qabspol 1       1       log     lin     "
    assert b[:len(exp)] == exp
    # values: theta outer, lambda, size inner; (Qabs, Qabspol) per entry
    vals = []
    for it in range(2):
        for il in range(3):
            for isz in range(2):
                vals += [table[isz, il, it, 0], table[isz, il, it, 1]]
    assert b[len(exp):-8] == np.array(vals, "<f8").tobytes()
    assert b[-8:] == b"STABEND\n"
    axes, qs = stab.read(p)
    assert [a[0] for a in axes] == ["a", "lambda", "theta"]
    assert np.array_equal(qs[0][3], table[..., 0])
    assert np.array_equal(qs[1][3], table[..., 1])
