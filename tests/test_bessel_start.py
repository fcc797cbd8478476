"""The automatic start of the downward Bessel ratio recurrence.

The reference starts the recurrence for j_n at n = 800 for every argument
(SpecialFunctions.hpp:40, :201-240). The CUDA table kernel starts it at
max(nmax, ceil|z|) + 48 (capped at 800). Above max(nmax, |z|) the recurrence
contracts the start error by about (|z| / 2n)^2 per step, so both starts end
on the same doubles. This test checks bit-equality with the oracle's
restatement of the reference arithmetic over the argument ranges of every
workload (x up to 120, |m| up to about 2.7, nmax up to 100)."""
import numpy as np

import oracle as O

MARGIN = 48


def rule(nmax, absz):
    return min(800, max(nmax, int(np.ceil(absz))) + MARGIN)


def test_real_argument_bitwise():
    rng = np.random.default_rng(123)
    for _ in range(400):
        nmax = int(rng.integers(4, 101))
        z = float(np.exp(rng.uniform(np.log(0.01), np.log(120.0))))
        a = O.bessel_j_real(nmax, z)
        b = O.bessel_j_real_start(nmax, rule(nmax, z), z)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (nmax, z)


def test_complex_argument_bitwise():
    rng = np.random.default_rng(321)
    for _ in range(400):
        nmax = int(rng.integers(4, 101))
        x = float(np.exp(rng.uniform(np.log(0.01), np.log(120.0))))
        m = rng.uniform(1.2, 2.2) + 1j * np.exp(rng.uniform(np.log(1e-4), np.log(1.5)))
        z = m * x
        a = O.bessel_j_complex(nmax, z)
        b = O.bessel_j_complex_start(nmax, rule(nmax, abs(z)), z)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (nmax, z)
