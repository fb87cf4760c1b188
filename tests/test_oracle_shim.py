"""The Boost.Math stand-in the oracle is compiled with, pinned against
independent implementations (mpmath / scipy / numpy) over the orders and arguments
the MLFMA setup uses: Legendre P_l(x) and P_l'(x) for l <= 120, spherical
Bessel / Neumann j_l, y_l for l <= ceil(x) + 2 with x = |k| R up to ~250
(transfer factors, Code/AlgoMLFMM.h:252-281), and Gauss-Legendre nodes and
weights (Code/OverloadAlgo.h:254-288)."""
import ctypes as C

import mpmath
import numpy as np
import pytest
from scipy import special

from conftest import needs_oracle


@pytest.fixture(scope="module")
def shim():
    from oracle import oracle as O
    lib = O._lib()
    for n in ("ref_shim_legendre_p", "ref_shim_legendre_p_prime", "ref_shim_sph_bessel", "ref_shim_sph_neumann"):
        getattr(lib, n).restype = C.c_double
        getattr(lib, n).argtypes = [C.c_int, C.c_double]
    lib.ref_gauss_legendre.restype = None
    lib.ref_gauss_legendre.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return lib


@needs_oracle
def test_legendre(shim):
    mpmath.mp.dps = 40
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(-1, 1, 200), [-1.0, 1.0, 0.0, 0.999999, -0.999999]])
    worst = 0.0
    for l in [0, 1, 2, 3, 7, 20, 50, 87, 120]:
        for x in xs:
            a = shim.ref_shim_legendre_p(l, x)
            b = float(mpmath.legendre(l, mpmath.mpf(float(x))))
            worst = max(worst, abs(a - b))
    assert worst < 1e-13  # ~l ulps accumulate in the recurrence up to l = 120


@needs_oracle
def test_legendre_derivative(shim):
    rng = np.random.default_rng(2)
    xs = rng.uniform(-0.999, 0.999, 100)
    for l in [1, 2, 5, 16, 40, 90]:
        for x in xs:
            a = shim.ref_shim_legendre_p_prime(l, x)
            # n (x P_n - P_{n-1}) / (x^2 - 1)
            b = l * (x * special.eval_legendre(l, x) - special.eval_legendre(l - 1, x)) / (x * x - 1)
            assert abs(a - b) <= 1e-11 * max(1.0, abs(b))


@needs_oracle
def test_spherical_bessel_and_neumann(shim):
    rng = np.random.default_rng(3)
    for x in np.concatenate([rng.uniform(0.5, 260.0, 60), [3.14, 6.3, 12.6, 100.0]]):
        Lmax = int(np.ceil(x)) + 2
        for l in range(0, Lmax + 1, max(1, Lmax // 25)):
            j = shim.ref_shim_sph_bessel(l, x)
            y = shim.ref_shim_sph_neumann(l, x)
            jr = special.spherical_jn(l, x)
            yr = special.spherical_yn(l, x)
            # |h2| = sqrt(j^2 + y^2) is the scale the transfer factor sees
            scale = np.hypot(jr, yr)
            assert abs(j - jr) <= 1e-12 * scale, (l, x, j, jr)
            assert abs(y - yr) <= 1e-12 * scale, (l, x, y, yr)


@needs_oracle
def test_gauss_legendre_nodes(shim):
    for n in [3, 12, 16, 25, 44, 97]:
        x = np.empty(n)
        w = np.empty(n)
        shim.ref_gauss_legendre(n, x.ctypes.data_as(C.POINTER(C.c_double)), w.ctypes.data_as(C.POINTER(C.c_double)))
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.max(np.abs(x - xr)) < 1e-14
        assert np.max(np.abs(w - wr)) < 1e-13
