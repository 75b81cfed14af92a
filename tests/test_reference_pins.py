"""The reference's own unit tests for the gridding helpers, restated against
the oracle (CPU).  Each test cites the reference test it follows.

These pin the oracle before it is trusted as the GPU path's checker."""
import math

import numpy as np
import pytest

from oracle import cf as cfmod
from oracle.spheroidal import SpheroidalFunction, schwab_grdsf


# ---- tests/gridding/FrequencyMapperTest.h --------------------------------
def _fm(freqs, nchan=8, start=1.308e9, end=1.42e9, single=False):
    import oracle
    return oracle.frequency_map(freqs, nchan, start, end, single_plane=single)


def test_freq_mapping(oracle_mod):
    freqs = 1.308e9 + 1.6e7 * (np.arange(10) - 1.0)
    m = _fm(freqs)
    for i in range(10):
        if i == 0 or i + 1 == 10:
            assert m[i] < 0
        else:
            assert m[i] + 1 == i
    assert np.all(_fm(freqs, single=True) == 0)


def test_approx_freq_mapping(oracle_mod):
    i = np.arange(10)
    freqs = 1.436e9 - 1.6e7 * i + np.where(i % 2 == 0, 1.0, -1.0) * 1e6
    m = _fm(freqs)
    for k in range(10):
        if k == 0 or k + 1 == 10:
            assert m[k] < 0
        else:
            assert m[k] + 1 == 10 - k - 1


def test_mfs_freq_mapping(oracle_mod):
    freqs = 1.304e9 + 8e6 * (np.arange(20) - 2.0)
    m = _fm(freqs)
    for k in range(20):
        if k < 2 or k + 2 >= 20:
            assert m[k] < 0
        else:
            assert m[k] + 1 == k // 2


# ---- tests/gridding/NonLinearWSamplingTest.h -----------------------------
def _conversion(smp):
    mid = 0.0
    for i in range(101):
        plane = 2.0 * (i - 50) / 100.0
        mapped = smp.map(plane)
        if -0.5 <= mapped <= 0.5:
            mid += 1.0 / 101
        assert abs(plane - smp.index(mapped)) < 1e-6
    assert abs(smp.index(0.0)) < 1e-6
    assert abs(smp.index(-1.0) + 1.0) < 1e-6
    assert abs(smp.index(1.0) - 1.0) < 1e-6
    return mid


def test_powerlaw_sampling(oracle_mod):
    import oracle
    for i in range(5):
        exponent = 2.0 * (i - 5) / 10.0
        _conversion(oracle.WSampling(3, 1.0, "powerlaw", exponent=exponent))


def test_gaussian_sampling(oracle_mod):
    import oracle
    for i in range(3, 11):
        w50 = i / 11.0 / math.sqrt(2)
        # WSampling takes nwplanes50 in planes; the sampler sees nwplanes50/nwplanes
        smp = oracle.WSampling(1001, 1.0, "gaussian", nwplanes50=w50 * 1001)
        mid = _conversion(smp)
        assert abs(w50 - mid) < 0.02


# ---- tests/gridding/SupportSearcherTest.h --------------------------------
@pytest.fixture
def gauss_buf():
    x = (np.arange(50) - 25 - (-3)) / 5.0
    y = (np.arange(50) - 25 - 7) / 5.0
    return (5.0 * np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / 2)).astype(np.complex64)


def _check_support(ss, shape, cutoff):
    half = 5.0 * math.sqrt(-2.0 * math.log(cutoff))
    assert abs(ss.support() - 2.0 * half) < 1.0
    assert abs(ss.symmetrical_support(shape) - 2.0 * (half + max(-3, 7))) < 1.0
    assert abs(ss.blc[0] - (shape[0] / 2 - 3 - half)) < 1.0
    assert abs(ss.blc[1] - (shape[1] / 2 + 7 - half)) < 1.0
    assert abs(ss.trc[0] - (shape[0] / 2 - 3 + half)) < 1.0
    assert abs(ss.trc[1] - (shape[1] / 2 + 7 + half)) < 1.0


def test_peak_find(gauss_buf):
    pos, val = cfmod.find_peak(gauss_buf)
    assert pos == (25 - 3, 25 + 7)
    assert abs(val - 5.0) < 1e-6


def test_support_search(gauss_buf):
    _check_support(cfmod.support_search(gauss_buf, 1e-2), gauss_buf.shape, 1e-2)


def test_support_search_abs_cutoff(gauss_buf):
    _, peak = cfmod.find_peak(gauss_buf)
    ss = cfmod.support_search(gauss_buf, 1.0, value=1e-2 * peak)
    _check_support(ss, gauss_buf.shape, 1e-2)


# ---- spheroidal function (base-scimath SpheroidalFunction, un-vendored) ---
def test_spheroidal_matches_schwab():
    f = SpheroidalFunction(math.pi * 3, 1.0)
    nu = np.linspace(0.0, 0.999, 200)
    ref = schwab_grdsf(nu) / schwab_grdsf(0.0)[0]
    assert np.max(np.abs(f(nu) - ref)) < 1e-6   # Schwab's stated ~7-digit accuracy
    assert f(1.0) == 0.0 and f(1.5) == 0.0
    assert abs(f(0.0) - 1.0) < 1e-15


def test_spheroidal_converged():
    a = SpheroidalFunction(math.pi * 3, 1.0, nterms=16)
    b = SpheroidalFunction(math.pi * 3, 1.0, nterms=40)
    nu = np.linspace(0, 0.99, 50)
    assert np.max(np.abs(a(nu) - b(nu))) < 1e-13


# ---- askap::nint (un-vendored base-askap) ---------------------------------
def test_nint_half_away_from_zero(oracle_mod):
    import oracle
    assert oracle.nint(0.5) == 1 and oracle.nint(-0.5) == -1
    assert oracle.nint(1.5) == 2 and oracle.nint(-1.5) == -2
    assert oracle.nint(2.4999999) == 2 and oracle.nint(-2.4999999) == -2
    # x + 0.5 rounds to 1.0 in FP64 for the largest double below 0.5
    assert oracle.nint(np.nextafter(0.5, 0.0)) == 1
    assert oracle.nint(0.0) == 0
