"""The oracle's tap loops pinned to the reference's own compiled GridKernel.

oracle/Makefile compiles askap/gridding/GridKernel.cc from the reference tree,
unchanged, with the flags of the reference's CMakeLists.txt (-std=c++11
-fcx-limited-range, ASKAP_GRID_WITH_POINTERS) against a minimal casacore
Matrix / Complex stand-in (oracle/refstub), into oracle/_ref.  The oracle's
generic loop (TableVisGridder::generic restated) is run once with its own tap
loops and once with the reference's GridKernel::grid / GridKernel::degrid in
their place, on the same seeded inputs with flags, non-unit noise and delays:
grids, sums of weights and degridded visibilities must agree bit for bit.
The GPU parity tests compare the CUDA kernels with the oracle, so they are
held to the reference's compiled arithmetic through this pin.

Skipped where oracle/_ref was not built (the reference tree was absent when
the oracle was built)."""
import math

import numpy as np
import pytest

ARCSEC = math.pi / (180 * 3600)


@pytest.fixture(scope="module")
def ref(oracle_mod):
    R = oracle_mod.reference_gridkernel()
    if R is None:
        pytest.skip("oracle/_ref/libref_gridkernel.so not built")
    yield R
    oracle_mod.use_reference_gridkernel(False)


def _data(npol, seed):
    from yandasoft_b200 import simulate
    ds = simulate.make_dataset(duration_s=120.0, nchan=3, npol=npol, seed=seed, freq0=700e6, freq1=1000e6)
    rng = np.random.default_rng(seed)
    flag = np.zeros(ds.vis.shape, dtype=bool, order="F")
    flag[rng.uniform(size=ds.vis.shape) < 0.03] = True
    noise = np.asfortranarray((rng.uniform(0.5, 2.0, ds.vis.shape) + 0j).astype(np.complex64))
    delay = rng.uniform(-3, 3, ds.nrow)
    return ds, flag, noise, delay


def _run(oracle, kind, kw, ds, flag, noise, delay, nx, cell, npol, use_ref):
    oracle.use_reference_gridkernel(use_ref)
    og = oracle.OracleGridder(kind, **kw)
    og.initialise_grid(nx, nx, npol, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=noise, flag=flag, delay=delay))
    grids = [g.copy() for g in og.grids]
    sumw = og.sumw.copy()
    rng = np.random.default_rng(4)
    og.grids = [np.asfortranarray((rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape))
                                  .astype(np.complex64)) for g in grids]
    og.model_empty = False
    vc = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=noise, flag=flag, delay=delay))
    oracle.use_reference_gridkernel(False)
    return grids, sumw, vc


def test_reference_gridkernel_is_the_pointer_path(ref):
    buf = __import__("ctypes").create_string_buffer(128)
    ref.ref_grid_kernel_info(buf, 128)
    assert buf.value.decode() == "Gridding with casacore::Matrix pointers"


@pytest.mark.parametrize("kind,npol", [("WProject", 1), ("WProject", 4), ("SphFunc", 2), ("WStackWProject", 2)])
def test_oracle_taps_equal_reference_gridkernel(oracle_mod, ref, kind, npol):
    ds, flag, noise, delay = _data(npol, seed=3 + npol)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / 299792458.0) * 1.05
    kw = {"SphFunc": dict(support=3, oversample=16),
          "WProject": dict(wmax=wmax, nwplanes=9, oversample=4, maxsupport=256),
          "WStackWProject": dict(wmax=wmax, nwstacks=5, nwplanes=5, oversample=4, maxsupport=256)}[kind]
    nx, cell = 256, 20.0 * ARCSEC
    g0, s0, v0 = _run(oracle_mod, kind, kw, ds, flag, noise, delay, nx, cell, npol, False)
    g1, s1, v1 = _run(oracle_mod, kind, kw, ds, flag, noise, delay, nx, cell, npol, True)
    assert np.abs(np.stack(g0)).max() > 0 and np.abs(v0).max() > 0
    for a, b in zip(g0, g1):
        assert np.array_equal(a, b)
    assert np.array_equal(s0, s1)
    assert np.array_equal(v0, v1)
