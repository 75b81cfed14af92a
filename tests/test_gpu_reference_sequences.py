"""The call sequences of the reference's TableVisGridderTest
(tests/gridding/TableVisGridderTest.h:94-260) on the GPU gridders, with its
gridder set-ups: SphFunc defaults, WProject(wmax 10000, 9 planes, cutoff
1e-3, oversample 1, maxsupport 128), WStack(10000, 9) and AWProject with a
120 m / 10 m disk (same w set-up, maxfeeds 1).  Reverse: a PSF pass and a
plain pass through one gridder (initialiseGrid, grid, finaliseGrid, then
finaliseWeights), their grids and sums of weights against the oracle.
Forward: an all-zero model leaves the visibilities untouched (the model is
empty).  The reference's data iterator stub is un-vendored; a seeded
36-antenna track stands in for it."""
import math

import numpy as np
import pytest

from parity_helpers import ARCSEC, make_pair, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
W = {"wmax": 10000.0, "nwplanes": 9}
CASES = {
    "SphFunc": {},
    "WProject": dict(W, cutoff=1e-3, oversample=1, maxsupport=128),
    "WStack": dict(W),
    "AWProject": dict(W, cutoff=1e-3, oversample=1, maxsupport=128, maxfeeds=1, diameter="120m", blockage="10m"),
}


@pytest.mark.parametrize("kind", sorted(CASES))
def test_reference_call_sequences(ygmod, oracle_mod, kind):
    import oracle
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, Axes
    ds = simulate.make_dataset(duration_s=60.0, nchan=2, seed=5)
    nx, cell = 512, 10.0 * ARCSEC
    axes = Axes(cell, cell)
    og, gg = make_pair(kind, CASES[kind])
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag)
    chunk = oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag)
    for psf in (True, False):
        gg.initialiseGrid(axes, (nx, nx, 1, 1), dopsf=psf)
        gg.grid(acc)
        og.initialise_grid(nx, nx, 1, 1, cell, cell, dopsf=psf)
        og.grid(chunk)
        g_gpu, g_cpu = np.stack(gg.grids()), np.stack(og.grids)
        assert rel_l2(g_gpu, g_cpu) < TOL, (psf, rel_l2(g_gpu, g_cpu))
        assert np.array_equal(gg.sum_weights(), og.sumw)
        img = gg.finaliseGrid()
        wg = gg.finaliseWeights() if not psf else None
        assert np.all(np.isfinite(img))
        if psf:
            assert np.unravel_index(np.argmax(img[:, :, 0, 0]), (nx, nx)) == (nx // 2, nx // 2)
        else:
            wc = og.finalise_weights()
            assert rel_l2(wg, wc) < (1e-4 if kind == "AWProject" else 1e-6)
    # forward with an all-zero model: nothing is added to the visibilities
    gd = gg.clone()
    gd.initialiseDegrid(axes, np.zeros((nx, nx, 1, 1), dtype=np.float32, order="F"))
    assert gd.isModelEmpty()
    vis = ds.vis.copy(order="F")
    gd.degrid(Accessor(ds.uvw, ds.freq, vis, noise=ds.noise, flag=ds.flag))
    assert np.array_equal(vis, ds.vis)
