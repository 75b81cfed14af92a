"""Known-answer tests of the oracle gridder (CPU), restating the value pins in
the reference's tests/measurementequation/ImageFFTEquationTest.h."""
import math

import numpy as np

ARCSEC = math.pi / (180 * 3600)


def _stub_chunk(nrow=400, nchan=2, npol=4, seed=3, umax=2000.0):
    rng = np.random.default_rng(seed)
    uvw = np.zeros((nrow, 3))
    uvw[:, 0] = rng.uniform(-umax, umax, nrow)
    uvw[:, 1] = rng.uniform(-umax, umax, nrow)
    uvw[:, 2] = rng.uniform(-500, 500, nrow)
    freq = np.array([1.4e9, 1.41e9])[:nchan]
    vis = np.zeros((nrow, nchan, npol), dtype=np.complex64, order="F")
    return uvw, freq, vis


def test_full_pol_degrid_sphfunc(oracle_mod):
    """testFullPol (ImageFFTEquationTest.h:124-175): degridding a centred 4-pol
    point image with the default SphFunc gridder gives (1, 0.01, -0.01, 0.9)
    to 1e-5 on every row and channel."""
    import oracle
    npix = 512
    img = np.zeros((npix, npix, 4, 1), dtype=np.float32, order="F")
    vals = [1.0, 0.01, -0.01, 0.9]
    for p, v in enumerate(vals):
        img[npix // 2, npix // 2, p, 0] = v
    g = oracle.OracleGridder("SphFunc")
    g.initialise_degrid(img, 8 * ARCSEC, 8 * ARCSEC)
    uvw, freq, vis = _stub_chunk()
    vis[:] = -10 + 15j   # the reference test pre-fills; degrid adds, so subtract afterwards
    before = vis.copy()
    ch = oracle.Chunk(uvw=uvw, freq=freq, vis=vis)
    g.degrid(ch)
    out = vis - before
    for p, v in enumerate(vals):
        assert np.max(np.abs(out[:, :, p] - v)) < 1e-5


def test_awproject_sums_of_weights_after_reinitialised_grid(oracle_mod):
    """An AWProject gridder that grids a PSF pass and then a plain pass (the
    reverse sequence of TableVisGridderTest) keeps its CF cache and gets
    fresh sums of weights with a row per CF plane at each initialiseGrid."""
    import math

    import numpy as np
    from yandasoft_b200 import simulate
    ds = simulate.make_dataset(duration_s=30.0, nchan=2, seed=5, diameter_m=2000.0)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    og = oracle_mod.OracleGridder("AWProject", wmax=wmax, nwplanes=5, oversample=1, maxsupport=128, maxfeeds=1,
                                  diameter=25.0, blockage=2.0, cutoff=1e-3)
    cell = 20 * math.pi / (180 * 3600)
    chunk = oracle_mod.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag)
    totals = []
    for psf in (True, False):
        og.initialise_grid(256, 256, 1, 1, cell, cell, dopsf=psf)
        og.grid(chunk)
        assert og.sumw.shape == (5 * 2, 1, 1)
        totals.append(og.sumw.sum())
    assert totals[0] == totals[1] > 0
