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
