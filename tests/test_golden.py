"""The oracle against the committed golden fixtures of tests/golden (made by
tests/golden/make_golden.py from the oracle itself): a regression pin of the
CPU restatement, so that a change of the oracle shows here before it moves
the parity bar of the GPU tests (test_gpu_golden.py checks the CUDA path
against the same fixtures)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def test_oracle_reproduces_wproject_golden(oracle_mod):
    import make_golden as mg
    import oracle
    gold = np.load(os.path.join(HERE, "golden", "wproject_small.npz"))
    ds, params, nx, cell, model = mg.wproject_case()
    og = oracle.OracleGridder("WProject", **params)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    iu, iv, fu, fv = oracle.indices(ds.uvw, ds.freq, og.uvcell[0], og.uvcell[1], og.os, nx, nx)
    for k, v in (("iu", iu), ("iv", iv), ("fu", fu), ("fv", fv), ("plane", og.ws.plane_map(ds.uvw, ds.freq))):
        assert np.array_equal(v, gold[k]), k
    assert og.cache.support == int(gold["support"])
    s = og.cache.support
    for i, k in enumerate(gold["cf_pick"]):
        c = og.cache.cfs[k]
        assert np.max(np.abs(c[s - 2:s + 3, s - 2:s + 3] - gold["cf_centre"][i])) <= 1e-6 * np.max(np.abs(c))
    grid = og.grids[0][:, :, 0, 0].ravel(order="F")
    assert _rel(grid[gold["grid_cells"]], gold["grid_values"]) < 1e-6
    assert abs(np.linalg.norm(grid) - float(gold["grid_l2"])) <= 1e-6 * float(gold["grid_l2"])
    assert np.array_equal(og.sumw, gold["sumw"])
    og.initialise_degrid(model, cell, cell)
    vis = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vis, noise=ds.noise, flag=ds.flag))
    assert _rel(vis, gold["degrid"]) < 1e-6


def test_oracle_reproduces_full_pol_golden(oracle_mod):
    import make_golden as mg
    import oracle
    gold = np.load(os.path.join(HERE, "golden", "sphfunc_full_pol.npz"))
    img, uvw, freq, cell = mg.full_pol_case()
    og = oracle.OracleGridder("SphFunc")
    og.initialise_degrid(img, cell, cell)
    vis = np.zeros((uvw.shape[0], 2, 4), dtype=np.complex64, order="F")
    og.degrid(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    assert np.max(np.abs(vis - gold["vis"])) <= 1e-6
    # the known answer of ImageFFTEquationTest::testFullPol, to 1e-5
    for p, v in enumerate([1.0, 0.01, -0.01, 0.9]):
        assert np.max(np.abs(gold["vis"][:, :, p] - v)) < 1e-5


def test_oracle_reproduces_awproject_golden(oracle_mod):
    import make_golden as mg
    import oracle
    gold = np.load(os.path.join(HERE, "golden", "awproject_small.npz"))
    ds, feed, pnt, params, nx, cell = mg.awproject_case()
    og = oracle.OracleGridder("AWProject", diameter=25.0, blockage=2.0, **params)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt))
    s = og.cache.support
    assert s == int(gold["support"])
    for i, k in enumerate(gold["cf_pick"]):
        c = og.cache.cfs[k]
        assert np.max(np.abs(c[s - 2:s + 3, s - 2:s + 3] - gold["cf_centre"][i])) <= 1e-6 * np.max(np.abs(c))
    grid = og.grids[0][:, :, 0, 0].ravel(order="F")
    assert _rel(grid[gold["grid_cells"]], gold["grid_values"]) < 1e-6
    assert np.array_equal(og.sumw, gold["sumw"])
