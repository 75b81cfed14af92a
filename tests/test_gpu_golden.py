"""The CUDA path against the committed golden fixtures of tests/golden (the
oracle's outputs on small seeded cases, tests/golden/make_golden.py):
cell, offset, plane and CF indices and on-grid status bit-exact, CF taps to
1e-5 of each plane's peak, gridded values and degridded visibilities to 1e-5
relative, sums of weights exact."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
TOL = 1e-5


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def test_wproject_against_golden(ygmod):
    import make_golden as mg
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    gold = np.load(os.path.join(HERE, "golden", "wproject_small.npz"))
    ds, params, nx, cell, model = mg.wproject_case()
    g = VisGridderFactory.make({"gridder": "WProject", **{"gridder.WProject.%s" % k: v for k, v in params.items()}})
    g.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag)
    g.grid(acc)
    s, os_, _ = g.support()
    assert s == int(gold["support"])
    dacc = acc.to_device()
    plan = g.plan(dacc)
    iu, iv, cfi, st = plan.samples(g, dacc)
    on = gold["on"]
    assert np.array_equal(st == 3, on)
    assert np.array_equal(iu[on], gold["iu"][on]) and np.array_equal(iv[on], gold["iv"][on])
    gcfi = gold["fu"] + os_ * (gold["fv"] + os_ * gold["plane"])
    assert np.array_equal(cfi[on], gcfi[on])
    cfs = g.convolution_functions()
    for i, k in enumerate(gold["cf_pick"]):
        c = cfs[k]
        assert np.max(np.abs(c[s - 2:s + 3, s - 2:s + 3] - gold["cf_centre"][i])) <= TOL * np.max(np.abs(c))
    grid = g.grids()[0][:, :, 0, 0].ravel(order="F")
    assert _rel(grid[gold["grid_cells"]], gold["grid_values"]) < TOL
    assert abs(np.linalg.norm(grid) - float(gold["grid_l2"])) <= TOL * float(gold["grid_l2"])
    assert np.array_equal(g.sum_weights(), gold["sumw"])
    gd = g.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vis = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vis, noise=ds.noise, flag=ds.flag))
    assert _rel(vis, gold["degrid"]) < TOL, _rel(vis, gold["degrid"])


def test_sphfunc_full_pol_against_golden(ygmod):
    import make_golden as mg
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    gold = np.load(os.path.join(HERE, "golden", "sphfunc_full_pol.npz"))
    img, uvw, freq, cell = mg.full_pol_case()
    g = VisGridderFactory.make({"gridder": "SphFunc"})
    g.initialiseDegrid(Axes(cell, cell), img)
    vis = np.zeros((uvw.shape[0], 2, 4), dtype=np.complex64, order="F")
    g.degrid(Accessor(uvw, freq, vis))
    assert np.max(np.abs(vis - gold["vis"])) <= TOL


def test_awproject_against_golden(ygmod):
    import make_golden as mg
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    gold = np.load(os.path.join(HERE, "golden", "awproject_small.npz"))
    ds, feed, pnt, params, nx, cell = mg.awproject_case()
    ps = {"gridder": "AWProject", "gridder.AWProject.diameter": "25m", "gridder.AWProject.blockage": "2m",
          **{"gridder.AWProject.%s" % k: v for k, v in params.items()}}
    g = VisGridderFactory.make(ps)
    g.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    g.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    s = g.support()[0]
    assert s == int(gold["support"])
    cfs = g.convolution_functions()
    for i, k in enumerate(gold["cf_pick"]):
        c = cfs[k]
        assert np.max(np.abs(c[s - 2:s + 3, s - 2:s + 3] - gold["cf_centre"][i])) <= TOL * np.max(np.abs(c))
    grid = g.grids()[0][:, :, 0, 0].ravel(order="F")
    assert _rel(grid[gold["grid_cells"]], gold["grid_values"]) < TOL
    assert abs(np.linalg.norm(grid) - float(gold["grid_l2"])) <= TOL * float(gold["grid_l2"])
    assert np.array_equal(g.sum_weights(), gold["sumw"])
