"""The major cycle recorded as one CUDA graph (yg_cycle_*): degrid the model,
subtract, grid the residual (and the PSF and preconditioner function), for
one and for several instances of uneven size, against the same steps run one
call at a time and against the oracle's steps."""
import numpy as np
import pytest

from parity_helpers import ARCSEC, rel_l2, snapped_model

pytestmark = pytest.mark.gpu


def _instance(nx, cellas, dur, nchan, seed, kind="WProject"):
    import torch
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    ds = simulate.make_dataset(duration_s=dur, nchan=nchan, npol=1, seed=seed, diameter_m=3000.0)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    ps = {"gridder": kind, "gridder.%s.wmax" % kind: wmax, "gridder.%s.nwplanes" % kind: 9,
          "gridder.%s.oversample" % kind: 4, "gridder.%s.maxsupport" % kind: 256}
    cell = cellas * ARCSEC
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=6, seed=seed)
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag).to_device()
    return dict(ds=ds, ps=ps, cell=cell, nx=nx, model=model, acc=acc,
                make=lambda: VisGridderFactory.make(ps), axes=Axes(cell, cell))


def _reference_residual_grid(I):
    """degrid, subtract and grid one call at a time (host round trip)."""
    from yandasoft_b200.gridder import Accessor
    ds = I["ds"]
    gd = I["make"]()
    gd.initialiseDegrid(I["axes"], I["model"])
    mv = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, mv, noise=ds.noise, flag=ds.flag))
    res = np.asfortranarray((ds.vis - mv).astype(np.complex64))
    gg = I["make"]()
    gg.initialiseGrid(I["axes"], (I["nx"], I["nx"], 1, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, res, noise=ds.noise, flag=ds.flag))
    return np.stack(gg.grids()), gg.sum_weights()


def _cycle_pair(I):
    gd = I["make"]()
    gd.initialiseDegrid(I["axes"], I["model"])
    gg = I["make"]()
    gg.initialiseGrid(I["axes"], (I["nx"], I["nx"], 1, 1))
    return gd, gg


def test_single_instance_cycle_matches_calls(ygmod, oracle_mod):
    from yandasoft_b200.gridder import MajorCycle
    I = _instance(512, 20.0, 600.0, 2, 41)
    gd, gg = _cycle_pair(I)
    cyc = MajorCycle([gd], [gg], [I["acc"]])
    assert cyc.nodes() > 3
    gg.initialiseGrid(I["axes"], (I["nx"], I["nx"], 1, 1))     # the creation ran one cycle
    cyc.run(1)
    ref, sw = _reference_residual_grid(I)
    assert rel_l2(np.stack(gg.grids()), ref) < 1e-6
    assert np.array_equal(gg.sum_weights(), sw)


def test_batched_uneven_instances_replay(ygmod, oracle_mod):
    from yandasoft_b200.gridder import MajorCycle
    specs = [(256, 40.0, 300.0, 1, 51), (512, 20.0, 900.0, 4, 52), (1024, 10.0, 600.0, 2, 53)]
    insts = [_instance(*s) for s in specs]
    pairs = [_cycle_pair(I) for I in insts]
    cyc = MajorCycle([p[0] for p in pairs], [p[1] for p in pairs], [I["acc"] for I in insts])
    for I, (gd, gg) in zip(insts, pairs):
        gg.initialiseGrid(I["axes"], (I["nx"], I["nx"], 1, 1))
    ms = cyc.run(2)                      # the model does not change: two residual passes
    assert ms > 0
    for I, (gd, gg) in zip(insts, pairs):
        ref, _ = _reference_residual_grid(I)
        assert rel_l2(np.stack(gg.grids()), 2 * ref) < 1e-6


def test_model_update_between_cycles(ygmod, oracle_mod):
    from yandasoft_b200.gridder import MajorCycle
    I = _instance(512, 20.0, 600.0, 2, 61)
    gd, gg = _cycle_pair(I)
    cyc = MajorCycle([gd], [gg], [I["acc"]])
    # a new model of the same shape: half the old one
    I["model"] = np.asfortranarray(0.5 * I["model"])
    gd.initialiseDegrid(I["axes"], I["model"])
    gg.initialiseGrid(I["axes"], (I["nx"], I["nx"], 1, 1))
    cyc.run(1)
    ref, _ = _reference_residual_grid(I)
    assert rel_l2(np.stack(gg.grids()), ref) < 1e-6


def test_cycle_residual_psf_pcf_against_oracle(ygmod, oracle_mod):
    """One instance with every role of ImageFFTEquation::calcImagingEquations
    (ImageFFTEquation.cc:437-479) in one graph: degrid the model, subtract,
    grid the residual, then the PSF and the preconditioner function from the
    same buffer.  Checked against the oracle's steps, not against the GPU's
    own per-call path: the oracle degrids the model grids the GPU transformed
    (the tap path; the FFT side is compared elsewhere), the residual is formed
    in FP32 as the graph forms it, and the oracle grids it three times
    (residual, PSF, preconditioner).  Grids 1e-5 relative L2, sums of weights
    exact."""
    import oracle
    from yandasoft_b200.gridder import MajorCycle
    I = _instance(512, 20.0, 300.0, 3, 71)
    ds, nx, cell = I["ds"], I["nx"], I["cell"]
    gd, gg = _cycle_pair(I)
    gp = I["make"]()
    gp.initialiseGrid(I["axes"], (nx, nx, 1, 1), dopsf=True)
    gc = I["make"]()
    gc.initialiseGrid(I["axes"], (nx, nx, 1, 1), dopcf=True)
    cyc = MajorCycle([gd], [gg], [I["acc"]], psf=[gp], pcf=[gc])
    assert cyc.nodes() > 4
    # the creation ran one uncaptured cycle: start every grid again, then replay
    gg.initialiseGrid(I["axes"], (nx, nx, 1, 1))
    gp.initialiseGrid(I["axes"], (nx, nx, 1, 1), dopsf=True)
    gc.initialiseGrid(I["axes"], (nx, nx, 1, 1), dopcf=True)
    cyc.run(1)
    ps = I["ps"]
    kw = dict(wmax=ps["gridder.WProject.wmax"], nwplanes=9, oversample=4, maxsupport=256)
    od = oracle.OracleGridder("WProject", **kw)
    od.initialise_degrid(I["model"], cell, cell)
    od.grids = [np.asfortranarray(g) for g in gd.grids()]
    mv = np.zeros_like(ds.vis)
    od.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=mv, noise=ds.noise, flag=ds.flag))
    resid = np.asfortranarray(ds.vis - mv)
    for g, flags in ((gg, {}), (gp, {"dopsf": True}), (gc, {"dopcf": True})):
        og = oracle.OracleGridder("WProject", **kw)
        og.initialise_grid(nx, nx, 1, 1, cell, cell, **flags)
        og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=resid, noise=ds.noise, flag=ds.flag))
        ref = np.stack(og.grids)
        assert np.abs(ref).max() > 0
        err = rel_l2(np.stack(g.grids()), ref)
        assert err < 1e-5, (flags, err)
        assert np.array_equal(g.sum_weights(), og.sumw), flags
