"""yg_degrid_noalloc: degridding for callers that cannot allocate device
memory (stream capture into a CUDA graph, fixed memory budgets).  It must
give what yg_degrid gives, on consecutive calls (the model is added into the
visibilities and the value carried into off-grid samples persists across
calls).  Its first call on a device is the set-up (the static array's address
is looked up, which makes the driver load the array); from then on a call
must not allocate device memory.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test."""
import numpy as np
import pytest

from parity_helpers import ARCSEC, rel_l2, snapped_model

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_degrid_noalloc_matches_degrid(ygmod):
    import torch
    from yandasoft_b200 import simulate
    G = ygmod
    ds, p = simulate.config0(duration_s=300.0)
    nx = p["nx"]
    cell = p["cell_arcsec"] * ARCSEC
    ps = {"gridder": "WProject", "gridder.WProject.wmax": p["wmax"], "gridder.WProject.nwplanes": p["nwplanes"],
          "gridder.WProject.oversample": p["oversample"], "gridder.WProject.cutoff": p["cutoff"],
          "gridder.WProject.maxsupport": p["maxsupport"]}
    existing = G.VisGridderFactory.make(ps)
    noalloc = G.VisGridderFactory.make(ps)
    model, _ = snapped_model(ds, nx, cell)
    axes = G.Axes(cell, cell)
    existing.initialiseDegrid(axes, model)
    noalloc.initialiseDegrid(axes, model)
    noalloc.build_cf()     # set-up (allocates); the degrid calls below must not
    acc_a = G.Accessor(ds.uvw, ds.freq, np.zeros_like(ds.vis), noise=ds.noise, flag=ds.flag).to_device()
    acc_b = G.Accessor(ds.uvw, ds.freq, np.zeros_like(ds.vis), noise=ds.noise, flag=ds.flag).to_device()
    for call in range(2):
        existing.degrid(acc_a)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        noalloc.degrid_noalloc(acc_b)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        a = acc_a.vis_numpy()
        b = acc_b.vis_numpy()
        assert np.abs(a).max() > 0
        err = rel_l2(b, a)
        assert err < TOL, "call %d: relative error %.3e" % (call, err)
        if call > 0:
            assert free_after >= free_before - (1 << 20), "device memory was allocated during the call"


def test_degrid_noalloc_rejects_oversize(ygmod):
    from yandasoft_b200 import simulate
    G = ygmod
    ds = simulate.make_dataset(duration_s=60.0, nchan=1, seed=4)
    g = G.VisGridderFactory.make({"gridder": "SphFunc"})
    img = np.zeros((256, 256, 1, 1), dtype=np.float32, order="F")
    img[128, 128, 0, 0] = 1.0
    g.initialiseDegrid(G.Axes(20 * ARCSEC, 20 * ARCSEC), img)
    g.build_cf()
    big = 1 << 20
    nrow = big // 4 + 1
    uvw = np.zeros((nrow, 3))
    freq = np.full(4, 1.0e9)
    vis = np.zeros((nrow, 4, 1), dtype=np.complex64, order="F")
    acc = G.Accessor(uvw, freq, vis).to_device()
    with pytest.raises(G.AskapError) as e:
        g.degrid_noalloc(acc)
    assert "at most" in str(e.value)
