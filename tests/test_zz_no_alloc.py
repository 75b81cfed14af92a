"""yg_degrid_noalloc: degridding for callers that cannot allocate device
memory (an application that fixes each GPU's memory budget when it starts and
forbids later allocations, or a host framework whose own pool allocator owns
the device's memory).  It must give what yg_degrid gives, within the 1e-5
relative tolerance of the other parity tests, on consecutive calls (the model
is added into the visibilities and the value carried into off-grid samples
persists across calls), for every gridder kind it takes, one and four
polarisations, and with MFS weights.  Its first call on a device is the
set-up (the static array's address is looked up); from then on a call must
not change the device's free memory at all.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test."""
import numpy as np
import pytest

from parity_helpers import ARCSEC, rel_l2, snapped_model

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _params(kind, wmax):
    if kind == "SphFunc":
        return {"gridder": "SphFunc"}
    p = {"gridder": kind, "gridder.%s.wmax" % kind: wmax, "gridder.%s.nwplanes" % kind: 9}
    if kind in ("WProject", "WStackWProject"):
        p.update({"gridder.%s.oversample" % kind: 4, "gridder.%s.maxsupport" % kind: 256})
    if kind == "WStackWProject":
        p["gridder.%s.nwstacks" % kind] = 5
    return p


@pytest.mark.parametrize("kind,npol,mfs", [("WProject", 1, False), ("WProject", 4, False), ("SphFunc", 1, False),
                                           ("WStack", 4, False), ("WStackWProject", 4, False),
                                           ("WProject", 1, True)])
def test_degrid_noalloc_matches_degrid(ygmod, kind, npol, mfs):
    import torch
    from yandasoft_b200 import simulate
    G = ygmod
    ds = simulate.make_dataset(duration_s=300.0, nchan=4, npol=npol, seed=17)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    nx, cell = 512, 20.0 * ARCSEC
    ps = _params(kind, wmax)
    existing = G.VisGridderFactory.make(ps)
    noalloc = G.VisGridderFactory.make(ps)
    if mfs:
        existing.initVisWeights(float(ds.freq.mean()) * 0.99)
        noalloc.initVisWeights(float(ds.freq.mean()) * 0.99)
    model, _ = snapped_model(ds, nx, cell, npol=npol, max_nu=0.5, extra=6)
    axes = G.Axes(cell, cell)
    existing.initialiseDegrid(axes, model)
    noalloc.initialiseDegrid(axes, model)
    noalloc.build_cf()     # set-up (allocates); the degrid calls below must not
    # two different chunks in turn (the second half of the rows, then the first),
    # so the value carried into off-grid samples crosses chunk boundaries
    half = ds.nrow // 2
    parts = [slice(half, ds.nrow), slice(0, half), slice(half, ds.nrow)]
    rng = np.random.default_rng(1)
    for call, sl in enumerate(parts):
        start = np.asfortranarray((rng.standard_normal(ds.vis[sl].shape) * (1 + 1j)).astype(np.complex64))
        uvw = np.ascontiguousarray(ds.uvw[sl])
        acc_a = G.Accessor(uvw, ds.freq, start.copy(order="F")).to_device()
        acc_b = G.Accessor(uvw, ds.freq, start.copy(order="F")).to_device()
        existing.degrid(acc_a)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        noalloc.degrid_noalloc(acc_b)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        a = acc_a.vis_numpy() - start
        b = acc_b.vis_numpy() - start
        assert np.abs(a).max() > 0
        err = rel_l2(b, a)
        assert err < TOL, "call %d: relative error %.3e" % (call, err)
        if call > 0:
            assert free_after == free_before, "device memory changed during the call: %d bytes" % (
                free_before - free_after)


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


def test_degrid_noalloc_rejects_awproject(ygmod):
    """AWProject builds its CFs per chunk: the call refuses it
    (YG_ERR_UNSUPPORTED) rather than degrid with CFs of another chunk."""
    from yandasoft_b200 import simulate
    G = ygmod
    ds = simulate.make_dataset(duration_s=60.0, nchan=1, seed=4)
    img = np.zeros((256, 256, 1, 1), dtype=np.float32, order="F")
    img[128, 128, 0, 0] = 1.0
    acc = G.Accessor(ds.uvw, ds.freq, np.zeros_like(ds.vis)).to_device()
    aw = G.VisGridderFactory.make({"gridder": "AWProject", "gridder.AWProject.wmax": 5000.0,
                                   "gridder.AWProject.nwplanes": 5, "gridder.AWProject.diameter": "12m",
                                   "gridder.AWProject.blockage": "1m"})
    aw.initialiseDegrid(G.Axes(20 * ARCSEC, 20 * ARCSEC), img)
    with pytest.raises(G.AskapError) as e:
        aw.degrid_noalloc(acc)
    assert e.value.code == 9
