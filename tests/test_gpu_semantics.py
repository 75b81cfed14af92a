"""TableVisGridder::generic semantics on the GPU against the oracle, on inputs
built to reach every branch of the sample path rather than the all-unit
defaults of the simulator:

* partial-polarisation flags: a vector with any flagged polarisation is
  skipped whole, in gridding and degridding (TableVisGridder.cc:657-663);
* non-unit noise: wt = 1/real(noise)^2 in float, rVis = phasor conj(vis) wt,
  sums of weights in double (TableVisGridder.cc:777-806), and a per-row delay
  phasor (:653-655);
* channels the FrequencyMapper leaves unmapped, including a data channel
  exactly half way between two image channels (FrequencyMapper.cc:72-107);
* uvw and w built so that the FP64 index block meets exact ties: uScaled on
  k + 1/2 and on oversampling ties, the strict on-grid edge
  (TableVisGridder.cc:763-764) from both sides, and w exactly on a w-plane or
  w-stack boundary and on the clipping edge (WDependentGridderBase.cc:118-150);
* the headline workload's geometry: 4096^2 x 4 pol, 17 w-stacks x 33
  w-planes, oversample 8, on a seeded 1% row subset, through the same tile and
  k_grid / k_degrid_t instantiation as the benchmark.

Tolerances: indices and statuses bit-exact; grids and visibilities 1e-5
relative L2.  Sums of weights are compared bit for bit: every weight is an
FP32 number between 1/4 and 4 (noise real parts in [0.5, 2]), so each
partial sum of fewer than 2^26 of them is an integer multiple of 2^-25 below
2^28 and is exact in FP64, whatever the order of the additions.
"""
import math

import numpy as np
import pytest

from parity_helpers import ARCSEC, make_pair, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
C = 299792458.0


def _data(duration=180.0, nchan=4, npol=4, seed=31, f0=700e6, f1=1000e6):
    from yandasoft_b200 import simulate
    return simulate.make_dataset(duration_s=duration, nchan=nchan, npol=npol, seed=seed, freq0=f0, freq1=f1)


def _wmax(uvw, freq):
    return float(np.max(np.abs(uvw[:, 2])) * np.max(freq) / C) * 1.05


def _flags_noise_delay(ds, seed):
    """Seeded flags (8% of vectors with one polarisation flagged, 2% with all),
    noise real parts uniform in [0.5, 2] (imaginary parts random: the weight
    reads only the real part) and delays of up to +-5 m."""
    rng = np.random.default_rng(seed)
    nrow, nchan, npol = ds.vis.shape
    flag = np.zeros((nrow, nchan, npol), dtype=bool, order="F")
    u = rng.uniform(size=(nrow, nchan))
    one = u < 0.08
    pol = rng.integers(0, npol, size=(nrow, nchan))
    r, c = np.nonzero(one)
    flag[r, c, pol[r, c]] = True
    flag[u > 0.98, :] = True
    noise = (rng.uniform(0.5, 2.0, (nrow, nchan, npol)) + 1j * rng.uniform(-1, 1, (nrow, nchan, npol)))
    noise = np.asfortranarray(noise.astype(np.complex64))
    delay = rng.uniform(-5.0, 5.0, nrow)
    return flag, noise, delay


def _grid_pair(og, gg, cell, shape, chunk_kw, freq_axis=None):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    nx, ny, npol, nchan = shape
    gg.initialiseGrid(Axes(cell, cell, freq=freq_axis), shape)
    gg.grid(Accessor(chunk_kw["uvw"], chunk_kw["freq"], chunk_kw["vis"], noise=chunk_kw.get("noise"),
                     flag=chunk_kw.get("flag"), delay=chunk_kw.get("delay")))
    og.initialise_grid(nx, ny, npol, nchan, cell, cell, freq_axis=freq_axis)
    og.grid(oracle.Chunk(**chunk_kw))


def _check_grid(og, gg, exact_sumw=True):
    gpu = gg.grids()
    assert len(gpu) == len(og.grids)
    ref = np.stack(og.grids)
    assert np.abs(ref).max() > 0
    err = rel_l2(np.stack(gpu), ref)
    assert err < TOL, err
    sw_gpu, sw_cpu = gg.sum_weights(), og.sumw
    assert sw_gpu.shape == sw_cpu.shape
    assert sw_cpu.sum() > 0
    if exact_sumw:
        assert np.array_equal(sw_gpu, sw_cpu), float(np.max(np.abs(sw_gpu - sw_cpu)))
    return err


def _point_model(nx, npol, nchan, seed=13, n=12):
    rng = np.random.default_rng(seed)
    img = np.zeros((nx, nx, npol, nchan), dtype=np.float32, order="F")
    q = nx // 4
    for _ in range(n):
        x, y = nx // 2 + int(rng.integers(-q, q)), nx // 2 + int(rng.integers(-q, q))
        img[x, y] += np.float32(rng.uniform(0.1, 1.0))
    return img


def _degrid_taps(og, gg, chunk_kw, start_vis, cell, model, freq_axis=None):
    """Degrids a point model: the GPU gridder transforms it to its grids
    (initialiseDegrid) and both degrid those same grids (the FFT side is
    compared elsewhere); visibilities are added into a copy of start_vis."""
    import copy

    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell, freq=freq_axis), model)
    grids = [np.asfortranarray(g) for g in gd.grids()]
    vg = np.asfortranarray(start_vis.copy())
    gd.degrid(Accessor(chunk_kw["uvw"], chunk_kw["freq"], vg, noise=chunk_kw.get("noise"), flag=chunk_kw.get("flag"),
                       delay=chunk_kw.get("delay")))
    oc = copy.copy(og)
    oc.carry = None if og.carry is None else og.carry.copy()
    oc.grids = grids
    oc.model_empty = False
    vc = np.asfortranarray(start_vis.copy())
    kw = dict(chunk_kw)
    kw["vis"] = vc
    oc.degrid(oracle.Chunk(**kw))
    return vg, vc


@pytest.mark.parametrize("kind,npol", [("WProject", 4), ("WProject", 2), ("WStackWProject", 4), ("SphFunc", 2),
                                       ("WStack", 1)])
def test_flags_noise_weights_delay(ygmod, oracle_mod, kind, npol):
    ds = _data(npol=npol, seed=31 + npol)
    flag, noise, delay = _flags_noise_delay(ds, seed=7)
    wmax = _wmax(ds.uvw, ds.freq)
    nx, cell = 512, 10.0 * ARCSEC
    params = {"SphFunc": {"support": 3, "oversample": 32},
              "WStack": {"wmax": wmax, "nwplanes": 9},
              "WProject": {"wmax": wmax, "nwplanes": 9, "oversample": 4, "maxsupport": 256},
              "WStackWProject": {"wmax": wmax, "nwstacks": 5, "nwplanes": 9, "oversample": 4,
                                 "maxsupport": 256}}[kind]
    okw = {"nwstacks": 5} if kind == "WStackWProject" else None
    og, gg = make_pair(kind, params, oracle_kw=okw)
    chunk = dict(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=noise, flag=flag, delay=delay)
    _grid_pair(og, gg, cell, (nx, nx, npol, 1), chunk)
    _check_grid(og, gg)
    # every vector that has a flagged polarisation is left out of the sums
    good = ~flag.any(axis=2)
    assert 0 < good.sum() < good.size
    # degridding: flagged vectors keep their values; the others match the oracle
    start = np.asfortranarray((np.random.default_rng(3).standard_normal(ds.vis.shape) * (1 + 1j)).astype(np.complex64))
    vg, vc = _degrid_taps(og, gg, chunk, start, cell, _point_model(nx, npol, 1))
    bad = ~good
    assert np.array_equal(vg[bad], start[bad])
    assert np.array_equal(vc[bad], start[bad])
    err = rel_l2(vg - start, vc - start)
    assert err < TOL, err


def test_unmapped_channels_and_frequency_ties(ygmod, oracle_mod):
    """Image cube of 4 channels at 942-945 MHz over data channels at
    940.5-947.5 MHz: 940.5, 941.5, 945.5, 946.5 and 947.5 MHz are unmapped
    (skipped), 942.5 MHz lies exactly half way and maps up (half away from
    zero)."""
    import oracle
    ds = _data(npol=2, nchan=8, f0=940e6, f1=948e6, seed=41)
    flag, noise, delay = _flags_noise_delay(ds, seed=9)
    wmax = _wmax(ds.uvw, ds.freq)
    nx, cell = 512, 10.0 * ARCSEC
    fa = (942e6, 945e6)
    cmap = oracle.frequency_map(ds.freq, 4, fa[0], fa[1])
    assert list(cmap) == [-1, -1, 1, 2, 3, -1, -1, -1]
    params = {"wmax": wmax, "nwplanes": 9, "oversample": 4, "maxsupport": 256}
    og, gg = make_pair("WProject", params)
    chunk = dict(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=noise, flag=flag, delay=delay)
    _grid_pair(og, gg, cell, (nx, nx, 2, 4), chunk, freq_axis=fa)
    _check_grid(og, gg)
    # image channel 0 receives nothing; the weights of unmapped channels are nowhere
    assert not np.stack(gg.grids())[:, :, :, :, 0].any()
    start = np.asfortranarray(np.full(ds.vis.shape, 0.5 - 0.25j, dtype=np.complex64))
    vg, vc = _degrid_taps(og, gg, chunk, start, cell, _point_model(nx, 2, 4), freq_axis=fa)
    unmapped = np.nonzero(cmap < 0)[0]
    assert np.array_equal(vg[:, unmapped, :], start[:, unmapped, :])
    err = rel_l2(vg - start, vc - start)
    assert err < TOL, err


def _exact_w(values, f):
    """Keeps the w (metres) whose FP64 w-term (w / c) * f, computed in the
    reference's order, equals the intended value exactly."""
    w = np.asarray(values, dtype=np.float64) * C / f
    got = (w / C) * f
    ok = got == np.asarray(values, dtype=np.float64)
    return w, ok


def _tie_dataset(nx, cellu, wscale, nclip, inner=0.0, seed=5):
    """Rows whose u and v, in units of the uv cell, run over every multiple of
    1/32 across the grid and past both edges, at two frequencies (c and c/2,
    where the FP64 scaling is exact); w at the first frequency on w-plane (or
    w-stack) ties k + 1/2, on plane centres, with `inner` > 0 on ties of the
    inner planes (spacing `inner`) inside a stack, and for nclip rows exactly
    on the clipping edge (plus or minus 4.5 planes)."""
    rng = np.random.default_rng(seed)
    half = nx // 2 + 4
    m = np.arange(-half * 32, half * 32 + 1)
    us = m / 32.0
    vs = rng.permutation(us)
    nrow = len(us)
    uvw = np.zeros((nrow, 3))
    uvw[:, 0] = us * cellu          # f = c: metres == wavelengths
    uvw[:, 1] = vs * cellu
    k = rng.integers(-4, 4, nrow)
    pick = rng.integers(0, 3, nrow)
    want = np.where(pick == 0, (k + 0.5) * wscale, k * wscale)
    if inner > 0:
        j = rng.integers(-4, 4, nrow)
        want = np.where(pick == 2, k * wscale + (j + 0.5) * inner, want)
    want[:nclip] = np.where(np.arange(nclip) % 2 == 0, 4.5, -4.5) * wscale
    w, ok = _exact_w(want, C)
    assert ok.mean() > 0.9
    uvw[:, 2] = np.where(ok, w, 0.0)
    freq = np.array([C, C / 2])
    return uvw, freq


@pytest.mark.parametrize("kind", ["WProject", "WStackWProject"])
def test_exact_ties_and_grid_edges(ygmod, oracle_mod, kind):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    nx = 128
    cell = 2.0 ** -9                 # rad: cellu = 1 / (cell nx) = 4 wavelengths exactly
    cellu = 1.0 / (cell * nx)
    assert cellu == 4.0
    os_ = 4
    if kind == "WProject":
        params = {"wmax": 64.0, "nwplanes": 9, "oversample": os_, "maxsupport": 128, "wmaxclip": True}
        okw = None
        wscale = 16.0
        nclip = 40
    else:
        params = {"wmax": 64.0, "nwstacks": 9, "nwplanes": 9, "oversample": os_, "maxsupport": 128}
        okw = {"nwstacks": 9}
        wscale = 16.0                # stack spacing; inner planes every 2 wavelengths
        nclip = 0
    uvw, freq = _tie_dataset(nx, cellu, wscale, nclip, inner=0.0 if kind == "WProject" else 2.0)
    nrow = uvw.shape[0]
    rng = np.random.default_rng(2)
    vis = np.asfortranarray((rng.standard_normal((nrow, 2, 1)) + 1j * rng.standard_normal((nrow, 2, 1)))
                            .astype(np.complex64))
    og, gg = make_pair(kind, params, oracle_kw=okw)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.build_cf()
    acc = Accessor(uvw, freq, vis).to_device()
    plan = gg.plan(acc)
    iu, iv, cfi, st = plan.samples(gg, acc)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.init_cf()
    S = og.cache.support
    assert gg.support()[0] == S
    oiu, oiv, ofu, ofv = oracle.indices(uvw, freq, og.uvcell[0], og.uvcell[1], og.os, nx, nx)
    cmap, gmap = og._maps(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    plane = cmap.astype(np.int64)
    gind = np.zeros_like(plane) if gmap is None else gmap.astype(np.int64)
    # the ties are really there: uScaled on k + 1/2 and on oversampling ties,
    # fracu = 0 after folding, and w on plane (and stack) boundaries
    us = freq[None, :] * uvw[:, 0:1] / (C * cellu)
    assert np.any(np.modf(np.abs(us))[0] == 0.5)
    assert np.any(np.modf(np.abs(us * os_))[0] == 0.5)
    wf = (uvw[:, 2:3] / C) * freq[None, :]
    assert np.any(np.modf(np.abs(wf / 16.0))[0] == 0.5)
    if kind == "WProject":
        assert np.any(plane < 0)                      # clipped at the edge
    else:
        # residual w inside its stack on a tie of the inner planes (spacing 2)
        res = wf - (gind - 4) * 16.0
        assert np.any(np.modf(np.abs(res / 2.0))[0] == 0.5)
    okplane = (plane >= 0) & (gind >= 0)
    on = okplane & (oiu - S > 0) & (oiv - S > 0) & (oiu + S < nx) & (oiv + S < nx)
    # the strict on-grid edge is met from both sides on both axes
    for a in (oiu, oiv):
        assert np.any(okplane & (a - S == 0)) and np.any(okplane & (a - S == 1))
        assert np.any(okplane & (a + S == nx)) and np.any(okplane & (a + S == nx - 1))
    ocfi = ofu + os_ * (ofv + os_ * plane)
    exp_st = np.where(~okplane, 1, np.where(on, 3, 2)).astype(np.uint8)
    assert np.array_equal(st, exp_st)
    assert np.array_equal(iu[on], oiu[on])
    assert np.array_equal(iv[on], oiv[on])
    assert np.array_equal(cfi[on], ocfi[on])
    # values: grid and degrid through the same plan-free calls
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.grid(Accessor(uvw, freq, vis))
    og.grid(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    _check_grid(og, gg)
    start = np.asfortranarray(np.zeros_like(vis))
    chunk = dict(uvw=uvw, freq=freq, vis=vis)
    vg, vc = _degrid_taps(og, gg, chunk, start, cell, _point_model(nx, 1, 1))
    assert rel_l2(vg, vc) < TOL, rel_l2(vg, vc)


def test_config1_geometry_subset(ygmod, oracle_mod):
    """The benchmark's headline geometry on a seeded 1% row subset: 36
    antennas in a 6 km disk, 8 h at 5 s, 96 channels 700-1000 MHz, 4
    polarisations; WStackWProject 4096^2 at 4", 17 w-stacks x 33 w-planes,
    oversample 8, cutoff 1e-3; device-resident chunk, 32-cell uv tiles (the
    benchmark's tuned tile), so the grid and degrid passes run the same
    kernel instantiations as the timed step (support 6: 13-wide CFs in
    16-wide planes, all four polarisations in one pass)."""
    import oracle
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, Axes
    arr = simulate.random_disk_array(36, 6000.0, -26.7, 1)
    uvw, ntime, nbl = simulate.uvw_track(arr, -45.0 * simulate.DEG, 8 * 3600.0, 5.0)
    freq = 700e6 + (np.arange(96) + 0.5) * 300e6 / 96
    wmax = math.ceil(float(np.max(np.abs(uvw[:, 2]))) * freq.max() / C * 1.02 / 100.0) * 100.0
    rng = np.random.default_rng(20240)
    rows = np.sort(rng.choice(uvw.shape[0], uvw.shape[0] // 100, replace=False))
    uvw = np.ascontiguousarray(uvw[rows])
    nrow = len(rows)
    vis = np.asfortranarray((rng.standard_normal((nrow, 96, 4)) + 1j * rng.standard_normal((nrow, 96, 4)))
                            .astype(np.complex64))
    nx, cell = 4096, 4.0 * ARCSEC
    params = {"wmax": wmax, "nwstacks": 17, "nwplanes": 33, "oversample": 8, "cutoff": 1e-3, "maxsupport": 512}
    og, gg = make_pair("WStackWProject", params, oracle_kw={"nwstacks": 17})
    gg.set_tile(32)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 4, 1))
    acc = Accessor(uvw, freq, vis).to_device()
    plan = gg.plan(acc)
    gg.grid_plan(plan, acc)
    og.initialise_grid(nx, nx, 4, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    assert og.cache.support == 6 and gg.support()[0] == 6
    assert plan.info()["tile"] == 32
    # indices and statuses
    iu, iv, cfi, st = plan.samples(gg, acc)
    oiu, oiv, ofu, ofv = oracle.indices(uvw, freq, og.uvcell[0], og.uvcell[1], og.os, nx, nx)
    cmap, gmap = og._maps(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    S = 6
    okplane = (cmap >= 0) & (gmap >= 0)
    on = okplane & (oiu - S > 0) & (oiv - S > 0) & (oiu + S < nx) & (oiv + S < nx)
    ocfi = ofu + 8 * (ofv + 8 * cmap.astype(np.int64))
    mism = int((st != np.where(~okplane, 1, np.where(on, 3, 2))).sum() + (iu[on] != oiu[on]).sum()
               + (iv[on] != oiv[on]).sum() + (cfi[on] != ocfi[on]).sum())
    assert mism == 0, mism
    # grid: compared plane by plane (17 x 512 MiB)
    gpu = gg.grids()
    num = den = 0.0
    for a, b in zip(gpu, og.grids):
        num += float(np.linalg.norm((a - b).ravel()) ** 2)
        den += float(np.linalg.norm(b.ravel()) ** 2)
    gerr = math.sqrt(num / den)
    assert gerr < TOL, gerr
    assert np.array_equal(gg.sum_weights(), og.sumw)
    del gpu
    # degrid a point model (200 sources inside the inner half of the field)
    # through the plan; the oracle degrids the GPU's own transformed grids
    import torch
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), _point_model(nx, 4, 1, n=200))
    out = torch.zeros_like(acc.vis)
    accm = Accessor(acc.uvw, acc.freq, out, shape=(nrow, 96, 4))
    gd.degrid_plan(plan, accm)
    vg = accm.vis_numpy()
    og.grids = [np.asfortranarray(g) for g in gd.grids()]
    del gd
    og.model_empty = False
    og.carry = None
    vc = np.zeros_like(vis)
    og.degrid(oracle.Chunk(uvw=uvw, freq=freq, vis=vc))
    assert np.abs(vc).max() > 0
    verr = rel_l2(vg, vc)
    assert verr < TOL, verr


@pytest.mark.parametrize("kind,npol", [("WProject", 1), ("WProject", 2), ("WStackWProject", 2)])
def test_preconditioner_function_gridder(ygmod, oracle_mod, kind, npol):
    """initialiseGrid(dopcf = true): the weights are gridded without the MFS
    factor, with the conjugate CF where (iv < ny/2 and iu >= nx/2) or
    (iv <= ny/2 and iu < nx/2), and nothing is added to the sums of weights
    (TableVisGridder.cc:825-851).  An MFS weight is configured to show that
    the preconditioner ignores it."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(npol=npol, nchan=3, seed=51)
    flag, noise, delay = _flags_noise_delay(ds, seed=11)
    wmax = _wmax(ds.uvw, ds.freq)
    nx, cell = 512, 10.0 * ARCSEC
    params = {"wmax": wmax, "nwplanes": 9, "oversample": 4, "maxsupport": 256}
    okw = None
    if kind == "WStackWProject":
        params["nwstacks"] = 5
        okw = {"nwstacks": 5}
    og, gg = make_pair(kind, params, oracle_kw=okw)
    gg.initVisWeights(850e6)
    gg.customiseForContext("image.i.field.taylor.1")
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, npol, 1), dopcf=True)
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=noise, flag=flag, delay=delay)
    gg.grid(acc)
    og.initialise_grid(nx, nx, npol, 1, cell, cell, dopcf=True)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=noise, flag=flag, delay=delay))
    gpu = np.stack(gg.grids())
    ref = np.stack(og.grids)
    assert np.abs(ref).max() > 0
    err = rel_l2(gpu, ref)
    assert err < TOL, err
    assert not gg.sum_weights().any() and not og.sumw.any()
    # the conjugate half is what sets it apart from the PSF of the same weights
    _, gp = make_pair(kind, params, oracle_kw=okw)
    gp.initialiseGrid(Axes(cell, cell), (nx, nx, npol, 1), dopsf=True)
    gp.grid(acc)
    assert rel_l2(gpu, np.stack(gp.grids())) > 1e-3
    # a preconditioner gridder does not degrid
    gd = gg.clone()
    with pytest.raises(Exception):
        gd.degrid(Accessor(ds.uvw, ds.freq, np.zeros_like(ds.vis)))


@pytest.mark.parametrize("variant,pcf,direct", [(65, False, False), (65, True, False), (66, False, False),
                                                (67, True, False), (193, False, False), (194, True, False),
                                                (49, False, False), (17, False, False), (193, False, True),
                                                (65, True, True)])
def test_grid_record_orders_against_oracle(ygmod, oracle_mod, variant, pcf, direct):
    """The k_grid variants the autotuner may pick, each against the oracle on
    flagged, weighted, phase-rotated data with 4 polarisations: 65 (records in
    plane-major order, each CF plane's oversampling offsets staged in shared
    memory, register accumulation; 7-wide CFs in 16-wide rows), 66 and 67
    (two polarisation groups, two rows per thread), 193 and 194 (the same
    with the tile in global memory, reductions at each flush), 49
    (position-major records, taps through L2) and 17 (register accumulation
    over the CF-major records).  Grids 1e-5, sums of weights exact; the
    preconditioner's conjugate half through the plane-major kernel.  direct:
    through grid() itself, whose plan serves gridding only and, for the
    plane-major kernel, is sorted once by the plane-major key."""
    from yandasoft_b200.gridder import Accessor, Axes
    import oracle
    ds = _data(npol=4, nchan=4, seed=61, duration=300.0)
    flag, noise, delay = _flags_noise_delay(ds, seed=13)
    wmax = _wmax(ds.uvw, ds.freq)
    nx, cell = 1024, 6.0 * ARCSEC
    params = {"wmax": wmax, "nwstacks": 9, "nwplanes": 9, "oversample": 8, "maxsupport": 512}
    og, gg = make_pair("WStackWProject", params, oracle_kw={"nwstacks": 9})
    gg.set_grid_variant(variant)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 4, 1), dopcf=pcf)
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=noise, flag=flag, delay=delay).to_device()
    if direct:
        gg.grid(acc)
    else:
        plan = gg.plan(acc)
        gg.grid_plan(plan, acc)
    og.initialise_grid(nx, nx, 4, 1, cell, cell, dopcf=pcf)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=noise, flag=flag, delay=delay))
    assert gg.support()[0] == og.cache.support <= 7
    gpu = np.stack(gg.grids())
    ref = np.stack(og.grids)
    assert np.abs(ref).max() > 0
    err = rel_l2(gpu, ref)
    assert err < TOL, err
    assert np.array_equal(gg.sum_weights(), og.sumw)


@pytest.mark.parametrize("variant,npol", [(0, 4), (256, 4), (0, 2), (0, 1), (256, 1)])
def test_degrid_kernels_against_oracle(ygmod, oracle_mod, variant, npol):
    """Both degrid kernels of 16-wide CFs against the oracle on flagged,
    phase-rotated data: the default (each lane keeps its column of the
    segment's CF plane in registers, two samples per warp pass, one per
    half-warp) and variant 256 (the CF read from the segment ring per tap).
    Segments of odd length leave one half-warp idle on their last pass; the
    run lengths here are mostly short and odd.  Visibilities 1e-5, added
    into a non-zero starting cube as the reference adds them."""
    from yandasoft_b200.gridder import Accessor, Axes
    import oracle
    ds = _data(npol=npol, nchan=4, seed=71, duration=240.0)
    flag, noise, delay = _flags_noise_delay(ds, seed=17)
    wmax = _wmax(ds.uvw, ds.freq)
    nx, cell = 1024, 6.0 * ARCSEC
    params = {"wmax": wmax, "nwstacks": 5, "nwplanes": 9, "oversample": 8, "maxsupport": 512}
    og, gg = make_pair("WStackWProject", params, oracle_kw={"nwstacks": 5})
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, npol, 1))
    og.initialise_grid(nx, nx, npol, 1, cell, cell)
    model = _point_model(nx, npol, 1, seed=3, n=40)
    gd = gg.clone()
    gd.set_grid_variant(variant)
    gd.initialiseDegrid(Axes(cell, cell), model)
    assert gd.support()[0] <= 7
    rng = np.random.default_rng(2)
    start = np.asfortranarray((rng.standard_normal(ds.vis.shape) + 1j * rng.standard_normal(ds.vis.shape))
                              .astype(np.complex64))
    vg = np.asfortranarray(start.copy())
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=noise, flag=flag, delay=delay))
    og.grids = [np.asfortranarray(g) for g in gd.grids()]
    og.model_empty = False
    og.carry = None
    vc = np.asfortranarray(start.copy())
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=noise, flag=flag, delay=delay))
    assert rel_l2(vc, start) > 1e-3
    err = rel_l2(vg - start, vc - start)
    assert err < TOL, err
    assert rel_l2(vg, vc) < TOL
