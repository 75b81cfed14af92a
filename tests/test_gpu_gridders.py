"""SphFunc, WStack, WStack+WProject and AWProject on the GPU against the
oracle, plus the reference's error conditions, PSF and MFS weighting.

Tolerances as for WProject: indices bit-exact (checked through sums of
weights, which count every gridded sample), grids and visibilities 1e-5
relative L2, CF taps 1e-5 of each plane's peak."""
import math

import numpy as np
import pytest

from parity_helpers import ARCSEC, degrid_error_bound, make_pair, rel_l2, snapped_model

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _data(duration=300.0, nchan=4, npol=1, seed=5, f0=940e6, f1=948e6, diameter=6000.0):
    from yandasoft_b200 import simulate
    return simulate.make_dataset(duration_s=duration, nchan=nchan, npol=npol, seed=seed, freq0=f0, freq1=f1,
                                 diameter_m=diameter)


def _wmax(ds):
    from yandasoft_b200 import simulate
    return float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05


def _run_pair(kind, params, ds, nx, cell, npol, generic=None, oracle_kw=None):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    og, gg = make_pair(kind, params, oracle_kw=oracle_kw, generic=generic)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, npol, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag))
    og.initialise_grid(nx, nx, npol, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    return og, gg


def _check_grid(og, gg):
    gpu = gg.grids()
    assert len(gpu) == len(og.grids)
    err = rel_l2(np.stack(gpu), np.stack(og.grids))
    assert err < TOL, err
    assert np.array_equal(gg.sum_weights(), og.sumw)


def _check_degrid(og, gg, ds, model, cell):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vg = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=ds.noise, flag=ds.flag))
    og.initialise_degrid(model, cell, cell)
    # the FFT side (model -> grids) and the tap side (grids -> visibilities) separately;
    # og2 is cloned before og degrids, so both start from the value og carried from gridding
    ginit = rel_l2(np.stack(gd.grids()), np.stack(og.grids))
    og2 = _clone_oracle(og)
    og2.grids = [np.asfortranarray(g) for g in gd.grids()]
    vc = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=ds.noise, flag=ds.flag))
    vt = np.zeros_like(ds.vis)
    og2.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vt, noise=ds.noise, flag=ds.flag))
    assert np.abs(vc).max() > 0
    taps = rel_l2(vg, vt)
    err = rel_l2(vg, vc)
    worst = np.unravel_index(np.argmax(np.abs(vg - vt)), vg.shape)
    msg = "grid init %.3g, taps %.3g (worst sample %s: gpu %s oracle %s), end to end %.3g" % (
        ginit, taps, worst, vg[worst], vt[worst], err)
    assert ginit < TOL and taps < TOL and err < TOL, msg


def _clone_oracle(og):
    """A copy of the oracle gridder as the reference's copy constructor makes
    it: the carried image-frame visibility is copied (TableVisGridder.cc:156)."""
    import copy
    c = copy.copy(og)
    c.carry = None if og.carry is None else og.carry.copy()
    return c


# ---- SphFunc ---------------------------------------------------------------
def test_sphfunc_grid_degrid(ygmod, oracle_mod):
    ds = _data(duration=120.0, nchan=2, npol=2)
    nx, cell = 512, 6.0 * ARCSEC
    og, gg = _run_pair("SphFunc", {"oversample": 128, "support": 3}, ds, nx, cell, 2)
    _check_grid(og, gg)
    model, _ = snapped_model(ds, nx, cell, npol=2, max_nu=0.5, extra=8)
    _check_degrid(og, gg, ds, model, cell)


def test_sphfunc_degrid_edge_sources_within_fp32_bound(ygmod, oracle_mod):
    """Sources out to the image edge: the spheroidal correction (up to ~1e3)
    makes the tap sum ill-conditioned, so the bar is the FP32 summation bound
    of each sample, 2 n u sum|CF||grid| (n taps, u = 2^-24, both sides rounding),
    rather than a relative error."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=2, npol=2)
    nx, cell = 512, 6.0 * ARCSEC
    og, gg = _run_pair("SphFunc", {"oversample": 128, "support": 3}, ds, nx, cell, 2)
    model, _ = snapped_model(ds, nx, cell, npol=2, extra=8)
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vg = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=ds.noise, flag=ds.flag))
    grids = [np.asfortranarray(g) for g in gd.grids()]
    og.grids = grids
    og.carry = None
    vt = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vt, noise=ds.noise, flag=ds.flag))
    bound = degrid_error_bound(og, ds, grids, cell, nx)
    on = bound > 0
    assert on.sum() > 0.9 * on.size
    n = 49
    excess = np.abs(vg - vt)[on] / (2 * n * 2.0 ** -24 * bound[on] + 1e-30)
    assert excess.max() <= 1.0, excess.max()


def test_sphfunc_full_pol_known_answer(ygmod):
    """ImageFFTEquationTest::testFullPol on the GPU: (1, 0.01, -0.01, 0.9) to 1e-5."""
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    npix = 512
    img = np.zeros((npix, npix, 4, 1), dtype=np.float32, order="F")
    vals = [1.0, 0.01, -0.01, 0.9]
    for p, v in enumerate(vals):
        img[npix // 2, npix // 2, p, 0] = v
    g = VisGridderFactory.make({"gridder": "SphFunc"})
    g.initialiseDegrid(Axes(8 * ARCSEC, 8 * ARCSEC), img)
    rng = np.random.default_rng(3)
    nrow = 400
    uvw = np.zeros((nrow, 3))
    uvw[:, :2] = rng.uniform(-2000, 2000, (nrow, 2))
    uvw[:, 2] = rng.uniform(-500, 500, nrow)
    freq = np.array([1.4e9, 1.41e9])
    vis = np.full((nrow, 2, 4), -10 + 15j, dtype=np.complex64, order="F")
    before = vis.copy()
    g.degrid(Accessor(uvw, freq, vis))
    out = vis - before
    for p, v in enumerate(vals):
        assert np.max(np.abs(out[:, :, p] - v)) < 1e-5


# ---- WStack ----------------------------------------------------------------
def test_wstack_grid_degrid_finalise(ygmod, oracle_mod):
    ds = _data(duration=180.0, nchan=2)
    nx, cell = 1024, 6.0 * ARCSEC
    og, gg = _run_pair("WStack", {"wmax": _wmax(ds), "nwplanes": 9}, ds, nx, cell, 1)
    _check_grid(og, gg)
    img_gpu = gg.finaliseGrid()
    og.grids = [g.copy() for g in gg.grids()]
    img_cpu = og.finalise_grid()
    # correction removed as in the WProject test: compare the stacked transforms
    from oracle import cf as cfm
    cx, cy = cfm.sph_correction_vectors((nx, nx), og.grdsf)
    corr = (cx[:, None] * cy[None, :])[:, :, None, None]
    assert rel_l2(img_gpu / corr, img_cpu / corr) < 1e-4
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=8)
    _check_degrid(og, gg, ds, model, cell)


# ---- WStack + WProject -------------------------------------------------------
def test_wstack_wproject_grid_degrid(ygmod, oracle_mod):
    ds = _data(duration=300.0, nchan=4, npol=4, f0=700e6, f1=1000e6)
    nx, cell = 1024, 6.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwstacks": 9, "nwplanes": 9, "oversample": 4, "maxsupport": 256}
    og, gg = _run_pair("WStackWProject", params, ds, nx, cell, 4, oracle_kw={"nwstacks": 9})
    assert gg.support()[0] == og.cache.support
    _check_grid(og, gg)
    model, _ = snapped_model(ds, nx, cell, npol=4, max_nu=0.5, extra=8)
    _check_degrid(og, gg, ds, model, cell)


# ---- AWProject with disk illumination -----------------------------------------
def test_awproject_cf_grid_degrid(ygmod, oracle_mod):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=2, seed=9, diameter=2000.0)
    nrow = ds.nrow
    feed = (np.arange(nrow) % 2).astype(np.int32)       # two beams
    pnt = np.zeros((nrow, 2))
    pnt[feed == 1, 0] = 0.5 * math.pi / 180               # second beam offset by 0.5 deg in ra
    nx, cell = 512, 10.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 5, "oversample": 4, "maxsupport": 256, "maxfeeds": 2,
              "diameter": "25m", "blockage": "2m", "cutoff": 1e-3}
    og, gg = make_pair("AWProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt))
    assert gg.support()[0] == og.cache.support
    cpu = og.cache.cfs
    gpu = gg.convolution_functions()
    worst = 0.0
    for a, b in zip(cpu, gpu):
        if a is None:
            continue
        worst = max(worst, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
    assert worst < TOL, worst
    _check_grid(og, gg)
    # finaliseWeights: CF-weighted sum of |IFFT(CF)|^2, Fourier-padded from 256^2 to 512^2
    wg = gg.finaliseWeights()
    wc = og.finalise_weights()
    assert np.max(wc) > 0
    assert rel_l2(wg, wc) < 1e-4, rel_l2(wg, wc)


def test_awproject_spheroidal_taper(ygmod, oracle_mod):
    """AWProject with spheroidaltaper: the anti-aliasing spheroidal multiplies
    the image-plane screen inside the central qnx x qny region
    (AWProjectVisGridder.cc:338-354, :405-414), finaliseGrid and
    initialiseDegrid apply the SphFunc grid correction, and finaliseWeights
    divides the taper (cut at spheroidalweightscutoff) out of every
    transformed CF."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=2, seed=9, diameter=2000.0)
    nrow = ds.nrow
    feed = (np.arange(nrow) % 2).astype(np.int32)
    pnt = np.zeros((nrow, 2))
    pnt[feed == 1, 0] = 0.5 * math.pi / 180
    nx, cell = 512, 10.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 5, "oversample": 4, "maxsupport": 256, "maxfeeds": 2,
              "diameter": "25m", "blockage": "2m", "cutoff": 1e-3, "spheroidaltaper": True,
              "spheroidalweightscutoff": 1e-3}
    og, gg = make_pair("AWProject", params, oracle_kw={"spheroidaltaper": True, "spheroidalweightscutoff": 1e-3})
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt)
    gg.grid(acc)
    chunk = oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(chunk)
    assert gg.support()[0] == og.cache.support
    worst = 0.0
    for a, b in zip(og.cache.cfs, gg.convolution_functions()):
        if a is None:
            continue
        worst = max(worst, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
    assert worst < TOL, worst
    _check_grid(og, gg)
    wg = gg.finaliseWeights()
    wc = og.finalise_weights()
    assert np.max(wc) > 0
    assert rel_l2(wg, wc) < 1e-4, rel_l2(wg, wc)
    # finaliseGrid with the grid correction, on the GPU's own grid
    grid = gg.grids()[0]
    img_gpu = gg.finaliseGrid()
    og.grids = [grid.copy()]
    img_cpu = og.finalise_grid()
    from oracle import cf as cfm
    cx, cy = cfm.sph_correction_vectors(grid.shape, og.grdsf)
    corr = (cx[:, None] * cy[None, :])[:, :, None, None]
    safe = np.where(corr == 0, 1.0, corr)
    assert rel_l2(img_gpu / safe, img_cpu / safe) < TOL
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=4)
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vg = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    og.initialise_degrid(model, cell, cell)
    vc = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=ds.noise, flag=ds.flag, feed1=feed,
                           pointing=pnt))
    assert np.abs(vc).max() > 0
    assert rel_l2(vg, vc) < TOL, rel_l2(vg, vc)


def test_padding(ygmod, oracle_mod):
    """gridder.padding = 2: the gridder works on the padded shape
    (TableVisGridder.cc:1002, paddedShape), so its grid equals the oracle's at
    twice the size with the same cell; finaliseGrid returns the centre of the
    padded image and initialiseDegrid pads the model with zeros."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=300.0, nchan=4)
    nx, cell = 256, 20.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 9, "oversample": 4, "maxsupport": 256}
    og, gg = make_pair("WProject", params, generic={"gridder.padding": 2.0})
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag))
    og.initialise_grid(2 * nx, 2 * nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    assert gg.grids()[0].shape[:2] == (2 * nx, 2 * nx)
    _check_grid(og, gg)
    grid = gg.grids()[0]
    img = gg.finaliseGrid()
    assert img.shape[:2] == (nx, nx)
    og.grids = [grid.copy()]
    full = og.finalise_grid()
    centre = full[nx // 2:nx // 2 + nx, nx // 2:nx // 2 + nx]
    from oracle import cf as cfm
    cx, cy = cfm.sph_correction_vectors(grid.shape, og.grdsf)
    corr = (cx[:, None] * cy[None, :])[nx // 2:nx // 2 + nx, nx // 2:nx // 2 + nx, None, None]
    safe = np.where(corr == 0, 1.0, corr)
    assert rel_l2(img / safe, centre / safe) < TOL
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=4)
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vg = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=ds.noise, flag=ds.flag))
    big = np.zeros((2 * nx, 2 * nx, 1, 1), dtype=np.float32, order="F")
    big[nx // 2:nx // 2 + nx, nx // 2:nx // 2 + nx] = model
    og.initialise_degrid(big, cell, cell)
    vc = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=ds.noise, flag=ds.flag))
    assert np.abs(vc).max() > 0
    assert rel_l2(vg, vc) < TOL, rel_l2(vg, vc)


# ---- WProject parset variants ---------------------------------------------------
# (parset keys, oracle keywords, generic keys): non-linear w-sampling
# (PowerWSampling, GaussianWSampling), per-plane supports with peak offsets,
# limitsupport, an absolute cutoff and sums of weights per oversampling offset
_VARIANTS = {
    "powerlaw": ({"wsampling": "powerlaw", "wsampling.exponent": 0.5}, {"wsampling": "powerlaw", "exponent": 0.5},
                 None),
    "gaussian": ({"wsampling": "gaussian", "wsampling.nwplanes50": 4.0},
                 {"wsampling": "gaussian", "nwplanes50": 4.0}, None),
    "variable_offset_support": ({"variablesupport": True, "offsetsupport": True}, {}, None),
    "limitsupport": ({"limitsupport": 8}, {}, None),
    "cutoff_absolute": ({"cutoff.absolute": True}, {}, None),
    "oversampleweight": ({}, {}, {"gridder.oversampleweight": True}),
}


@pytest.mark.parametrize("variant", sorted(_VARIANTS))
def test_wproject_parset_variants(ygmod, oracle_mod, variant):
    keys, okw, generic = _VARIANTS[variant]
    ds = _data(duration=300.0, nchan=4)
    nx, cell = 512, 20.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 9, "oversample": 4, "maxsupport": 256, "cutoff": 1e-3}
    params.update(keys)
    og, gg = _run_pair("WProject", params, ds, nx, cell, 1, generic=generic, oracle_kw=okw)
    cpu = og.cache.cfs
    gpu = gg.convolution_functions()
    assert [c.shape for c in cpu] == [c.shape for c in gpu]
    worst = max(float(np.max(np.abs(a - b)) / np.max(np.abs(a))) for a, b in zip(cpu, gpu))
    assert worst < TOL, worst
    _check_grid(og, gg)
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=4)
    _check_degrid(og, gg, ds, model, cell)


def test_awproject_36_beam_footprint(ygmod, oracle_mod):
    """The 36-beam AWProject case at reduced size, gridded as one mosaic:
    12 m dishes with 1 m blockage, a 6 x 6 beam footprint at 0.9 deg pitch
    (beams observed in turn, one integration each), 4 channels over
    700-1000 MHz with a CF set per channel, 2 polarisations, 33 w-planes,
    oversample 4.  Reduced (2 km array, 5 min track, 256^2 grid at 30") so
    that the oracle's 76,032 CF matrices take seconds.  The first row's beam
    is the footprint's corner, whose w-plane 0 sets the common support."""
    import oracle
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, Axes
    ds = simulate.make_dataset(duration_s=300.0, dt_s=5.0, nchan=4, npol=2, seed=21, freq0=700e6, freq1=1000e6,
                               diameter_m=2000.0)
    foot = simulate.beam_footprint(6, 0.9)
    feed = simulate.multibeam_rows(ds.ntime, ds.nbl, 36)
    pnt = foot[feed]
    nx, cell = 256, 30.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 33, "oversample": 4, "maxsupport": 256, "maxfeeds": 36,
              "diameter": "12m", "blockage": "1m", "cutoff": 1e-3}
    og, gg = make_pair("AWProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 2, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    og.initialise_grid(nx, nx, 2, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt))
    assert gg.support()[0] == og.cache.support
    cpu = og.cache.cfs
    gpu = gg.convolution_functions()
    assert len(cpu) == len(gpu) == 36 * 4 * 33 * 16
    worst = 0.0
    for a, b in zip(cpu, gpu):
        worst = max(worst, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
    assert worst < TOL, worst
    _check_grid(og, gg)
    # degrid a model of points at the central beams' centres through a clone
    model = np.zeros((nx, nx, 2, 1), dtype=np.float32, order="F")
    for k, (dx, dy) in enumerate(foot):
        x, y = nx // 2 + int(round(dx / cell)), nx // 2 + int(round(dy / cell))
        if 0 <= x < nx and 0 <= y < nx:
            model[x, y, :, 0] = 0.1 + 0.01 * k
    assert np.count_nonzero(model) > 0
    gd = gg.clone()
    gd.initialiseDegrid(Axes(cell, cell), model)
    vg = np.zeros_like(ds.vis)
    gd.degrid(Accessor(ds.uvw, ds.freq, vg, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    og.initialise_degrid(model, cell, cell)
    vc = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vc, noise=ds.noise, flag=ds.flag, feed1=feed,
                           pointing=pnt))
    assert np.abs(vc).max() > 0
    assert rel_l2(vg, vc) < TOL, rel_l2(vg, vc)


# ---- error conditions (ASKAPCHECK) ------------------------------------------
def test_w_out_of_range_raises(ygmod):
    from yandasoft_b200.gridder import Accessor, AskapError, Axes, VisGridderFactory
    ds = _data(duration=60.0, nchan=1)
    g = VisGridderFactory.make({"gridder": "WProject", "gridder.WProject.wmax": 10.0, "gridder.WProject.nwplanes": 3,
                                "gridder.WProject.oversample": 4, "gridder.WProject.maxsupport": 256})
    g.initialiseGrid(Axes(30 * ARCSEC, 30 * ARCSEC), (512, 512, 1, 1))
    with pytest.raises(AskapError) as e:
        g.grid(Accessor(ds.uvw, ds.freq, ds.vis))
    assert e.value.code == 4


def test_wmaxclip_skips(ygmod, oracle_mod):
    ds = _data(duration=60.0, nchan=1)
    nx, cell = 512, 30 * ARCSEC
    params = {"wmax": _wmax(ds) * 0.5, "nwplanes": 5, "oversample": 4, "maxsupport": 256, "wmaxclip": True}
    og, gg = _run_pair("WProject", params, ds, nx, cell, 1)
    _check_grid(og, gg)


def test_nonpositive_weight_raises(ygmod):
    from yandasoft_b200.gridder import Accessor, AskapError, Axes, VisGridderFactory
    ds = _data(duration=60.0, nchan=1)
    noise = np.asfortranarray(ds.noise.copy())
    noise[:] = 0
    g = VisGridderFactory.make({"gridder": "SphFunc"})
    g.initialiseGrid(Axes(60 * ARCSEC, 60 * ARCSEC), (512, 512, 1, 1))
    with pytest.raises(AskapError) as e:
        g.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=noise))
    assert e.value.code == 5


# ---- PSF and MFS weights -----------------------------------------------------
def test_psf_gridder(ygmod, oracle_mod):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=2)
    nx, cell = 512, 30 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 5, "oversample": 4, "maxsupport": 256}
    og, gg = make_pair("WProject", params, generic={"gridder.alldatapsf": True})
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1), dopsf=True)
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag))
    og.initialise_grid(nx, nx, 1, 1, cell, cell, dopsf=True)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    _check_grid(og, gg)


@pytest.mark.parametrize("case", ["frequency_independent", "psf_first_beam"])
def test_awproject_variants(ygmod, oracle_mod, case):
    """AWProject with frequencydependent = false (one CF set per beam, at the
    chunk's first frequency, indexed without the channel) and the PSF gridder
    (CFs without the beam-offset slope, only the rows of the first row's beam
    and pointing gridded unless alldatapsf)."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=3, seed=9, diameter=2000.0, f0=900e6, f1=1000e6)
    feed = (np.arange(ds.nrow) % 2).astype(np.int32)
    pnt = np.zeros((ds.nrow, 2))
    pnt[feed == 1, 0] = 0.5 * math.pi / 180
    nx, cell = 512, 10.0 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 5, "oversample": 4, "maxsupport": 256, "maxfeeds": 2,
              "diameter": "25m", "blockage": "2m", "cutoff": 1e-3}
    psf = case == "psf_first_beam"
    if not psf:
        params["frequencydependent"] = False
    og, gg = make_pair("AWProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1), dopsf=psf)
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    og.initialise_grid(nx, nx, 1, 1, cell, cell, dopsf=psf)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt))
    assert gg.support()[0] == og.cache.support
    worst = 0.0
    n = 0
    for a, b in zip(og.cache.cfs, gg.convolution_functions()):
        if a is None:
            continue
        n += 1
        worst = max(worst, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
    assert n > 0 and worst < TOL, worst
    if not psf:
        assert len(og.cache.cfs) == 16 * 5 * 2
    _check_grid(og, gg)


def test_mfs_weights(ygmod, oracle_mod):
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds = _data(duration=120.0, nchan=4, f0=900e6, f1=1000e6)
    nx, cell = 512, 30 * ARCSEC
    params = {"wmax": _wmax(ds), "nwplanes": 5, "oversample": 4, "maxsupport": 256}
    og, gg = make_pair("WProject", params)
    gg.initVisWeights(950e6)
    gg.customiseForContext("image.i.field.taylor.1")
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.grid(Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag))
    og.mfs = lambda f: ((np.asarray(f) - 950e6) / 950e6).astype(np.float32)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    _check_grid(og, gg)


# ---- wide CFs: the staged-CF ring (Wp 80) and taps from global memory (Wp 144) ----
def _adopt_cf(og, gg):
    """Gives the oracle the GPU's CF planes, so that the tap path is compared
    on identical taps."""
    gpu = gg.convolution_functions()
    og.cache.cfs = [None if c is None else np.asfortranarray(c) for c in gpu]
    og._flat = og.cache.flatten()


@pytest.mark.parametrize("wmax", [6000.0, 12000.0])
def test_wproject_wide_support(ygmod, oracle_mod, wmax):
    """Supports of 35 and 67 cells.  The CF planes agree to 1e-5 of each
    plane's peak; at these widths most taps are 1e-3 of the peak or less, so
    the FFT's rounding (cuFFT against the oracle's FFT) reaches ~1e-4 of the
    grid's L2 norm, and the tap path is compared on the GPU's own CFs."""
    import oracle
    ds = _data(duration=240.0, nchan=2, diameter=3000.0, seed=21)
    nx, cell = 512, 40.0 * ARCSEC
    params = {"wmax": wmax, "nwplanes": 5, "oversample": 4, "maxsupport": 1024, "cutoff": 1e-3}
    og, gg = _run_pair("WProject", params, ds, nx, cell, 1)
    assert gg.support()[0] == og.cache.support
    assert og.cache.support >= 30
    worst = 0.0
    for a, b in zip(og.cache.cfs, gg.convolution_functions()):
        worst = max(worst, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
    assert worst < TOL, worst
    end_to_end = rel_l2(np.stack(gg.grids()), np.stack(og.grids))
    assert end_to_end < 1e-3, end_to_end
    _adopt_cf(og, gg)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    _check_grid(og, gg)
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=8)
    _check_degrid(og, gg, ds, model, cell)


# ---- host chunks in row pieces (upload overlapping the passes) ----------------
def test_pipelined_host_chunk_matches_device_chunk(ygmod, oracle_mod):
    """A host chunk above the piece threshold is uploaded and processed in row
    pieces; its grid (summed in another order: 1e-5), sums of weights and
    degridded visibilities equal those of the same chunk passed
    device-resident in one piece."""
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, Axes, VisGridderFactory
    ds = simulate.make_dataset(duration_s=2 * 3600.0, nchan=48, npol=2, seed=81, diameter_m=3000.0,
                               freq0=900e6, freq1=1000e6)
    assert ds.vis.nbytes >= 300 * 2 ** 20
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    ps = {"gridder": "WProject", "gridder.WProject.wmax": wmax, "gridder.WProject.nwplanes": 9,
          "gridder.WProject.oversample": 4, "gridder.WProject.maxsupport": 256}
    nx, cell = 1024, 10.0 * ARCSEC
    axes = Axes(cell, cell)
    host = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag)
    dev = host.to_device()
    a, b = VisGridderFactory.make(ps), VisGridderFactory.make(ps)
    for g in (a, b):
        g.initialiseGrid(axes, (nx, nx, 2, 1))
    a.grid(host)
    b.grid(dev)
    assert rel_l2(np.stack(a.grids()), np.stack(b.grids())) < TOL
    assert np.array_equal(a.sum_weights(), b.sum_weights())
    model, _ = snapped_model(ds, nx, cell, npol=2, max_nu=0.5, extra=6)
    vh = np.zeros_like(ds.vis)
    a.initialiseDegrid(axes, model)
    a.degrid(Accessor(ds.uvw, ds.freq, vh, noise=ds.noise, flag=ds.flag))
    dvis = Accessor(ds.uvw, ds.freq, np.zeros_like(ds.vis), noise=ds.noise, flag=ds.flag).to_device()
    b.initialiseDegrid(axes, model)
    b.degrid(dvis)
    assert rel_l2(vh, dvis.vis_numpy()) < TOL
