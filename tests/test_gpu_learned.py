"""The learned convolution function on the GPU: the fused training kernel's
loss and gradient against the CPU restatement (oracle/learned.py), batch
inference against the restatement, training on a WProject CF table, the
in-kernel evaluation in the grid and degrid kernels judged by the tabulated
path, and what the network gains over the table (memory, continuity in w)."""
import math

import numpy as np
import pytest

from parity_helpers import ARCSEC, make_pair, rel_l2, snapped_model

pytestmark = pytest.mark.gpu


def _random_net(seed):
    from oracle import learned as L
    return L.init_params(seed)


def test_mlp_gradient_matches_oracle(ygmod, oracle_mod):
    from oracle import learned as L
    rng = np.random.default_rng(7)
    p = _random_net(3)
    n = 300                                     # several 32-tap tiles and a ragged tail
    X = rng.uniform(-1, 1, (n, L.NIN)).astype(np.float32)
    T = rng.uniform(-1, 1, (n, L.NOUT)).astype(np.float32)
    loss, g = ygmod.mlp_loss_grad(p, X, T, scale=1.0 / n)
    lref, gref = L.loss_and_grad(p, X, T, scale=1.0 / n)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    for k in ["W0", "b0", "W1", "b1", "W2", "b2", "W3", "b3", "Wo", "bo"]:
        o = L.OFF[k]
        size = {"W0": L.NIN * L.H, "Wo": L.H * L.NOUT, "bo": L.NOUT}.get(k, L.H * L.HP if k.startswith("W") else L.H)
        err = rel_l2(g[o:o + size], gref[o:o + size])
        assert err < 1e-4, (k, err)


def test_mlp_eval_matches_oracle(ygmod, oracle_mod):
    """Batch inference (the tensor-core network, 32 inputs per warp) against
    the restatement.  Both round h0, h1, h2 to FP16; an activation whose FP32
    and FP64 values fall on the two sides of an FP16 rounding boundary moves
    by one FP16 ulp (at most 2^-11 of it), which moves the output by about
    that times the weights behind it: so the bar is 1e-5 of the output scale
    for the median sample and 3e-3 for the worst of 1000."""
    from oracle import learned as L
    rng = np.random.default_rng(8)
    p = _random_net(5)
    X = rng.uniform(-1, 1, (1000, L.NIN)).astype(np.float32)
    y = ygmod.mlp_eval(p, X)
    yref, _ = L.forward(p, X)
    scale = np.max(np.abs(yref))
    err = np.abs(y - yref)
    assert np.median(err) <= 1e-5 * scale, np.median(err) / scale
    assert err.max() <= 3e-3 * scale, err.max() / scale


def _wproject_case():
    from yandasoft_b200 import simulate
    ds = simulate.make_dataset(duration_s=600.0, nchan=2, npol=1, seed=31, diameter_m=2000.0)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    return ds, {"wmax": wmax, "nwplanes": 9, "oversample": 4, "maxsupport": 256, "cutoff": 1e-3}


def _learned_cf_error(gg, params, scale, planes, os_, wterms, wnorm):
    """Relative L2 error of the network over whole CF planes of `planes`
    (a list of CF matrices indexed like the gridder's cache)."""
    from oracle import learned as L
    num = den = 0.0
    for cfi, c in enumerate(planes):
        if c is None:
            continue
        w = c.shape[0]
        S = (w - 1) // 2
        jx, jy = np.meshgrid(np.arange(w), np.arange(w), indexing="ij")
        fu, fv, pl = cfi % os_, (cfi // os_) % os_, cfi // (os_ * os_)
        X = L.tap_inputs(jx.ravel(), jy.ravel(), fu, fv, os_, S, wterms[pl], wnorm)
        from yandasoft_b200.gridder import mlp_eval
        Y = mlp_eval(params, X) * scale
        pred = (Y[:, 0] + 1j * Y[:, 1]).reshape(w, w)
        num += float(np.sum(np.abs(pred - c) ** 2))
        den += float(np.sum(np.abs(c) ** 2))
    return math.sqrt(num / den)


def test_learned_cf_training_and_in_kernel_use(ygmod, oracle_mod):
    import oracle
    from oracle import learned as L
    from yandasoft_b200.gridder import Accessor, Axes
    ds, params = _wproject_case()
    nx, cell = 512, 20.0 * ARCSEC
    og, gg = make_pair("WProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.build_cf()
    cfs = gg.convolution_functions()
    wterms = oracle.WSampling(params["nwplanes"], params["wmax"]).wterms()
    wnorm = float(np.max(np.abs(wterms)))
    # the untrained network, for comparison
    gg.set_learned_params(L.init_params(1), 1.0)
    p0, s0 = gg.learned_params()
    rep = gg.learned_train(ntrain=1 << 22, batch=16384, steps=20000, lr=1e-2, seed=2)
    p1, s1 = gg.learned_params()
    e1 = _learned_cf_error(gg, p1, s1, cfs, params["oversample"], wterms, wnorm)
    e0 = _learned_cf_error(gg, p0, s1, cfs, params["oversample"], wterms, wnorm)
    print("learned CF: rel L2 %.3e (untrained %.3e), loss %.3e, %.0f ms, table %.1f MB vs network %.1f kB"
          % (e1, e0, rep["final_loss"], rep["train_ms"], rep["cf_table_bytes"] / 1e6, rep["network_bytes"] / 1e3))
    assert e1 < 1e-3 * e0
    assert e1 < 1e-2
    # 9 planes x 16 fractions here; the table grows with planes, oversampling, beams
    # and channels, the network does not
    assert rep["network_bytes"] < 0.1 * rep["cf_table_bytes"]
    # in-kernel evaluation: grid and degrid with the network, judged by the tabulated path
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag)
    gg.grid(acc)
    plain_grid = np.stack(gg.grids()).copy()
    gl = gg.clone()
    gl.set_cf_form(1)
    gl.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gl.grid(acc)
    grid_err = rel_l2(np.stack(gl.grids()), plain_grid)
    assert np.array_equal(gl.sum_weights(), gg.sum_weights())
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=8)
    vp = np.zeros_like(ds.vis)
    vl = np.zeros_like(ds.vis)
    gd = gg.clone()
    gd.set_cf_form(0)
    gd.initialiseDegrid(Axes(cell, cell), model)
    gd.degrid(Accessor(ds.uvw, ds.freq, vp, noise=ds.noise, flag=ds.flag))
    gdl = gg.clone()
    gdl.set_cf_form(1)
    gdl.initialiseDegrid(Axes(cell, cell), model)
    gdl.degrid(Accessor(ds.uvw, ds.freq, vl, noise=ds.noise, flag=ds.flag))
    vis_err = rel_l2(vl, vp)
    print("in-kernel learned CF: grid rel error %.3e, degrid rel error %.3e vs the tabulated path" % (grid_err, vis_err))
    # the network reproduces the table to its CF error in both kernels
    assert grid_err < 2 * e1 + 1e-4
    assert vis_err < 2 * e1 + 1e-4


def test_learned_awproject_beams_and_channels(ygmod, oracle_mod):
    """AWProject: one network for every CF plane of the cache, plane z =
    w-plane + nw (channel + nchan beam) with inputs (w / wmax, frequency,
    beam), the last two mapped onto [-1, 1]; trained on the gridder's own CFs
    of two beams (0.5 deg apart) and two channels, then evaluated in the grid
    and degrid kernels (form 1) and judged by the tabulated path."""
    import oracle
    from oracle import learned as L
    from yandasoft_b200 import simulate
    from yandasoft_b200.gridder import Accessor, AskapError, Axes
    ds = simulate.make_dataset(duration_s=120.0, nchan=2, npol=1, seed=9, diameter_m=2000.0, freq0=800e6,
                               freq1=1000e6)
    feed = (np.arange(ds.nrow) % 2).astype(np.int32)
    pnt = np.zeros((ds.nrow, 2))
    pnt[feed == 1, 0] = 0.5 * math.pi / 180
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    params = {"wmax": wmax, "nwplanes": 5, "oversample": 4, "maxsupport": 256, "maxfeeds": 2,
              "diameter": "25m", "blockage": "2m", "cutoff": 1e-3}
    nx, cell = 512, 10.0 * ARCSEC
    _, gg = make_pair("AWProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    acc = Accessor(ds.uvw, ds.freq, ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt)
    gg.grid(acc)
    plain_grid = np.stack(gg.grids()).copy()
    cfs = gg.convolution_functions()
    os_, nw = 4, 5
    assert len(cfs) == os_ * os_ * nw * 2 * 2
    wterms = oracle.WSampling(nw, wmax).wterms()
    wnorm = float(np.max(np.abs(wterms)))
    gg.set_learned_params(L.init_params(1), 1.0)
    p0, _ = gg.learned_params()
    rep = gg.learned_train(ntrain=1 << 22, batch=16384, steps=20000, lr=1e-2, seed=2)
    p1, s1 = gg.learned_params()

    def cf_error(params_):
        num = den = 0.0
        for cfi, c in enumerate(cfs):
            w = c.shape[0]
            S = (w - 1) // 2
            jx, jy = np.meshgrid(np.arange(w), np.arange(w), indexing="ij")
            fu, fv, z = cfi % os_, (cfi // os_) % os_, cfi // (os_ * os_)
            iw, ch, b = z % nw, (z // nw) % 2, z // (2 * nw)
            X = L.tap_inputs(jx.ravel(), jy.ravel(), fu, fv, os_, S, wterms[iw], wnorm, freq=2.0 * ch - 1.0,
                             beam=2.0 * b - 1.0)
            Y = ygmod.mlp_eval(params_, X) * s1
            pred = (Y[:, 0] + 1j * Y[:, 1]).reshape(w, w)
            num += float(np.sum(np.abs(pred - c) ** 2))
            den += float(np.sum(np.abs(c) ** 2))
        return math.sqrt(num / den)

    e1, e0 = cf_error(p1), cf_error(p0)
    print("learned AWProject CF: rel L2 %.3e (untrained %.3e), %.0f ms" % (e1, e0, rep["train_ms"]))
    assert e1 < 0.05 * e0
    assert e1 < 5e-2
    gl = gg.clone()
    gl.set_cf_form(1)
    gl.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gl.grid(acc)
    grid_err = rel_l2(np.stack(gl.grids()), plain_grid)
    model, _ = snapped_model(ds, nx, cell, max_nu=0.5, extra=4)
    vp = np.zeros_like(ds.vis)
    vl = np.zeros_like(ds.vis)
    for form, out in ((0, vp), (1, vl)):
        gd = gg.clone()
        gd.set_cf_form(form)
        gd.initialiseDegrid(Axes(cell, cell), model)
        gd.degrid(Accessor(ds.uvw, ds.freq, out, noise=ds.noise, flag=ds.flag, feed1=feed, pointing=pnt))
    vis_err = rel_l2(vl, vp)
    print("in-kernel learned AWProject CF: grid %.3e, degrid %.3e vs the tabulated path" % (grid_err, vis_err))
    assert grid_err < 2 * e1 + 1e-4
    assert vis_err < 2 * e1 + 1e-4
    with pytest.raises(AskapError):
        gl.set_cf_form(2)


def test_learned_cf_continuous_in_w(ygmod, oracle_mod):
    """Trained on a table 4x denser in w, the network at the planes between
    the gridder's own planes is closer to the exact CF there than the nearest
    of the gridder's planes is: the gain of a continuous w kernel."""
    import oracle
    from oracle import learned as L
    from yandasoft_b200.gridder import Axes, VisGridderFactory
    ds, params = _wproject_case()
    nx, cell = 512, 20.0 * ARCSEC
    nw, nd = params["nwplanes"], 4 * (params["nwplanes"] - 1) + 1
    mk = lambda n: VisGridderFactory.make({"gridder": "WProject", **{"gridder.WProject.%s" % k: v for k, v in
                                                                      dict(params, nwplanes=n).items()}})
    coarse, dense = mk(nw), mk(nd)
    for g in (coarse, dense):
        g.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
        g.build_cf()
    assert coarse.support()[0] == dense.support()[0]
    coarse.learned_train(ntrain=1 << 22, batch=16384, steps=20000, lr=1e-2, seed=3, nwplanes_train=nd)
    p, s = coarse.learned_params()
    os_ = params["oversample"]
    dcf = dense.convolution_functions()
    ccf = coarse.convolution_functions()
    wd = oracle.WSampling(nd, params["wmax"]).wterms()
    wc = oracle.WSampling(nw, params["wmax"]).wterms()
    wnorm = float(np.max(np.abs(wc)))
    between = [k for k in range(nd) if k % 4 == 2]          # halfway between two coarse planes
    net_num = near_num = den = 0.0
    for k in between:
        near = int(np.argmin(np.abs(wc - wd[k])))
        for f in range(os_ * os_):
            exact = dcf[f + os_ * os_ * k]
            w = exact.shape[0]
            S = (w - 1) // 2
            jx, jy = np.meshgrid(np.arange(w), np.arange(w), indexing="ij")
            X = L.tap_inputs(jx.ravel(), jy.ravel(), f % os_, f // os_, os_, S, wd[k], wnorm)
            Y = ygmod.mlp_eval(p, X) * s
            pred = (Y[:, 0] + 1j * Y[:, 1]).reshape(w, w)
            net_num += float(np.sum(np.abs(pred - exact) ** 2))
            near_num += float(np.sum(np.abs(ccf[f + os_ * os_ * near] - exact) ** 2))
            den += float(np.sum(np.abs(exact) ** 2))
    e_net, e_near = math.sqrt(net_num / den), math.sqrt(near_num / den)
    print("between planes: network %.3e, nearest tabulated plane %.3e" % (e_net, e_near))
    assert e_net < 0.5 * e_near


def test_learned_continuous_closer_to_dft(ygmod, oracle_mod):
    """Evaluated at each sample's own fractional offset and w, the network
    removes the oversampling and w-plane quantisation of the table: its
    degridded visibilities are closer to the FP64 DFT than the tabulated
    path's (oversample 4, 9 planes)."""
    import oracle
    from yandasoft_b200.gridder import Accessor, Axes
    ds, params = _wproject_case()
    nx, cell = 512, 20.0 * ARCSEC
    og, gg = make_pair("WProject", params)
    gg.initialiseGrid(Axes(cell, cell), (nx, nx, 1, 1))
    gg.build_cf()
    gg.learned_train(ntrain=1 << 22, batch=16384, steps=20000, lr=1e-2, seed=4,
                     nwplanes_train=4 * (params["nwplanes"] - 1) + 1)
    model, comp = snapped_model(ds, nx, cell, max_nu=0.5, extra=8)
    ref = oracle.dft(ds.uvw, ds.freq, comp)
    out = {}
    for form in (0, 1, 2):
        g = gg.clone()
        g.set_cf_form(form)
        g.initialiseDegrid(Axes(cell, cell), model)
        v = np.zeros_like(ds.vis)
        g.degrid(Accessor(ds.uvw, ds.freq, v, noise=ds.noise, flag=ds.flag))
        out[form] = v[:, :, 0]
    uvcell = 1.0 / (cell * nx)
    iu, iv, _, _ = oracle.indices(ds.uvw, ds.freq, uvcell, uvcell, params["oversample"], nx, nx)
    s = gg.support()[0]
    on = (iu - s > 0) & (iv - s > 0) & (iu + s < nx) & (iv + s < nx)
    e = {f: rel_l2(out[f][on], ref[on]) for f in out}
    print("degrid rel error vs FP64 DFT: tabulated %.3e, learned planes %.3e, learned continuous %.3e"
          % (e[0], e[1], e[2]))
    assert e[2] < 0.5 * e[0]
