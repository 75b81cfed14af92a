"""The learned-CF restatement (oracle/learned.py) checked on the CPU: its
analytic gradient against central finite differences in FP64, and Adam
against the published update rule."""
import numpy as np


def test_gradient_matches_finite_differences():
    from oracle import learned as L
    rng = np.random.default_rng(3)
    p = L.init_params(1)
    # weights exactly representable in FP16, so rounding does not perturb the difference quotient
    p = L.round16(p)
    X = rng.uniform(-1, 1, (7, L.NIN)).astype(np.float32)
    T = rng.uniform(-1, 1, (7, L.NOUT)).astype(np.float32)
    # the calculus of the backward pass, without the FP16 rounding of the
    # activations (whose gradient is passed straight through)
    _, g = L.loss_and_grad(p, X, T, scale=0.5, round_act=False)
    idx = np.concatenate([rng.choice(np.arange(L.OFF[k], L.OFF[k] + n), min(4, n), replace=False)
                          for k, n in [("W0", 40), ("b0", 40), ("W1", 40), ("b2", 40), ("W3", 40), ("Wo", 40),
                                       ("bo", 2)]])
    base = p.astype(np.float64)

    def lossd(q):
        # forward in FP64 on unrounded weights (the step is below FP16 resolution)
        d = L.unpack(q)
        z = L.OMEGA0 * (X.astype(np.float64) @ d["W0"] + d["b0"])
        h = np.sin(z)
        for k in range(1, L.NHID + 1):
            h = np.sin(h @ d["W%d" % k] + d["b%d" % k])
        y = h @ d["Wo"] + d["bo"]
        return 0.5 * float(np.sum((y - T) ** 2))
    for i in idx:
        e = 1e-6
        qp, qm = base.copy(), base.copy()
        qp[i] += e
        qm[i] -= e
        fd = (lossd(qp) - lossd(qm)) / (2 * e)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_padding_columns_have_no_gradient():
    from oracle import learned as L
    rng = np.random.default_rng(4)
    p = L.init_params(2)
    X = rng.uniform(-1, 1, (5, L.NIN)).astype(np.float32)
    T = rng.uniform(-1, 1, (5, L.NOUT)).astype(np.float32)
    _, g = L.loss_and_grad(p, X, T)
    for k in range(1, L.NHID + 1):
        gw = g[L.OFF["W%d" % k]:L.OFF["W%d" % k] + L.H * L.HP].reshape(L.H, L.HP)
        assert np.all(gw[:, L.H:] == 0)


def test_adam_step_rule():
    from oracle import learned as L
    p = L.init_params(0)
    g = np.linspace(-1, 1, L.NPARAM)
    m = np.zeros(L.NPARAM)
    v = np.zeros(L.NPARAM)
    p0 = p.copy()
    L.adam(p, g, m, v, 1, 1e-3)
    # first step: m_hat = g, v_hat = g^2, so each weight moves by lr * sign(g)
    live = np.ones(L.NPARAM, dtype=bool)
    for k in range(1, L.NHID + 1):
        live[L.OFF["W%d" % k]:L.OFF["W%d" % k] + L.H * L.HP].reshape(L.H, L.HP)[:, L.H:] = False
    sel = live & (np.abs(g) > 1e-3)
    assert np.allclose(np.abs(p0 - p)[sel], 1e-3, rtol=1e-3)
    assert np.all(p[~live] == 0)


def test_tap_inputs_continuous_offset():
    from oracle import learned as L
    # fraction fu of tap jx sits between taps jx and jx + 1: u = (jx - S + fu/os) / (S + 1)
    x = L.tap_inputs(np.array([3, 3, 4]), np.array([0, 0, 0]), np.array([0, 2, 0]), 0, 4, 3, 100.0, 200.0)
    assert np.allclose(x[:, 0], [0.0, 0.125, 0.25])
    assert np.allclose(x[:, 2], 0.5)
