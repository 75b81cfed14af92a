"""Synthetic-data helpers of the benchmark workloads (CPU): the 36-beam
footprint, the beam of each row, and the beam power pattern that attenuates
each source (the far field of a uniformly illuminated disk with a central
blockage)."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_beam_footprint_square_and_centred():
    from yandasoft_b200 import simulate
    foot = simulate.beam_footprint(6, 0.9)
    assert foot.shape == (36, 2)
    np.testing.assert_allclose(foot.mean(axis=0), 0.0, atol=1e-15)
    pitch = 0.9 * math.pi / 180
    np.testing.assert_allclose(np.diff(np.unique(np.round(foot[:, 0] / pitch, 9))), 1.0)
    np.testing.assert_allclose(np.abs(foot).max(), 2.5 * pitch)
    # row-major: the first beam is the corner (-x, -y)
    assert foot[0, 0] < 0 and foot[0, 1] < 0


def test_multibeam_rows_cycle_per_integration():
    from yandasoft_b200 import simulate
    feed = simulate.multibeam_rows(ntime=80, nbl=630, nbeam=36)
    assert feed.dtype == np.int32 and feed.shape == (80 * 630,)
    t = np.arange(80)
    np.testing.assert_array_equal(feed[::630], t % 36)
    # every row of one integration belongs to one beam
    assert np.all(feed.reshape(80, 630) == (t % 36)[:, None])


def test_beam_power_pattern():
    import bench
    w = bench.workload(2, 0.01)
    freq = np.array([700e6, 1000e6])
    # sources at each beam centre and at the first null of an unblocked 12 m dish
    foot_src = np.zeros((2, 8))
    foot_src[0, 1:3] = 0.0
    lam = bench.C_LIGHT / 1000e6
    theta_null = 1.2196698912665045 * lam / w["dish"]
    foot_src[1, 1] = theta_null
    w0 = dict(w, blockage=0.0, nbeam=1, pitch=0.9)
    p, foot = bench.beam_power(w0, foot_src, freq)
    assert p.shape == (1, 2, 2)
    np.testing.assert_allclose(p[0, 0], 1.0, rtol=1e-12)       # the beam centre
    assert p[0, 1, 1] < 1e-8                                    # first null at 1000 MHz
    assert 0.0 < p[0, 1, 0] < 0.5                               # inside the wider main lobe at 700 MHz
    # with the 1 m blockage the centre stays at 1 and the pattern falls off monotonically in the main lobe
    p2, _ = bench.beam_power(dict(w, nbeam=1, pitch=0.9), np.array([[1, t, 0, 0, 0, 0, 0, 1] for t in
                                                                   np.linspace(0, 0.8 * theta_null, 9)], float),
                             freq[1:])
    assert abs(p2[0, 0, 0] - 1.0) < 1e-12
    assert np.all(np.diff(p2[0, :, 0]) < 0)
