"""Generates the golden fixtures of this folder from the oracle (the CPU
restatement of the reference gridder; the reference itself cannot be built
here).  Small seeded cases, so the fixtures stay a few tens of kB:

  wproject_small.npz    WProject, 36 antennas in a 2 km disk, 60 s at 10 s,
                        2 channels (940-948 MHz), XX; 256^2 at 60"; 9 w-planes,
                        oversample 4.  Per sampled (row, channel): grid cell,
                        oversample offsets, CF index and on-grid status; the
                        CF support and the central taps of three CF planes; the
                        gridded values at the 64 largest cells; the sum of
                        weights; degridded visibilities of a 3-point model.
  awproject_small.npz   AWProject, 2 beams 0.5 deg apart (25 m dishes, 2 m
                        blockage), 2 channels, 5 w-planes, oversample 4, 512^2
                        at 10": the CF support and the central taps of three CF
                        planes, the gridded values at the 64 largest cells, the
                        grid's L2 norm and the sums of weights.
  sphfunc_full_pol.npz  SphFunc, the ImageFFTEquationTest::testFullPol setup:
                        degridded 4-pol visibilities of a centred point
                        (1, 0.01, -0.01, 0.9) at 40 seeded uvw.

Run from the repository root:  python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

ARCSEC = math.pi / (180 * 3600)


def wproject_case():
    from yandasoft_b200 import simulate
    ds = simulate.make_dataset(duration_s=60.0, dt_s=10.0, nchan=2, seed=41, diameter_m=2000.0)
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    params = dict(wmax=wmax, nwplanes=9, oversample=4, maxsupport=256, cutoff=1e-3)
    nx, cell = 256, 60.0 * ARCSEC
    model = np.zeros((nx, nx, 1, 1), dtype=np.float32, order="F")
    for (x, y, f) in ((nx // 2, nx // 2, 1.0), (nx // 2 + 7, nx // 2 - 4, 0.5), (nx // 2 - 11, nx // 2 + 9, 0.25)):
        model[x, y, 0, 0] = f
    return ds, params, nx, cell, model


def make_wproject(path):
    import oracle
    ds, params, nx, cell, model = wproject_case()
    og = oracle.OracleGridder("WProject", **params)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag))
    grid = og.grids[0][:, :, 0, 0]
    iu, iv, fu, fv = oracle.indices(ds.uvw, ds.freq, og.uvcell[0], og.uvcell[1], og.os, nx, nx)
    planes = og.ws.plane_map(ds.uvw, ds.freq)
    s = og.cache.support
    on = (iu - s > 0) & (iv - s > 0) & (iu + s < nx) & (iv + s < nx)
    top = np.argsort(np.abs(grid).ravel(order="F"))[::-1][:64]
    cfs = og.cache.cfs
    pick = [0, len(cfs) // 2, len(cfs) - 1]
    c0 = [cfs[k][s - 2:s + 3, s - 2:s + 3] for k in pick]
    sumw = og.sumw.astype(np.float64).copy()
    og.initialise_degrid(model, cell, cell)
    vis = np.zeros_like(ds.vis)
    og.degrid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=vis, noise=ds.noise, flag=ds.flag))
    np.savez_compressed(path, iu=iu.astype(np.int32), iv=iv.astype(np.int32), fu=fu.astype(np.int32),
                        fv=fv.astype(np.int32), plane=planes.astype(np.int32), on=on, support=np.int32(s),
                        cf_pick=np.array(pick, dtype=np.int32), cf_centre=np.stack(c0).astype(np.complex64),
                        grid_cells=top.astype(np.int64), grid_values=grid.ravel(order="F")[top].astype(np.complex64),
                        grid_l2=np.float64(np.linalg.norm(grid)), sumw=sumw,
                        degrid=vis.astype(np.complex64))


def awproject_case():
    from yandasoft_b200 import simulate
    ds = simulate.make_dataset(duration_s=60.0, dt_s=10.0, nchan=2, seed=43, diameter_m=2000.0)
    feed = (np.arange(ds.nrow) % 2).astype(np.int32)
    pnt = np.zeros((ds.nrow, 2))
    pnt[feed == 1, 0] = 0.5 * math.pi / 180
    wmax = float(np.max(np.abs(ds.uvw[:, 2])) * ds.freq.max() / simulate.C_LIGHT) * 1.05
    params = dict(wmax=wmax, nwplanes=5, oversample=4, maxsupport=256, maxfeeds=2, cutoff=1e-3)
    return ds, feed, pnt, params, 512, 10.0 * ARCSEC


def make_awproject(path):
    import oracle
    ds, feed, pnt, params, nx, cell = awproject_case()
    og = oracle.OracleGridder("AWProject", diameter=25.0, blockage=2.0, **params)
    og.initialise_grid(nx, nx, 1, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis, noise=ds.noise, flag=ds.flag, feed1=feed,
                         pointing=pnt))
    grid = og.grids[0][:, :, 0, 0]
    s = og.cache.support
    top = np.argsort(np.abs(grid).ravel(order="F"))[::-1][:64]
    cfs = og.cache.cfs
    pick = [0, len(cfs) // 2, len(cfs) - 1]
    np.savez_compressed(path, support=np.int32(s), cf_pick=np.array(pick, dtype=np.int32),
                        cf_centre=np.stack([cfs[k][s - 2:s + 3, s - 2:s + 3] for k in pick]).astype(np.complex64),
                        grid_cells=top.astype(np.int64), grid_values=grid.ravel(order="F")[top].astype(np.complex64),
                        grid_l2=np.float64(np.linalg.norm(grid)), sumw=og.sumw.astype(np.float64))


def full_pol_case():
    npix = 512
    img = np.zeros((npix, npix, 4, 1), dtype=np.float32, order="F")
    for p, v in enumerate([1.0, 0.01, -0.01, 0.9]):
        img[npix // 2, npix // 2, p, 0] = v
    rng = np.random.default_rng(3)
    nrow = 40
    uvw = np.zeros((nrow, 3))
    uvw[:, :2] = rng.uniform(-2000, 2000, (nrow, 2))
    uvw[:, 2] = rng.uniform(-500, 500, nrow)
    freq = np.array([1.4e9, 1.41e9])
    return img, uvw, freq, 8.0 * ARCSEC


def make_full_pol(path):
    import oracle
    img, uvw, freq, cell = full_pol_case()
    og = oracle.OracleGridder("SphFunc")
    og.initialise_degrid(img, cell, cell)
    vis = np.zeros((uvw.shape[0], 2, 4), dtype=np.complex64, order="F")
    og.degrid(oracle.Chunk(uvw=uvw, freq=freq, vis=vis))
    np.savez_compressed(path, vis=vis)


if __name__ == "__main__":
    import oracle
    oracle.build()
    make_wproject(os.path.join(HERE, "wproject_small.npz"))
    make_awproject(os.path.join(HERE, "awproject_small.npz"))
    make_full_pol(os.path.join(HERE, "sphfunc_full_pol.npz"))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
