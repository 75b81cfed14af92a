"""Helpers shared by the GPU parity tests: run the oracle and the CUDA gridder
(through the C-ABI) on the same seeded inputs."""
import math

import numpy as np

ARCSEC = math.pi / (180 * 3600)

# parset keys of each gridder that the oracle understands under the same name
_KEYS = ["wmax", "nwplanes", "cutoff", "oversample", "maxsupport", "limitsupport", "alpha", "support",
         "variablesupport", "offsetsupport", "wmaxclip", "maxfeeds", "maxfields", "frequencydependent"]


def make_pair(kind, params, oracle_kw=None, generic=None):
    import oracle
    from yandasoft_b200.gridder import VisGridderFactory
    ps = {"gridder": kind}
    okw = dict(oracle_kw or {})
    for k, v in params.items():
        ps["gridder.%s.%s" % (kind, k)] = v
        if k in _KEYS:
            okw[k] = v
        if k == "cutoff.absolute":
            okw["cutoff_absolute"] = v
        if k == "diameter":
            okw["diameter"] = float(str(v).rstrip("m"))
        if k == "blockage":
            okw["blockage"] = float(str(v).rstrip("m"))
    for k, v in (generic or {}).items():
        ps[k] = v
        if k == "gridder.oversampleweight":
            okw["oversampleweight"] = v
        if k == "gridder.alldatapsf":
            okw["alldatapsf"] = v
    return oracle.OracleGridder(kind, **okw), VisGridderFactory.make(ps)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def snapped_model(ds, nx, cell, npol=1, nchan=1, max_nu=1.0, extra=0, seed=11):
    """Point sources of the simulated sky snapped to pixel centres; returns the
    model image (nx, nx, npol, nchan) and the FP64 DFT components.

    ``max_nu`` keeps sources whose offset from the centre is below that fraction
    of the half-width.  Near the edge the spheroidal correction (1/grdsf) grows
    to hundreds, the grid values grow with it and the degridding sum cancels
    them again, so FP32 results of any two summation orders differ by
    ~eps x correction: see ``degrid_error_bound``.  ``extra`` adds that many
    seeded random point sources (0.1-1 Jy) inside the same region."""
    c = ds.sky.components
    img = np.zeros((nx, nx, npol, nchan), dtype=np.float32, order="F")
    comp = []
    half = nx // 2
    for k in range(len(c)):
        x = int(round(nx // 2 + c[k, 1] / cell))
        y = int(round(nx // 2 + c[k, 2] / cell))
        if abs(x - half) > max_nu * half or abs(y - half) > max_nu * half:
            continue
        if 0 <= x < nx and 0 <= y < nx:
            img[x, y, :, :] += np.float32(c[k, 0])
            comp.append([c[k, 0], (x - nx // 2) * cell, (y - nx // 2) * cell, 0, 0, 0, 0, 1])
    rng = np.random.default_rng(seed)
    lim = int(max_nu * half) - 1
    for _ in range(extra):
        x, y = half + int(rng.integers(-lim, lim + 1)), half + int(rng.integers(-lim, lim + 1))
        f = float(rng.uniform(0.1, 1.0))
        img[x, y, :, :] += np.float32(f)
        comp.append([f, (x - half) * cell, (y - half) * cell, 0, 0, 0, 0, 1])
    return img, np.array(comp)


def degrid_error_bound(og, ds, grids, cell, nx):
    """Per sample and polarisation: sum over taps of |CF| x |grid cell|, the
    quantity that bounds the rounding error of an FP32 tap sum in any order
    (recursive summation: |error| <= (n - 1) u sum |terms|).  Uses the oracle's
    CF cache and index restatement; samples that are not degridded get 0.
    grids: list of (nx, nx, npol, 1) complex64 arrays as the gridder holds them."""
    import oracle
    nrow, nchan = ds.uvw.shape[0], len(ds.freq)
    npol = grids[0].shape[2]
    uvcell = 1.0 / (cell * nx)
    iu, iv, fu, fv = oracle.indices(ds.uvw, ds.freq, uvcell, uvcell, og.os, nx, nx)
    cmap, gmap = og._maps(oracle.Chunk(uvw=ds.uvw, freq=ds.freq, vis=ds.vis))
    plane = np.zeros((nrow, nchan), dtype=np.int64) if cmap is None else cmap.astype(np.int64)
    gind = np.zeros((nrow, nchan), dtype=np.int64) if gmap is None else gmap.astype(np.int64)
    bound = np.zeros((nrow, nchan, npol))
    cfs = og.cache.cfs
    for r in range(nrow):
        for c in range(nchan):
            if plane[r, c] < 0 or gind[r, c] < 0:
                continue
            k = fu[r, c] + og.os * (fv[r, c] + og.os * plane[r, c])
            cf = cfs[k]
            s = (cf.shape[0] - 1) // 2
            x0, y0 = iu[r, c] - s, iv[r, c] - s
            if x0 <= 0 or y0 <= 0 or iu[r, c] + s >= nx or iv[r, c] + s >= nx:
                continue
            g = grids[gind[r, c]][x0:x0 + 2 * s + 1, y0:y0 + 2 * s + 1, :, 0]
            bound[r, c, :] = np.einsum("xy,xyp->p", np.abs(cf), np.abs(g))
    return bound
