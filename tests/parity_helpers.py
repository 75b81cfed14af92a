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


def snapped_model(ds, nx, cell, npol=1, nchan=1):
    """Point sources of the simulated sky snapped to pixel centres; returns the
    model image (nx, nx, npol, nchan) and the FP64 DFT components."""
    c = ds.sky.components
    img = np.zeros((nx, nx, npol, nchan), dtype=np.float32, order="F")
    comp = []
    for k in range(len(c)):
        x = int(round(nx // 2 + c[k, 1] / cell))
        y = int(round(nx // 2 + c[k, 2] / cell))
        if 0 <= x < nx and 0 <= y < nx:
            img[x, y, :, :] += np.float32(c[k, 0])
            comp.append([c[k, 0], (x - nx // 2) * cell, (y - nx // 2) * cell, 0, 0, 0, 0, 1])
    return img, np.array(comp)
