#!/usr/bin/env python
"""Benchmark: grid+degrid visibility throughput on one B200 (Mvis/s).

One step = one degrid pass (model -> visibilities) plus one grid pass
(visibilities -> grid) over every visibility sample of the workload: the
major-cycle shape of ImageFFTEquation::calcImagingEquations.  A visibility
sample is one (row, channel, polarisation).

Workloads (seeded synthetic data with the shapes of the benchmark configs):
  --config 1  W-stacking + W-projection, full-track continuum: 36 antennas in a
              6 km disk, 8 h at 5 s, 96 channels 700-1000 MHz, 4 polarisations
              (348,364,800 rows x channels, 1.39e9 samples, 11 GB), 4096^2 x 4
              grid at 4", 17 w-stacks x 33 w-planes, oversample 8.  Default.
  --config 0  WProject: 36 antennas, 1 h at 10 s, 8 channels 940-948 MHz, XX,
              2048^2 at 8", 65 w-planes, oversample 4.
  --config 2  AWProject, 36 beams: 12 m dishes with 1 m blockage, a 6 x 6 beam
              footprint at 0.9 deg pitch (beams observed in turn, one 5 s
              integration each), 2 h at 5 s (1440 integrations), 48 channels
              700-1000 MHz, 2 polarisations (87,091,200 samples), sources
              attenuated by each beam's power pattern.  One imaging instance
              per beam (rows phased to the beam centre, 2048^2 x 2 grid at 4"),
              33 w-planes, oversample 4, a CF set per channel built on the GPU;
              all beams' degrid -> subtract -> grid in one CUDA graph.

`value` is measured with inputs resident in HBM (plan-based passes on device
buffers); `e2e` goes through the C-ABI IVisGridder calls with pinned host
buffers, copies included.  `--impl reference` times the CPU restatement of the
reference gridder (oracle/, single-threaded gridder per host thread over
channel slices, as the reference runs one gridder per thread or rank).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ARCSEC = math.pi / (180 * 3600)
C_LIGHT = 299792458.0


METRIC = "grid+degrid Mvis/s on 1 B200, plain vs learned-CF at <=1e-3 degrid error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3],
                    help="0, 1: one instance; 2: one instance per beam; 3: 64 uneven instances, major cycles as "
                         "one CUDA graph")
    ap.add_argument("--instances", type=int, default=64, help="config 3: number of imaging instances")
    ap.add_argument("--cycles", type=int, default=5, help="config 3: major cycles timed")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity leg (1% row subset against the oracle)")
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the track (tests only)")
    ap.add_argument("--grid-nx", type=int, default=0,
                    help="grid side override with --cell-arcsec (small profiling cases: 2048 at 8 arcsec keeps "
                         "config 1's field and CF support at a quarter of the grid memory)")
    ap.add_argument("--cell-arcsec", type=float, default=0.0, help="cell override (see --grid-nx)")
    ap.add_argument("--tile", type=int, default=0, help="uv tile side (0 = automatic)")
    ap.add_argument("--variant", type=int, default=0, help="k_grid thread layout variant (0 = automatic)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-CF leg")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner")
    ap.add_argument("--learned-rows", type=float, default=0.01, help="fraction of the track the learned leg times")
    ap.add_argument("--learned-steps", type=int, default=60000, help="Adam steps of the learned CF")
    return ap.parse_args()


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------
def workload(cfg: int, scale: float = 1.0):
    if cfg == 0:
        return dict(name="config0_wproject_2048", gridder="WProject", nant=36, diameter=6000.0, lat=-26.7, dec=-45.0,
                    duration=3600.0 * scale, dt=10.0, f0=940e6, f1=948e6, nchan=8, npol=1, nsrc=20, ngauss=0,
                    field=2.0, sigma=0.01, nx=2048, cell=8.0, nwplanes=65, oversample=4, cutoff=1e-3,
                    maxsupport=1024, seed=0)
    if cfg == 2:
        return dict(name="config2_awproject_36beams_2048x2pol", gridder="AWProject", nant=36, diameter=6000.0,
                    lat=-26.7, dec=-45.0, duration=7200.0 * scale, dt=5.0, f0=700e6, f1=1000e6, nchan=48, npol=2,
                    nsrc=100, ngauss=0, field=2.0, sigma=0.01, nx=2048, cell=4.0, nwplanes=33, oversample=4,
                    cutoff=1e-3, maxsupport=256, seed=2, nbeam=36, pitch=0.9, dish=12.0, blockage=1.0)
    return dict(name="config1_wstack17_wproject33_4096x4pol", gridder="WStackWProject", nant=36, diameter=6000.0,
                lat=-26.7, dec=-45.0, duration=8 * 3600.0 * scale, dt=5.0, f0=700e6, f1=1000e6, nchan=96, npol=4,
                nsrc=200, ngauss=10, field=2.0, sigma=0.01, nx=4096, cell=4.0, nwstacks=17, nwplanes=33, oversample=8,
                cutoff=1e-3, maxsupport=512, seed=1)


def gen_device(w):
    """Synthetic data in HBM (torch).  uvw from the hour-angle rotation, FP64;
    visibilities from the point/Gaussian measurement equation (phase reduced
    in FP64, sin/cos in FP32), noise N(0, sigma)."""
    import torch
    from yandasoft_b200 import simulate
    arr = simulate.random_disk_array(w["nant"], w["diameter"], w["lat"], w["seed"])
    uvw, ntime, nbl = simulate.uvw_track(arr, w["dec"] * simulate.DEG, w["duration"], w["dt"])
    nchan, npol = w["nchan"], w["npol"]
    df = (w["f1"] - w["f0"]) / nchan
    freq = w["f0"] + (np.arange(nchan) + 0.5) * df
    sky = simulate.random_point_sky(w["nsrc"], w["field"], w["seed"] + 1)
    comp = sky.components.copy()
    if w["ngauss"]:
        rng = np.random.default_rng(w["seed"] + 3)
        g = rng.choice(len(comp), w["ngauss"], replace=False)
        comp[g, 3] = rng.uniform(10, 60, len(g)) * ARCSEC   # FWHM major
        comp[g, 4] = comp[g, 3] * rng.uniform(0.3, 1.0, len(g))
        comp[g, 5] = rng.uniform(0, math.pi, len(g))
    dev = torch.device("cuda")
    nrow = uvw.shape[0]
    feed = att = feed_d = foot = None
    if w.get("nbeam"):
        # beams observed in turn, one integration each; each beam's rows are
        # phased to the beam's centre and every source is attenuated by the
        # beam's power pattern
        feed = simulate.multibeam_rows(ntime, nbl, w["nbeam"])
        pw, foot = beam_power(w, comp, freq)
        att = torch.from_numpy(pw).to(dev)
        feed_d = torch.from_numpy(feed).to(dev)
        lb = torch.from_numpy(np.sin(foot[:, 0]) * np.cos(foot[:, 1])).to(dev)
        mb = torch.from_numpy(np.sin(foot[:, 1])).to(dev)
    U = torch.from_numpy(uvw).to(dev)
    F = torch.from_numpy(freq).to(dev)
    l = torch.from_numpy(comp[:, 1]).to(dev)
    m = torch.from_numpy(comp[:, 2]).to(dev)
    flux = torch.from_numpy(comp[:, 0]).to(dev)
    n = torch.sqrt(1 - l * l - m * m)
    gauss = torch.from_numpy((comp[:, 3] > 0) | (comp[:, 4] > 0)).to(dev)
    bmaj = torch.from_numpy(comp[:, 3]).to(dev)
    bmin = torch.from_numpy(comp[:, 4]).to(dev)
    bpa = torch.from_numpy(comp[:, 5]).to(dev)
    scale_g = math.pi ** 2 / (4 * math.log(2.0))
    model = torch.empty((nchan, nrow), dtype=torch.complex64, device=dev)   # transposed for coalescing
    R = 1 << 16
    for r0 in range(0, nrow, R):
        r1 = min(nrow, r0 + R)
        u, v, ww = U[r0:r1, 0:1], U[r0:r1, 1:2], U[r0:r1, 2:3]
        if att is None:
            cyc = (l[None] * u + m[None] * v + (n[None] - 1) * ww) / C_LIGHT       # cycles per Hz (FP64)
        else:
            fr = feed_d[r0:r1].long()
            lr = l[None] - lb[fr][:, None]
            mr = m[None] - mb[fr][:, None]
            nr = torch.sqrt(1 - lr * lr - mr * mr)
            cyc = (lr * u + mr * v + (nr - 1) * ww) / C_LIGHT
        r = None
        if bool(gauss.any()):
            up = (torch.cos(bpa)[None] * u + torch.sin(bpa)[None] * v) / C_LIGHT
            vp = (-torch.sin(bpa)[None] * u + torch.cos(bpa)[None] * v) / C_LIGHT
            r = (bmaj[None] ** 2 * up * up + bmin[None] ** 2 * vp * vp) * scale_g
        for c in range(nchan):
            f = float(freq[c])
            ph = cyc * f
            ph = (ph - torch.floor(ph)).float() * (2 * math.pi)
            amp = flux[None].expand_as(ph)
            if att is not None:
                amp = amp * att[fr, :, c]
            if r is not None:
                amp = amp * torch.exp(-r * f * f)
            amp = amp.float()
            re = (amp * torch.cos(ph)).sum(1)
            im = (amp * torch.sin(ph)).sum(1)
            model[c, r0:r1] = torch.complex(re, im)
    gen = torch.Generator(device=dev)
    gen.manual_seed(w["seed"] + 2)
    # cube (nrow, nchan, npol) column-major == memory [pol][chan][row]
    vis = torch.empty((npol, nchan, nrow), dtype=torch.complex64, device=dev)
    for p in range(npol):
        sig = model if (npol == 1 or p in (0, npol - 1)) else 0
        nz = torch.complex(torch.randn((nchan, nrow), generator=gen, device=dev),
                           torch.randn((nchan, nrow), generator=gen, device=dev)) * w["sigma"]
        vis[p] = sig + nz
    del model
    wmax_data = float(torch.max(torch.abs(U[:, 2]))) * float(freq.max()) / C_LIGHT
    return dict(uvw=U, freq=F, vis=vis, nrow=nrow, nchan=nchan, npol=npol, freq_np=freq, uvw_np=uvw, sky=comp,
                wmax=math.ceil(wmax_data * 1.02 / 100.0) * 100.0, feed_np=feed, foot=foot)


def parset_for(w, wmax):
    g = w["gridder"]
    p = {"gridder": g, "gridder.%s.wmax" % g: wmax, "gridder.%s.nwplanes" % g: w["nwplanes"],
         "gridder.%s.oversample" % g: w["oversample"], "gridder.%s.cutoff" % g: w["cutoff"],
         "gridder.%s.maxsupport" % g: w["maxsupport"]}
    if g == "WStackWProject":
        p["gridder.%s.nwstacks" % g] = w["nwstacks"]
    if g == "AWProject":
        p["gridder.%s.maxfeeds" % g] = 1          # one beam per imaging instance
        p["gridder.%s.diameter" % g] = "%gm" % w["dish"]
        p["gridder.%s.blockage" % g] = "%gm" % w["blockage"]
    return p


def beam_power(w, comp, freq):
    """Power pattern of each beam at each source, (nbeam, nsrc, nchan): the
    far field of a uniformly illuminated annular aperture (dish diameter D,
    central blockage d) at the source's distance from the beam centre,
    V = (D^2 jinc(pi D theta / lambda) - d^2 jinc(pi d theta / lambda)) / (D^2 - d^2)
    with jinc(x) = 2 J1(x) / x, and P = V^2."""
    from scipy.special import j1
    from yandasoft_b200 import simulate
    foot = simulate.beam_footprint(int(round(math.sqrt(w["nbeam"]))), w["pitch"])
    lb = np.sin(foot[:, 0]) * np.cos(foot[:, 1])
    mb = np.sin(foot[:, 1])
    theta = np.hypot(comp[None, :, 1] - lb[:, None], comp[None, :, 2] - mb[:, None])     # (nbeam, nsrc)
    lam = C_LIGHT / np.asarray(freq)

    def jinc(x):
        x = np.where(x == 0, 1e-30, x)
        return 2.0 * j1(x) / x

    D, b = w["dish"], w["blockage"]
    x = math.pi * theta[:, :, None] / lam[None, None, :]
    v = (D * D * jinc(D * x) - b * b * jinc(b * x)) / (D * D - b * b)
    return (v * v).astype(np.float64), foot


def model_image(w, sky, npol):
    nx = w["nx"]
    cell = w["cell"] * ARCSEC
    img = np.zeros((nx, nx, npol, 1), dtype=np.float32, order="F")
    for k in range(len(sky)):
        x = int(round(nx // 2 + sky[k, 1] / cell))
        y = int(round(nx // 2 + sky[k, 2] / cell))
        if 0 <= x < nx and 0 <= y < nx:
            img[x, y, 0, 0] += sky[k, 0]
            if npol > 1:
                img[x, y, npol - 1, 0] += sky[k, 0]
    return img


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0:
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, nm in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def max_over_ranks(ms, dist=None, device="cuda"):
    """The job's time for the timed steps: the slowest rank's (every rank
    takes part in the reduction)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, nvis_per_rank, ms_step):
    """Whole-job throughput (Mvis/s): every replica processes its own copy of
    the workload (weak scaling), the job takes the slowest rank's time."""
    return world * nvis_per_rank / (ms_step / 1e3) / 1e6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
# CPU baseline (oracle restatement), bounded sample
# --------------------------------------------------------------------------
class CpuBaseline:
    """The oracle's C restatement of TableVisGridder::generic timed on a row
    subset of the same workload: one degrid + one grid pass per run.  Threads
    run independent gridders over channel slices, as the reference
    parallelises (one gridder clone per thread); each holds its own grids, so
    the thread count is capped by host memory.  Every gridder, its grids
    (zeroed and touched) and its chunk are made before the timed region; a
    run times only the two passes.  The degridding grids are shared and left
    zero: the tap loop does the same work whatever the cell values."""

    def __init__(self, w, d, target_s=15.0, threads=None):
        import oracle
        import psutil
        threads = threads or (os.cpu_count() or 1)
        self.w, self.d = w, d
        nx = w["nx"]
        cell = w["cell"] * ARCSEC
        kind = w["gridder"]
        kw = dict(nwplanes=w["nwplanes"], wmax=d["wmax"], oversample=w["oversample"], cutoff=w["cutoff"],
                  maxsupport=w["maxsupport"])
        if kind == "WStackWProject":
            kw["nwstacks"] = w["nwstacks"]
        g0 = oracle.OracleGridder(kind, **kw)
        g0.initialise_grid(nx, nx, d["npol"], 1, cell, cell)
        g0.init_cf()
        self.grid_bytes = sum(g.nbytes for g in g0.grids)
        self.support = int(g0.cache.support)
        avail = psutil.virtual_memory().available
        mem_threads = int((0.6 * avail - self.grid_bytes) // max(1, self.grid_bytes))
        self.threads = threads = max(1, min(threads, mem_threads))
        nrow_all = d["nrow"]
        freq = d["freq_np"]
        # calibrate a row count: ~1.2 ns per tap per polarisation per pass, two passes
        taps = (2 * g0.cache.support + 1) ** 2
        per_sample = 2 * taps * d["npol"] * 1.2e-9 / threads
        nrows = int(min(nrow_all, max(1000, target_s / (per_sample * len(freq)))))
        step = max(1, nrow_all // nrows)
        rows = np.arange(0, nrow_all, step)[:nrows]
        uvw = np.ascontiguousarray(d["uvw_np"][rows])
        vis = d["vis"][:, :, torch_index(rows)].cpu().numpy()          # [pol][chan][row]
        cube = np.asfortranarray(np.transpose(vis, (2, 1, 0)))
        self.jobs = []
        for ch in np.array_split(np.arange(len(freq)), threads):
            if len(ch) == 0:
                continue
            gd = oracle.OracleGridder(kind, **kw)
            gd._init_axes(nx, nx, d["npol"], 1, cell, cell, None)   # initialise_degrid without the FFTs
            gd.psf = False
            gd.model_empty = False
            gd.sumw = None
            gd._init_sumw()
            gd.grids = g0.grids
            gd.cache, gd._flat = g0.cache, g0._flat
            gg = oracle.OracleGridder(kind, **kw)
            gg.initialise_grid(nx, nx, d["npol"], 1, cell, cell)
            gg._grid_buffer()[:] = 0                                # touch every page now
            gg.cache, gg._flat = g0.cache, g0._flat
            sub = np.asfortranarray(cube[:, ch, :])
            fch = np.ascontiguousarray(freq[ch])
            self.jobs.append((gd, gg, oracle.Chunk(uvw=uvw, freq=fch, vis=np.zeros_like(sub)),
                              oracle.Chunk(uvw=uvw, freq=fch, vis=sub)))
        self.sample = ("%d of %d rows (every %d-th), all %d channels x %d pols; one degrid + one grid pass; %d "
                       "threads over channel slices, each with its own %.1f GB of grids (made before timing)"
                       % (len(rows), nrow_all, step, len(freq), d["npol"], threads, self.grid_bytes / 1e9))

    def run(self):
        """One degrid + grid pass of every thread's gridders; (Mvis/s, seconds)."""
        import concurrent.futures as cf

        def work(job):
            gd, gg, cd, cg = job
            gd.degrid(cd)
            gg.grid(cg)
            return cg.vis.size

        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=len(self.jobs)) as ex:
            n = sum(ex.map(work, self.jobs))
        t = time.perf_counter() - t0
        return n / t / 1e6, t


def cpu_baseline(w, d, target_s=15.0, threads=None):
    """All host threads (one gridder per channel slice), then one thread on a
    smaller subset.  Returns (Mvis/s, info)."""
    cb = CpuBaseline(w, d, target_s=target_s, threads=threads)
    cb.run()                      # warm (first touch of the CF cache and the data)
    v, t = cb.run()
    info = dict(cores=cb.threads, seconds=t, sample=cb.sample)
    del cb
    one = CpuBaseline(w, d, target_s=target_s / 3.0, threads=1)
    v1, t1 = one.run()
    info["single_core"] = {"value": round(v1, 4), "unit": "Mvis/s", "cores": 1, "seconds": round(t1, 2),
                           "sample": one.sample}
    return v, info


def cpu_baseline_aw(w, d, ps=None, target_s=15.0, threads=None):
    """AWProject, one beam's imaging instance (the footprint's corner beam,
    its rows phased to its own centre): the oracle's CF generation (the numpy
    restatement of AWProjectVisGridder::initConvolutionFunction) timed per
    (beam, channel) set of w-planes, and one degrid + one grid pass of its C
    gridder on that beam's rows and channels (its whole chunk), threads over
    row slices (one gridder each, sharing the CF cache), repeated until about
    target_s seconds have passed.  With a
    parset `ps`, the GPU gridder grids the same sample with it and its CF
    matrices and grid are compared with the oracle's.
    Returns (Mvis/s, info)."""
    import concurrent.futures as cf
    import oracle
    threads = threads or (os.cpu_count() or 1)
    nx = w["nx"]
    cell = w["cell"] * ARCSEC
    chans = np.arange(d["nchan"])
    rows_all = np.nonzero(d["feed_np"] == 0)[0]
    freq = np.ascontiguousarray(d["freq_np"][chans])
    kw = dict(nwplanes=w["nwplanes"], wmax=d["wmax"], oversample=w["oversample"], cutoff=w["cutoff"],
              maxsupport=w["maxsupport"], maxfeeds=1, diameter=w["dish"], blockage=w["blockage"])
    g0 = oracle.OracleGridder("AWProject", **kw)
    g0.initialise_grid(nx, nx, d["npol"], 1, cell, cell)
    t0 = time.perf_counter()
    # the CF cache depends on the beam, its pointing and the chunk's frequencies
    g0.init_cf(oracle.Chunk(uvw=np.zeros((1, 3)), freq=freq, vis=None))
    t_cf = time.perf_counter() - t0
    njobs = len(chans)
    support = g0.cache.support
    taps = (2 * support + 1) ** 2
    per_sample = 2 * taps * d["npol"] * 1.5e-9 / max(1, threads)
    nrows = int(min(len(rows_all), max(2000, target_s / (per_sample * len(chans)))))
    rows = rows_all[np.linspace(0, len(rows_all) - 1, nrows).astype(np.int64)]
    uvw = np.ascontiguousarray(d["uvw_np"][rows])
    vis = d["vis"][:, :, torch_index(rows)][:, torch_index(chans), :].cpu().numpy()      # [pol][chan][row]
    cube = np.asfortranarray(np.transpose(vis, (2, 1, 0)))
    chunk = oracle.Chunk(uvw=uvw, freq=freq, vis=cube)
    check = {}
    if ps is not None:
        # the GPU gridder on the same sample: CF matrices and grid against the oracle
        from yandasoft_b200 import gridder as G
        gs = G.VisGridderFactory.make(ps)
        gs.initialiseGrid(G.Axes(cell, cell), (nx, nx, d["npol"], 1))
        gs.grid(G.Accessor(uvw, freq, cube))
        cf_err = 0.0
        ncmp = 0
        for a, b in zip(g0.cache.cfs, gs.convolution_functions()):
            if a is None:
                continue
            cf_err = max(cf_err, float(np.max(np.abs(a - b)) / np.max(np.abs(a))))
            ncmp += 1
        og = oracle.OracleGridder("AWProject", **kw)
        og.initialise_grid(nx, nx, d["npol"], 1, cell, cell)
        og.grid(chunk)
        grid_err = float(np.linalg.norm(gs.grids()[0] - og.grids[0]) / np.linalg.norm(og.grids[0]))
        check = {"sample_cf_matrices_compared": ncmp, "sample_cf_max_rel_err_vs_oracle": cf_err,
                 "sample_grid_rel_err_vs_oracle": grid_err, "sample_support_gpu": int(gs.support()[0]),
                 "sample_support_oracle": int(support)}
        del gs, og
    slices = np.array_split(np.arange(len(rows)), threads)

    def work(sl):
        if len(sl) == 0:
            return 0
        sub = oracle.Chunk(uvw=np.ascontiguousarray(uvw[sl]), freq=freq, vis=np.asfortranarray(cube[sl]))
        out = np.zeros_like(sub.vis)
        gd = oracle.OracleGridder("AWProject", **kw)
        gd._init_axes(nx, nx, d["npol"], 1, cell, cell, None)
        gd.psf = False
        gd.grids = g0.grids
        gd.cache, gd._flat, gd.aw_params, gd.aw_nchan = g0.cache, g0._flat, g0.aw_params, g0.aw_nchan
        gd.sumw = np.zeros((1, d["npol"], 1), order="F")
        gd._run(oracle.Chunk(uvw=sub.uvw, freq=freq, vis=out), forward=True)
        gg = oracle.OracleGridder("AWProject", **kw)
        gg.initialise_grid(nx, nx, d["npol"], 1, cell, cell)
        gg.cache, gg._flat, gg.aw_params, gg.aw_nchan = g0.cache, g0._flat, g0.aw_params, g0.aw_nchan
        gg.sumw = np.zeros_like(g0.sumw)
        gg._run(sub, forward=False)
        return sub.vis.size

    t0 = time.perf_counter()
    n = reps = 0
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        while True:
            n += sum(ex.map(work, slices))
            reps += 1
            t = time.perf_counter() - t0
            if t >= target_s or reps >= 50:
                break
    info = dict(cores=threads, seconds=t,
                sample="%d of %d rows (beam 0's instance), all %d channels, %d pols; one degrid + one grid pass, "
                       "repeated %d times; %d threads over row slices sharing the oracle's CF cache"
                % (len(rows), d["nrow"], d["nchan"], d["npol"], reps, threads),
                cf={"cpu_port_s_per_beam_channel": round(t_cf / njobs, 3),
                    "cpu_port_s_all_%d_beams_x_%d_channels" % (w["nbeam"], d["nchan"]):
                        round(t_cf / njobs * w["nbeam"] * d["nchan"], 1), **check})
    return n / t / 1e6, info


def torch_index(a):
    import torch
    return torch.from_numpy(np.asarray(a, dtype=np.int64)).to("cuda")


# --------------------------------------------------------------------------
# arms
# --------------------------------------------------------------------------
def kernel_names(variant, support):
    """The grid and degrid kernels a pass runs for a k_grid variant: the
    plane-major k_grid_pl with variant bit 64, else k_grid; k_degrid_r for
    16-wide CFs unless variant bit 256 asks for k_degrid_t."""
    v = variant or 1
    grid = "k_grid_pl" if v & 64 else "k_grid"
    degrid = "k_degrid_r" if (2 * support + 1 <= 16 and not v & 256) else "k_degrid_t"
    return grid, degrid


def roofline(w, d, info, support, npol, nvalid_vis, kgrid_ms, kdeg_ms, hbm_peak, peak_kind, sm_hz, cf_bytes,
             names=("k_grid", "k_degrid_t")):
    """Roofline of the dominant kernel (the grid pass's) and of the degrid kernel, per launch
    (one grid or degrid pass over the workload).  The binding roofline time is
    t_roof = max(algorithmic HBM bytes / measured HBM bandwidth,
    8 flops per tap x taps / FP32 peak at the sampled SM clock); frac =
    t_roof / kernel time.  Algorithmic HBM bytes of a grid pass: every on-grid
    sample's visibility (8 B) and weight (4 B), uvw (24 B per row), flags
    (1 B per row and channel), one write of every grid plane (8 B per cell)
    and one read of the CF cache; of a degrid pass: one read of every grid
    plane, every sample's visibility written (8 B), uvw and the CF cache."""
    taps = (2 * support + 1) ** 2
    nrowchan = d["nrow"] * d["nchan"]
    planes = w.get("nwstacks", 1) if w["gridder"] in ("WStack", "WStackWProject") else 1
    grid_bytes = planes * w["nx"] * w["nx"] * npol * 8.0
    hbm_grid = nvalid_vis * 12.0 + d["nrow"] * 24.0 + nrowchan * 1.0 + grid_bytes + cf_bytes
    hbm_degrid = grid_bytes + nvalid_vis * 8.0 + d["nrow"] * 24.0 + cf_bytes
    flops = 8.0 * taps * nvalid_vis
    fp32_peak = 148 * 128 * 2 * sm_hz                      # FMA lanes x 2 flops at the sampled clock
    smem_peak = 148 * 128 * sm_hz                          # bytes per second, 128 B per clock per SM

    def one(ms, hbm_bytes, smem_per_tap):
        t = ms / 1e3
        t_hbm = hbm_bytes / (hbm_peak * 1e9)
        t_fp = flops / fp32_peak
        out = {"ms": round(ms, 4), "t_roof_ms": round(1e3 * max(t_hbm, t_fp), 4),
               "bound": "fp32" if t_fp >= t_hbm else "hbm",
               "frac": round(max(t_hbm, t_fp) / t, 4) if t > 0 else 0.0,
               "fp32": {"achieved_tflops": round(flops / t / 1e12, 3) if t > 0 else 0.0,
                        "peak_tflops": round(fp32_peak / 1e12, 2), "frac": round(t_fp / t, 4) if t > 0 else 0.0},
               "hbm": {"bytes": int(hbm_bytes), "achieved_gbs": round(hbm_bytes / t / 1e9, 2) if t > 0 else 0.0,
                       "peak_gbs": hbm_peak, "peak_kind": peak_kind, "frac": round(t_hbm / t, 4) if t > 0 else 0.0},
               "smem": {"bytes_per_tap": smem_per_tap,
                        "frac": round(nvalid_vis / npol * taps * smem_per_tap / smem_peak / t, 4) if t > 0 else 0.0}}
        return out

    g = one(kgrid_ms, hbm_grid, 16.0 * npol + 8.0)
    dg = one(kdeg_ms, hbm_degrid, 8.0 * npol + 8.0)
    traffic = kgrid_traffic(info, support, npol, names[0])
    return {"bound": g["bound"], "kernel": names[0], "achieved": g["fp32"]["achieved_tflops"],
            "peak": g["fp32"]["peak_tflops"], "peak_kind": "nominal FP32 (148 SMs x 128 lanes x 2 flops) at the "
                                                           "sampled SM clock",
            "unit": "TFLOP/s", "frac": g["frac"], "traffic": traffic,
            "traffic_note": "DRAM bytes per %s launch, scaled from a single-kernel ncu capture of a small case "
                            "of this workload by samples and work items" % names[0],
            "t_roof_ms": g["t_roof_ms"], "kgrid_ms": round(kgrid_ms, 4), "kdegrid_ms": round(kdeg_ms, 4),
            names[0]: g, names[1]: dg, "taps_per_s": round(taps * nvalid_vis / (kgrid_ms / 1e3), 1)
            if kgrid_ms > 0 else 0,
            "note": "t_roof = max(algorithmic HBM bytes / measured HBM bandwidth, 8 flops x taps / FP32 peak); "
                    "frac = t_roof / kernel time; smem frac: the named shared-memory bytes per tap and sample "
                    "over 128 B per clock per SM"}


# DRAM bytes of one grid launch per on-grid sample and per work item x
# polarisation x padded-tile cell, from single-kernel ncu captures of a small
# case of config 1 (k_grid: the sorted records and visibilities read per
# sample, the padded tiles written per item)
# (k_grid_pl: records and the cube's visibility sectors read per sample, the
# item's global tile reduced and read back per cell)
TRAFFIC_RATES = {"k_grid": (48.9, 0.84 * 8), "k_grid_pl": (303.0, 26.6)}


def kgrid_traffic(info, support, npol, name="k_grid"):
    """DRAM bytes of one grid launch from the kernel's captured rates (None
    when no capture of the kernel gives them)."""
    if name not in TRAFFIC_RATES:
        return None
    per_sample, per_cell = TRAFFIC_RATES[name]
    pad = info["tile"] + 2 * support
    return int(per_sample * info["nvalid"] + per_cell * info["nitems"] * npol * pad * pad)


def run_b200(args, w):
    import torch
    from yandasoft_b200 import build
    from yandasoft_b200 import gridder as G
    build.build()
    G.load()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    d = gen_device(w)
    nx = w["nx"]
    cell = w["cell"] * ARCSEC
    axes = G.Axes(cell, cell)
    ps = parset_for(w, d["wmax"])
    npol = d["npol"]
    nvis = d["nrow"] * d["nchan"] * npol
    acc = G.Accessor(d["uvw"], d["freq"], d["vis"], shape=(d["nrow"], d["nchan"], npol))
    model_buf = torch.zeros_like(d["vis"])
    acc_model = G.Accessor(d["uvw"], d["freq"], model_buf, shape=(d["nrow"], d["nchan"], npol))
    tune = None
    if not args.no_tune and not args.tile and not args.variant:
        # the autotuner on the workload itself (sample density per tile sets the
        # optimum); its choice serves every gridder of this CF width
        tuner = G.VisGridderFactory.make(ps)
        tuner.initialiseGrid(axes, (nx, nx, npol, 1))
        t0 = time.perf_counter()
        tune = tuner.autotune(acc, max_trials=10)
        tune["seconds"] = round(time.perf_counter() - t0, 2)
        del tuner
        torch.cuda.empty_cache()
    gg = G.VisGridderFactory.make(ps)
    if args.tile:
        gg.set_tile(args.tile)
    if args.variant:
        gg.set_grid_variant(args.variant)
    gg.initialiseGrid(axes, (nx, nx, npol, 1))
    gd = gg.clone()
    img = model_image(w, d["sky"], npol)
    gd.initialiseDegrid(axes, img)
    t0 = time.perf_counter()
    plan = gg.plan(acc)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t0
    info = plan.info()
    support = gg.support()[0]
    stream = torch.cuda.ExternalStream(gg.stream_handle())

    def step():
        gd.degrid_plan(plan, acc_model)
        gg.grid_plan(plan, acc)

    for _ in range(args.warmup):
        step()
    gg.synchronize()
    gd.synchronize()
    k0 = gg.kernel_times()
    k0d = gd.kernel_times()
    launches0 = G.kernel_launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = G.kernel_launch_count() - launches0
    ms = max_over_ranks(ms, dist)
    if dist:
        dist.barrier()
    k1 = gg.kernel_times()
    k1d = gd.kernel_times()
    ms_step = ms / args.steps
    value = job_value(world, nvis, ms_step)
    kgrid_ms = (k1["kgrid_ms"] - k0["kgrid_ms"]) / max(1.0, k1["kgrid_calls"] - k0["kgrid_calls"])
    kdeg_ms = (k1d["kdegrid_ms"] - k0d["kdegrid_ms"]) / max(1.0, k1d["kdegrid_calls"] - k0d["kdegrid_calls"])
    nvalid_vis = info["nvalid"] * npol
    taps = (2 * support + 1) ** 2
    hbm_peak, peak_kind = peaks()
    sm_hz = (clk.summary().get("sm_mhz") or 1965.0) * 1e6
    variant = args.variant or ((tune or {}).get("variant") or 0)
    roof = roofline(w, d, info, support, npol, nvalid_vis, kgrid_ms, kdeg_ms, hbm_peak, peak_kind, sm_hz,
                    gg.cf_bytes(), kernel_names(variant, support))
    line = {
        "metric": METRIC,
        "cf_form": "plain (tabulated CF)",
        "value": round(value, 3), "unit": "Mvis/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded; see bench.py workload())",
        "config": {"workload": w["name"], "gridder": w["gridder"], "vis_samples": int(nvis),
                   "rows": int(d["nrow"]), "channels": d["nchan"], "pols": npol, "grid": [nx, nx, npol, 1],
                   "support": support, "taps_per_sample": taps, "oversample": w["oversample"],
                   "tile": info["tile"], "work_items": info["nitems"], "on_grid_samples": int(info["nvalid"]),
                   "l2": "inputs (%.1f GB of visibilities) larger than L2" % (nvis * 8 / 1e9),
                   "step": "one degrid pass + one grid pass over all samples, inputs resident in HBM",
                   "plan_build_s": round(t_plan, 3), "autotune": tune},
        "roofline": roof,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    del plan, gg, gd, acc, acc_model, model_buf
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if not args.no_learned and w["gridder"] in ("WProject", "WStackWProject"):
        try:
            line["learned"] = learned_leg(args, w, d, ps, axes, img)
        except Exception as e:  # the learned leg must not hide the plain result
            line["learned"] = {"error": repr(e)}
    if not args.no_e2e:
        line["e2e"] = e2e_b200(args, w, d, ps, axes, img)
    if rank == 0 and not args.no_parity and w["gridder"] in ("WProject", "WStackWProject"):
        try:
            line["parity"] = parity_subset(w, d, ps, axes, img)
        except Exception as e:  # the parity leg must not hide the GPU result
            line["parity"] = {"error": repr(e)}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, inf = cpu_baseline(w, d)
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mvis/s", "cores": inf["cores"], "kind": "port",
                                    "sample": inf["sample"], "seconds": round(inf["seconds"], 2),
                                    "single_core": inf.get("single_core")}
        except Exception as e:  # the baseline must not hide the GPU result
            line["cpu_baseline"] = {"value": None, "error": repr(e)}
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def dft_model(img, cell, uvw, freq, rows, chans):
    """FP64 direct DFT of the model image's pixels (polarisation 0) at the
    given (row, channel) samples: V = sum_k S_k exp(+2 pi i f/c (u l + v m +
    w (n - 1))) with l, m the pixel offsets from the image centre (the
    measurement equation of UnpolarizedPointSource::calcPoint)."""
    import torch
    nx = img.shape[0]
    xs, ys = np.nonzero(img[:, :, 0, 0])
    flux = torch.tensor(img[xs, ys, 0, 0].astype(np.float64), device="cuda")
    lm = torch.tensor(np.stack([(xs - nx // 2) * cell, (ys - nx // 2) * cell], 1), device="cuda")
    nn = torch.sqrt(1 - lm[:, 0] ** 2 - lm[:, 1] ** 2) - 1
    U = torch.as_tensor(np.asarray(uvw)[rows], device="cuda")
    f = torch.tensor(np.asarray(freq)[chans], device="cuda")
    ph = 2 * math.pi * (f / C_LIGHT)[:, None] * (U[:, 0:1] * lm[None, :, 0] + U[:, 1:2] * lm[None, :, 1]
                                                 + U[:, 2:3] * nn[None, :])
    return (flux[None] * torch.exp(1j * ph)).sum(1).cpu().numpy()


def parity_subset(w, d, ps, axes, img, frac=0.01, seed=20240):
    """The timed workload's parity on a seeded row subset (1% of the rows,
    every channel and polarisation): the GPU gridder, with the tile and
    kernel choice of the timed run, against the oracle's restatement of the
    reference gridder on the same samples.  Grid: relative L2 error over every
    w-stack, sums of weights compared exactly, index mismatches (cell, CF
    index and status of every sample).  Degrid of the model image: the oracle
    degrids the GPU's own transformed grids (the tap path), relative L2 error
    of the visibilities; each degrid result's error against the FP64 DFT of
    the model on a sample of 4096 gridded points (polarisation 0) is stated."""
    import torch
    import oracle
    from yandasoft_b200 import gridder as G
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    nrow_all, nchan, npol = d["nrow"], d["nchan"], d["npol"]
    rows = np.sort(rng.choice(nrow_all, max(1, int(nrow_all * frac)), replace=False))
    nr = len(rows)
    uvw = np.ascontiguousarray(d["uvw_np"][rows])
    freq = d["freq_np"]
    vis_dev = d["vis"][:, :, torch_index(rows)].contiguous()          # [pol][chan][row]
    cube = np.asfortranarray(np.transpose(vis_dev.cpu().numpy(), (2, 1, 0)))
    nx = w["nx"]
    cell = w["cell"] * ARCSEC
    acc = G.Accessor(torch.from_numpy(uvw).cuda(), d["freq"], vis_dev, shape=(nr, nchan, npol))
    gg = G.VisGridderFactory.make(ps)
    gg.initialiseGrid(axes, (nx, nx, npol, 1))
    plan = gg.plan(acc)
    gg.grid_plan(plan, acc)
    iu, iv, cfi, st = plan.samples(gg, acc)
    kw = dict(nwplanes=w["nwplanes"], wmax=d["wmax"], oversample=w["oversample"], cutoff=w["cutoff"],
              maxsupport=w["maxsupport"])
    if w["gridder"] == "WStackWProject":
        kw["nwstacks"] = w["nwstacks"]
    og = oracle.OracleGridder(w["gridder"], **kw)
    og.initialise_grid(nx, nx, npol, 1, cell, cell)
    og.grid(oracle.Chunk(uvw=uvw, freq=freq, vis=cube))
    S = og.cache.support
    oiu, oiv, ofu, ofv = oracle.indices(uvw, freq, og.uvcell[0], og.uvcell[1], og.os, nx, nx)
    cmap, gmap = og._maps(oracle.Chunk(uvw=uvw, freq=freq, vis=cube))
    gmap = np.zeros_like(cmap) if gmap is None else gmap
    okp = (cmap >= 0) & (gmap >= 0)
    on = okp & (oiu - S > 0) & (oiv - S > 0) & (oiu + S < nx) & (oiv + S < nx)
    ocfi = ofu + og.os * (ofv + og.os * cmap.astype(np.int64))
    mism = int((st != np.where(~okp, 1, np.where(on, 3, 2))).sum() + (iu[on] != oiu[on]).sum()
               + (iv[on] != oiv[on]).sum() + (cfi[on] != ocfi[on]).sum())
    num = den = 0.0
    for a, b in zip(gg.grids(), og.grids):
        num += float(np.linalg.norm((a - b).ravel()) ** 2)
        den += float(np.linalg.norm(b.ravel()) ** 2)
    sumw_equal = bool(np.array_equal(gg.sum_weights(), og.sumw))
    tile = plan.info()["tile"]
    gd = gg.clone()
    del gg
    gd.initialiseDegrid(axes, img)
    out = torch.zeros_like(vis_dev)
    accm = G.Accessor(acc.uvw, acc.freq, out, shape=(nr, nchan, npol))
    gd.degrid_plan(plan, accm)
    vg = accm.vis_numpy()
    og.grids = [np.asfortranarray(g) for g in gd.grids()]
    del gd, plan
    og.model_empty = False
    og.carry = None
    vc = np.zeros_like(cube)
    og.degrid(oracle.Chunk(uvw=uvw, freq=freq, vis=vc))
    og.grids = None
    vis_rel = float(np.linalg.norm((vg - vc).ravel()) / np.linalg.norm(vc.ravel()))
    r, c = np.nonzero(on)
    k = rng.choice(len(r), min(4096, len(r)), replace=False)
    dft = dft_model(img, cell, uvw, freq, r[k], c[k])
    e_dft = lambda v: float(np.linalg.norm(v[r[k], c[k], 0] - dft) / np.linalg.norm(dft))
    torch.cuda.empty_cache()
    return {"subset": "%d of %d rows (seeded %.0f%%), all %d channels x %d pols; tile %d as timed"
                      % (nr, nrow_all, 100 * frac, nchan, npol, tile),
            "grid_rel": math.sqrt(num / den) if den > 0 else None, "vis_rel": vis_rel, "index_mismatch": mism,
            "sumw_equal": sumw_equal, "tolerance": 1e-5,
            "degrid_rel_err_vs_dft": {"gpu": e_dft(vg), "oracle": e_dft(vc), "samples": int(len(k))},
            "seconds": round(time.perf_counter() - t0, 1)}


def learned_leg(args, w, d, ps, axes, img):
    """The learned CF beside the tabulated one on the same data: the network is
    trained on the GPU on a table of 257 w-planes (oversampling as configured),
    then a degrid + grid step runs with the network evaluated inside the
    kernels, on a contiguous slice of the track (the in-kernel network costs
    far more per tap than a table lookup), in two forms: at the tabulated
    offsets and planes (form 1) and at every sample's own offsets and w
    (form 2, continuous).  Reports Mvis/s of the three forms on that slice,
    CF memory, the degridded-visibility error of each learned form against
    the tabulated one and of all three against the FP64 DFT of the model on a
    sample of gridded visibilities, and the form kept: a learned form only
    where its error against the tabulated path is at most 1e-3."""
    import torch
    from yandasoft_b200 import gridder as G
    npol, nchan, nrow = d["npol"], d["nchan"], d["nrow"]
    nr = max(1, int(nrow * args.learned_rows))
    uvw = d["uvw"][:nr].contiguous()
    vis = d["vis"][:, :, :nr].contiguous()
    nvis = nr * nchan * npol
    acc = G.Accessor(uvw, d["freq"], vis, shape=(nr, nchan, npol))
    nx = w["nx"]
    gl = G.VisGridderFactory.make(ps)
    gl.initialiseGrid(axes, (nx, nx, npol, 1))
    gl.build_cf()
    support = gl.support()[0]
    rep = gl.learned_train(steps=args.learned_steps, nwplanes_train=257, seed=w["seed"] + 11)
    dense_bytes = 257 * w["oversample"] ** 2 * (2 * support + 1) ** 2 * 8
    out = {"cf_form_kept": None, "trained_on": "257 w-planes x oversample %d (dense table built on the GPU)"
                                                 % w["oversample"],
           "train_steps": rep["steps"], "train_ms": round(rep["train_ms"], 1),
           "final_loss": rep["final_loss"], "network_bytes": int(rep["network_bytes"]),
           "cf_table_bytes": int(rep["cf_table_bytes"]), "cf_table_257_planes_bytes": int(dense_bytes),
           "slice": "first %d of %d rows (%.2f%% of the track), all %d channels x %d pols"
                    % (nr, nrow, 100.0 * nr / nrow, nchan, npol)}
    results = {}
    stream = None
    for form in (0, 1, 2):
        gg = gl.clone()
        gg.set_cf_form(form)
        gg.initialiseGrid(axes, (nx, nx, npol, 1))
        gd = gl.clone()
        gd.set_cf_form(form)
        gd.initialiseDegrid(axes, img)
        model_buf = torch.zeros_like(vis)
        accm = G.Accessor(uvw, d["freq"], model_buf, shape=(nr, nchan, npol))
        plan = gg.plan(acc)
        stream = torch.cuda.ExternalStream(gg.stream_handle())
        gd.degrid_plan(plan, accm)         # warm-up (and the model visibilities of this form)
        gg.grid_plan(plan, acc)
        gg.synchronize()
        gd.synchronize()
        vis_model = model_buf.clone()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gd.degrid_plan(plan, accm)
        gg.grid_plan(plan, acc)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        iu, iv, cfi, st = plan.samples(gg, acc)
        results[form] = dict(ms=ms, vis=vis_model, status=st)
        del plan, gg, gd, accm, model_buf
    v0 = results[0]["vis"][0]
    err_plain = {f: float(torch.linalg.norm(results[f]["vis"][0] - v0) / torch.linalg.norm(v0)) for f in (1, 2)}
    # FP64 DFT of the model image at a sample of gridded (row, channel) points, pol 0
    st = results[0]["status"]                     # (nr, nchan) Fortran
    rows, chans = np.nonzero(st == 3)
    rng = np.random.default_rng(5)
    k = rng.choice(len(rows), min(4096, len(rows)), replace=False)
    rows, chans = rows[k], chans[k]
    cell = w["cell"] * ARCSEC
    xs, ys = np.nonzero(img[:, :, 0, 0])
    flux = torch.tensor(img[xs, ys, 0, 0].astype(np.float64), device="cuda")
    lm = torch.tensor(np.stack([(xs - nx // 2) * cell, (ys - nx // 2) * cell], 1), device="cuda")
    nn = torch.sqrt(1 - lm[:, 0] ** 2 - lm[:, 1] ** 2) - 1
    U = d["uvw"][torch.tensor(rows, device="cuda")]
    f = torch.tensor(d["freq_np"][chans], device="cuda")
    ph = 2 * math.pi * (f / C_LIGHT)[:, None] * (U[:, 0:1] * lm[None, :, 0] + U[:, 1:2] * lm[None, :, 1]
                                                 + U[:, 2:3] * nn[None, :])
    dft = (flux[None] * torch.exp(1j * ph)).sum(1)
    ri, ci = torch.tensor(rows, device="cuda"), torch.tensor(chans, device="cuda")
    edft = {}
    for f in (0, 1, 2):
        pv = results[f]["vis"][0][ci, ri].to(torch.complex128)
        edft[f] = float(torch.linalg.norm(pv - dft) / torch.linalg.norm(dft))
    names = {0: "tabulated", 1: "learned_planes", 2: "learned_continuous"}
    out.update({
        "mvis_s": {names[f]: round(nvis / (results[f]["ms"] / 1e3) / 1e6, 3) for f in (0, 1, 2)},
        "ms_per_step": {names[f]: round(results[f]["ms"], 3) for f in (0, 1, 2)},
        "degrid_rel_err_vs_tabulated": {names[f]: err_plain[f] for f in (1, 2)},
        "degrid_rel_err_vs_dft": {**{names[f]: edft[f] for f in (0, 1, 2)}, "samples": int(len(rows))},
        "tolerance": 1e-3,
    })
    ok = [f for f in (1, 2) if err_plain[f] <= 1e-3]
    out["cf_form_kept"] = (names[ok[0]] if ok else
                           "tabulated (fallback: the learned forms differ from the tabulated path by more than 1e-3)")
    return out


def e2e_b200(args, w, d, ps, axes, img):
    """The same step through the IVisGridder C-ABI calls with pinned host
    buffers: initialiseDegrid, degrid (host cube in/out), initialiseGrid, grid,
    finaliseGrid (image to host)."""
    import torch
    from yandasoft_b200 import gridder as G
    npol, nchan, nrow = d["npol"], d["nchan"], d["nrow"]
    vis_h = torch.empty(d["vis"].shape, dtype=d["vis"].dtype, pin_memory=True)
    vis_h.copy_(d["vis"])
    model_h = torch.zeros(d["vis"].shape, dtype=d["vis"].dtype, pin_memory=True)
    uvw_h = torch.from_numpy(d["uvw_np"]).pin_memory()
    freq_h = torch.from_numpy(d["freq_np"]).pin_memory()

    vis_np = vis_h.numpy().view(np.complex64).reshape(-1)
    cube = vis_np.reshape((nrow, nchan, npol), order="F")
    mcube = model_h.numpy().view(np.complex64).reshape(-1).reshape((nrow, nchan, npol), order="F")
    uvw_np = uvw_h.numpy()
    freq_np = freq_h.numpy()
    acc = G.Accessor(uvw_np, freq_np, cube)
    accm = G.Accessor(uvw_np, freq_np, mcube)
    gd = G.VisGridderFactory.make(ps)
    gg = G.VisGridderFactory.make(ps)
    nx = w["nx"]
    out = np.zeros((nx, nx, npol, 1), dtype=np.float32, order="F")

    def step():
        gd.initialiseDegrid(axes, img)
        gd.degrid(accm)
        gg.initialiseGrid(axes, (nx, nx, npol, 1))
        gg.grid(acc)
        gg.finaliseGrid(out)

    step()   # warm (CF generation, allocations)
    torch.cuda.synchronize()
    k = max(1, args.steps)
    t0 = time.perf_counter()
    for _ in range(k):
        step()
    torch.cuda.synchronize()
    t = (time.perf_counter() - t0) / k
    # one more step, each call timed on its own (the calls return with their
    # results on the host, so the host clock brackets each)
    parts = {}
    for name, fn in (("initialiseDegrid", lambda: gd.initialiseDegrid(axes, img)), ("degrid", lambda: gd.degrid(accm)),
                     ("initialiseGrid", lambda: gg.initialiseGrid(axes, (nx, nx, npol, 1))),
                     ("grid", lambda: gg.grid(acc)), ("finaliseGrid", lambda: gg.finaliseGrid(out))):
        t1 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        parts[name] = round(1e3 * (time.perf_counter() - t1), 1)
    nvis = nrow * nchan * npol
    h2d = nvis * 8 * 2 + nrow * 24 * 2 + nchan * 8 * 2 + img.nbytes
    d2h = nvis * 8 + out.nbytes
    return {"value": round(nvis / t / 1e6, 3), "unit": "Mvis/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": round(t * 1e3, 2),
            "path": "C-ABI initialiseDegrid+degrid+initialiseGrid+grid+finaliseGrid, pinned host buffers",
            "calls_ms": parts, **copy_bound(h2d, d2h)}


def pcie_bandwidth(nbytes=1 << 30):
    """Pinned host <-> device copy bandwidth (GB/s) of one nbytes copy each
    way, best of three, CUDA events on the copying stream: the bound of the
    end-to-end path's copies."""
    import torch
    h = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dv = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    best = {"h2d": 0.0, "d2h": 0.0}
    with torch.cuda.stream(st):
        for _ in range(3):
            for k in ("h2d", "d2h"):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                if k == "h2d":
                    dv.copy_(h, non_blocking=True)
                else:
                    h.copy_(dv, non_blocking=True)
                e1.record(st)
                st.synchronize()
                best[k] = max(best[k], nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del h, dv
    return best


def copy_bound(h2d, d2h):
    """The copy-bound time (ms) of a step moving h2d bytes up and d2h down with
    the two directions overlapped, at the measured pinned bandwidth."""
    bw = pcie_bandwidth()
    return {"pcie_gbs": {k: round(v, 1) for k, v in bw.items()},
            "copy_bound_ms": round(1e3 * max(h2d / (bw["h2d"] * 1e9), d2h / (bw["d2h"] * 1e9)), 1)}


def ctypes_ptr(t):
    return t.data_ptr()


def run_reference(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    if torch.cuda.is_available():
        d = gen_device(w)
    else:
        raise SystemExit("the reference arm needs the same synthetic generator (GPU)")
    times = []
    vals = []
    if w["gridder"] == "AWProject":
        for s in range(args.warmup + args.steps):
            v, inf = cpu_baseline_aw(w, d, target_s=8.0)
            if s >= args.warmup:
                vals.append(v)
                times.append(inf["seconds"])
        cores, sample, support = inf["cores"], inf["sample"], None
    else:
        # gridders, grids and chunks made once; each step times one degrid +
        # grid pass of every thread's gridders
        cb = CpuBaseline(w, d, target_s=8.0)
        for s in range(args.warmup + args.steps):
            v, t = cb.run()
            if s >= args.warmup:
                vals.append(v)
                times.append(t)
        cores, sample, support = cb.threads, cb.sample, cb.support
    value = float(np.mean(vals))
    npol = d["npol"]
    cfg = {"workload": w["name"], "gridder": w["gridder"], "vis_samples": int(d["nrow"] * d["nchan"] * npol),
           "rows": int(d["nrow"]), "channels": d["nchan"], "pols": npol, "grid": [w["nx"], w["nx"], npol, 1],
           "oversample": w["oversample"]}
    if support is not None:
        cfg.update(support=support, taps_per_sample=(2 * support + 1) ** 2)
    cfg["step"] = "one degrid pass + one grid pass over a bounded row sample of the workload, on the host cores"
    line = {"metric": METRIC, "impl": "reference",
            "value": round(value, 4), "unit": "Mvis/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * float(np.mean(times)), 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; see bench.py workload())",
            "config": cfg,
            "cpu_baseline": {"value": round(value, 4), "unit": "Mvis/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "Mvis/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def batch_instances(n, seed=7, scale=1.0):
    """Config 3: n imaging instances generated as config 0 (36 antennas in a
    6 km disk, WProject, 20 sources, noise 0.01) with their own seeds, grid
    sizes drawn from {512, 1024, 2048, 4096}^2 (field of view 1.1-4.6 deg),
    visibility counts log-uniform in [1e5, 5e7] and 1-32 channels."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = int(rng.choice([512, 1024, 2048, 4096]))
        nvis = float(np.exp(rng.uniform(math.log(1e5), math.log(5e7)))) * scale
        nchan = int(rng.integers(1, 33))
        ntime = max(1, int(round(nvis / (630 * nchan))))
        w = workload(0)
        w.update(name="instance%02d" % i, nx=nx, cell=8.0 if nx <= 2048 else 4.0, nchan=nchan, duration=ntime * 10.0,
                 seed=1000 + i, nwplanes=33)
        out.append(w)
    return out


def run_batch(args):
    """Config 3: `instances` independent imaging instances, each a degridder
    with its model and a gridder for the residual over a device-resident
    chunk, recorded as one CUDA graph (yandasoft_b200.gridder.MajorCycle) and
    replayed for `cycles` major cycles.  value = visibility samples degridded
    and gridded per second over all instances and cycles."""
    import torch
    from yandasoft_b200 import build
    from yandasoft_b200 import gridder as G
    build.build()
    G.load()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ws = batch_instances(args.instances, scale=args.scale)
    t0 = time.perf_counter()
    insts, dgs, ggs, accs, nvis, shapes = [], [], [], [], 0, []
    for w in ws:
        d = gen_device(w)
        ps = parset_for(w, d["wmax"])
        cell = w["cell"] * ARCSEC
        axes = G.Axes(cell, cell)
        nx = w["nx"]
        acc = G.Accessor(d["uvw"], d["freq"], d["vis"], shape=(d["nrow"], d["nchan"], d["npol"]))
        gd = G.VisGridderFactory.make(ps)
        gg = G.VisGridderFactory.make(ps)
        if args.variant:
            gd.set_grid_variant(args.variant)
            gg.set_grid_variant(args.variant)
        gd.initialiseDegrid(axes, model_image(w, d["sky"], d["npol"]))
        gg.initialiseGrid(axes, (nx, nx, d["npol"], 1))
        insts.append(d)
        dgs.append(gd)
        ggs.append(gg)
        accs.append(acc)
        nvis += d["nrow"] * d["nchan"] * d["npol"]
        shapes.append((nx, int(d["nrow"] * d["nchan"])))
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    cyc = G.MajorCycle(dgs, ggs, accs)
    t_build = time.perf_counter() - t0
    supports = sorted({g.support()[0] for g in ggs})
    cyc.run(1)                                   # warm replay
    with ClockSampler(0) as clk:
        ms = cyc.run(args.cycles)
    launches = G.kernel_launch_count()
    line = {
        "metric": "major-cycle degrid+subtract+grid Mvis/s over %d instances on 1 B200 (one CUDA graph)"
                  % len(ws),
        "value": round(nvis * args.cycles / (ms / 1e3) / 1e6, 3), "unit": "Mvis/s", "n_gpus": 1,
        "steps": args.cycles, "warmup": 1, "ms_per_step": round(ms / args.cycles, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded per instance)",
        "config": {"workload": "config3_batched_major_cycle", "instances": len(ws), "vis_samples": int(nvis),
                   "grid_sizes": sorted({s[0] for s in shapes}), "supports": supports,
                   "graph_nodes": cyc.nodes(), "setup_s": round(t_build, 2), "generate_s": round(t_gen, 2),
                   "step": "one major cycle: every instance degrids its model, subtracts, grids the residual"},
        "clocks": clk.summary(),
        "gpu_launches": int(cyc.nodes() * args.cycles),
        "gpu_launches_note": "graph nodes (kernels and memsets) x cycles",
    }
    del launches
    print(json.dumps(line))


def run_beams(args, w):
    """Config 2: one AWProject imaging instance per beam (its rows phased to
    the beam's centre, image centred there, a CF set per channel), a degridder
    with the beam's model and a gridder for the residual each, over
    device-resident chunks; the degrid -> subtract -> grid sequence of all
    beams recorded as one CUDA graph (yandasoft_b200.gridder.MajorCycle) and
    replayed.  value = visibility samples degridded and gridded per second
    over all beams; e2e = the same through the C-ABI calls of each beam with
    pinned host buffers."""
    import torch
    from yandasoft_b200 import build
    from yandasoft_b200 import gridder as G
    build.build()
    G.load()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    d = gen_device(w)
    t_gen = time.perf_counter() - t0
    nx, npol, nchan = w["nx"], d["npol"], d["nchan"]
    cell = w["cell"] * ARCSEC
    axes = G.Axes(cell, cell)
    ps = parset_for(w, d["wmax"])
    nvis = d["nrow"] * nchan * npol
    foot = d["foot"]
    beams = []
    t0 = time.perf_counter()
    for b in range(w["nbeam"]):
        rows = np.nonzero(d["feed_np"] == b)[0]
        ri = torch_index(rows)
        uvw_b = d["uvw"][ri].contiguous()
        vis_b = d["vis"][:, :, ri].contiguous()
        acc = G.Accessor(uvw_b, d["freq"], vis_b, shape=(len(rows), nchan, npol))
        sky_b = d["sky"].copy()
        sky_b[:, 1] -= math.sin(foot[b, 0]) * math.cos(foot[b, 1])
        sky_b[:, 2] -= math.sin(foot[b, 1])
        gd = G.VisGridderFactory.make(ps)
        gd.initialiseDegrid(axes, model_image(w, sky_b, npol))
        gg = G.VisGridderFactory.make(ps)
        gg.initialiseGrid(axes, (nx, nx, npol, 1))
        beams.append(dict(rows=rows, uvw=uvw_b, vis=vis_b, acc=acc, gd=gd, gg=gg, sky=sky_b))
    cyc = G.MajorCycle([x["gd"] for x in beams], [x["gg"] for x in beams], [x["acc"] for x in beams])
    t_build = time.perf_counter() - t0
    ms_cf = sum(x["gg"].stats()["ms_cf"] + x["gd"].stats()["ms_cf"] for x in beams)
    support, os_, ncf = beams[0]["gg"].support()
    for _ in range(args.warmup):
        cyc.run(1)
    with ClockSampler(0) as clk:
        ms = cyc.run(args.steps)
    ms_step = ms / args.steps
    taps = (2 * support + 1) ** 2
    line = {
        "metric": METRIC, "cf_form": "plain (tabulated CF)",
        "value": round(nvis / (ms_step / 1e3) / 1e6, 3), "unit": "Mvis/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; see bench.py workload())",
        "config": {"workload": w["name"], "gridder": "AWProject", "vis_samples": int(nvis), "rows": int(d["nrow"]),
                   "channels": nchan, "pols": npol, "beams": w["nbeam"], "grid_per_beam": [nx, nx, npol, 1],
                   "cell_arcsec": w["cell"], "support": int(support), "taps_per_sample": taps,
                   "oversample": w["oversample"], "dish_m": w["dish"], "blockage_m": w["blockage"],
                   "footprint": "6x6 at %g deg" % w["pitch"],
                   "step": "every beam: degrid model, subtract, grid residual (one CUDA graph, %d nodes)"
                           % cyc.nodes(),
                   "l2": "inputs (%.2f GB of visibilities, %.1f GB of CF caches) larger than L2"
                         % (nvis * 8 / 1e9, 2 * w["nbeam"] * ncf * taps * 8 / 1e9),
                   "generate_s": round(t_gen, 1), "setup_s": round(t_build, 1)},
        "cf_cache": {"cf_matrices_per_gridder": int(ncf), "gridders": 2 * w["nbeam"],
                     "built_on": "GPU (cuFFT + own kernels) when each gridder first sees its chunk",
                     "gpu_build_s_all_gridders": round(ms_cf / 1e3, 3),
                     "bytes_per_gridder": int(ncf * taps * 8),
                     "padded_bytes_per_gridder": int(ncf * ((2 * support + 1 + 15) // 16 * 16) ** 2 * 8)},
        "binding": {"resource": "shared memory", "note": "k_grid and k_degrid_t, whole step",
                    "taps_per_s": round(2 * taps * nvis / (ms_step / 1e3), 1)},
        "clocks": clk.summary(),
        "gpu_launches": int(cyc.nodes() * args.steps),
        "gpu_launches_note": "graph nodes (kernels and memsets) x steps",
    }
    del cyc
    if not args.no_learned:
        try:
            # a central beam: its field holds sources (the corner beams' fields hold none)
            line["learned"] = learned_leg_aw(args, w, d, beams[min(14, len(beams) - 1)], ps, axes)
        except Exception as e:  # the learned leg must not hide the plain result
            line["learned"] = {"error": repr(e)}
    for x in beams:
        del x["gd"], x["gg"], x["acc"]
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    if not args.no_e2e:
        line["e2e"] = e2e_beams(args, w, d, beams, ps, axes)
    if not args.no_cpu:
        try:
            v, inf = cpu_baseline_aw(w, d, ps)
            line["cf_cache"].update(inf["cf"])
            line["cpu_baseline"] = {"value": round(v, 4), "unit": "Mvis/s", "cores": inf["cores"], "kind": "port",
                                    "sample": inf["sample"], "seconds": round(inf["seconds"], 2),
                                    "single_core": inf.get("single_core")}
        except Exception as e:  # the baseline must not hide the GPU result
            line["cpu_baseline"] = {"value": None, "error": repr(e)}
    print(json.dumps(line))


def learned_leg_aw(args, w, d, beam, ps, axes):
    """The learned CF beside the tabulated one for one beam's AWProject
    instance: the network is trained on the gridder's own CF cache (every
    channel's CF set, w, frequency and beam as inputs), then a degrid + grid
    step runs with the network evaluated inside the kernels at the tabulated
    planes (form 1) on a slice of the beam's rows.  Reports Mvis/s of both
    forms, CF memory, the degridded-visibility error of the learned form
    against the tabulated one, and the form kept (the learned one only within
    1e-3 of the tabulated path)."""
    import torch
    from yandasoft_b200 import gridder as G
    npol, nchan = d["npol"], d["nchan"]
    gg0 = beam["gg"]
    rep = gg0.learned_train(steps=args.learned_steps, seed=w["seed"] + 11)
    nr = max(1, int(len(beam["rows"]) * args.learned_rows * 10))
    uvw = beam["uvw"][:nr].contiguous()
    vis = beam["vis"][:, :, :nr].contiguous()
    acc = G.Accessor(uvw, d["freq"], vis, shape=(nr, nchan, npol))
    img = model_image(w, beam["sky"], npol)
    nx = w["nx"]
    res = {}
    for form in (0, 1):
        gg = gg0.clone()
        gg.set_cf_form(form)
        gg.initialiseGrid(axes, (nx, nx, npol, 1))
        gd = gg0.clone()
        gd.set_cf_form(form)
        gd.initialiseDegrid(axes, img)
        mb = torch.zeros_like(vis)
        accm = G.Accessor(uvw, d["freq"], mb, shape=(nr, nchan, npol))
        plan = gg.plan(acc)
        st = torch.cuda.ExternalStream(gg.stream_handle())
        gd.degrid_plan(plan, accm)
        gg.grid_plan(plan, acc)
        gg.synchronize()
        gd.synchronize()
        vm = mb.clone()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        gd.degrid_plan(plan, accm)
        gg.grid_plan(plan, acc)
        e1.record(st)
        torch.cuda.synchronize()
        res[form] = (e0.elapsed_time(e1), vm)
        del plan, gg, gd, accm, mb
    nvis = nr * nchan * npol
    ref = float(torch.linalg.norm(res[0][1]))
    err = float(torch.linalg.norm(res[1][1] - res[0][1])) / ref if ref > 0 else None
    return {"trained_on": "the beam's CF cache: %d planes (%d w x %d channels), oversample %d"
                          % (w["nwplanes"] * nchan, w["nwplanes"], nchan, w["oversample"]),
            "train_steps": rep["steps"], "train_ms": round(rep["train_ms"], 1), "final_loss": rep["final_loss"],
            "network_bytes": int(rep["network_bytes"]), "cf_table_bytes": int(rep["cf_table_bytes"]),
            "slice": "first %d of the beam's %d rows, all %d channels x %d pols" % (nr, len(beam["rows"]), nchan, npol),
            "mvis_s": {"tabulated": round(nvis / (res[0][0] / 1e3) / 1e6, 3),
                       "learned_planes": round(nvis / (res[1][0] / 1e3) / 1e6, 3)},
            "degrid_rel_err_vs_tabulated": {"learned_planes": err}, "tolerance": 1e-3,
            "cf_form_kept": "learned_planes" if err is not None and err <= 1e-3 else
                            "tabulated (fallback: the learned form differs from the tabulated path by more than 1e-3)"}


def e2e_beams(args, w, d, beams, ps, axes):
    """Every beam through the IVisGridder C-ABI calls with pinned host
    buffers: initialiseDegrid, degrid (host cube in and out), initialiseGrid,
    grid (host cube in), finaliseGrid (image to host)."""
    import torch
    from yandasoft_b200 import gridder as G
    nx, npol, nchan = w["nx"], d["npol"], d["nchan"]
    host = []
    for x in beams:
        nr = len(x["rows"])
        vh = torch.empty(x["vis"].shape, dtype=x["vis"].dtype, pin_memory=True)
        vh.copy_(x["vis"])
        mh = torch.zeros(x["vis"].shape, dtype=x["vis"].dtype, pin_memory=True)
        uh = torch.empty(x["uvw"].shape, dtype=x["uvw"].dtype, pin_memory=True)
        uh.copy_(x["uvw"])
        cube = vh.numpy().view(np.complex64).reshape(-1).reshape((nr, nchan, npol), order="F")
        mcube = mh.numpy().view(np.complex64).reshape(-1).reshape((nr, nchan, npol), order="F")
        host.append(dict(keep=(vh, mh, uh), acc=G.Accessor(uh.numpy(), d["freq_np"], cube),
                         accm=G.Accessor(uh.numpy(), d["freq_np"], mcube), img=model_image(w, x["sky"], npol)))
    out = np.zeros((nx, nx, npol, 1), dtype=np.float32, order="F")
    # one degridder and one gridder serve every beam in turn: each beam's
    # chunk has the same frequencies and its beam at the image centre, so the
    # CF caches built for the first stay valid
    gd, gg = G.VisGridderFactory.make(ps), G.VisGridderFactory.make(ps)

    def step():
        for h in host:
            gd.initialiseDegrid(axes, h["img"])
            gd.degrid(h["accm"])
            gg.initialiseGrid(axes, (nx, nx, npol, 1))
            gg.grid(h["acc"])
            gg.finaliseGrid(out)

    step()   # warm (CF generation, allocations)
    torch.cuda.synchronize()
    k = max(1, min(args.steps, 2))
    t0 = time.perf_counter()
    for _ in range(k):
        step()
    torch.cuda.synchronize()
    t = (time.perf_counter() - t0) / k
    nvis = d["nrow"] * nchan * npol
    h2d = nvis * 8 * 2 + d["nrow"] * 24 * 2 + len(host) * (nchan * 8 * 2 + host[0]["img"].nbytes)
    d2h = nvis * 8 + len(host) * out.nbytes
    return {"value": round(nvis / t / 1e6, 3), "unit": "Mvis/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": round(t * 1e3, 2),
            "path": "per beam: C-ABI initialiseDegrid+degrid+initialiseGrid+grid+finaliseGrid, pinned host buffers",
            **copy_bound(h2d, d2h)}


def main():
    args = parse()
    if args.config == 3:
        run_batch(args)
        return
    w = workload(args.config, args.scale)
    if args.grid_nx:
        w.update(nx=args.grid_nx, cell=args.cell_arcsec or w["cell"])
    if args.impl == "reference":
        run_reference(args, w)
    elif args.config == 2:
        run_beams(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()
