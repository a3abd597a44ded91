#!/usr/bin/env python
"""Headline benchmark: antenna-pair x source terms/s on the HERA-350-like workload.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]
                    [--config 2|3|4 [--sparse] [--nsrc N --nfreq F --ntimes T]]

--config 3 is the precision form (1,000,000 isotropic power-law sources, one
slice per job by default; --sparse times its 5,000 seeded pairs on the
VectorDot path), --config 4 the batched form (500,000 sources, 256 frequencies
x 64 LSTs over 6 h).  Without --config:

Workload (one "step"): the whole config-2 job -- 350 antennas (320 on a 14.6 m
hexagon + 30 outriggers), 196,608 sources (nside = 128 equal-area centres,
lognormal flux), 64 frequencies x 16 LSTs, polarised (2 feeds x 2 axes), 4
gridded beams with per-antenna beam_idx.  Seeded synthetic inputs.

Terms per job = sum over (f, t) of Nant^2 * n_t, n_t the sources above the
horizon at time t (the reference's all-pairs output, wrapper.py:168-174).

`value` times graph replays of the job with inputs resident in HBM; `e2e` times
``simulate_vis`` with host numpy inputs and outputs (H2D and D2H inside the
timed region).  `roofline` is the Hermitian-product kernel (mvb_herk), timed
live with CUDA events on its own launch stream.  `cpu_baseline` is the FP64
oracle on a bounded sample of the same workload on this host's cores, and
`plain_gpu` a complex64 torch restatement of the reference GPU driver (per-slice
stages, full cgemm, per-time device->host copy) on a sample of slices.

With --impl reference, rank 0 times the reference's CPU algorithm (the FP64
oracle restatement; the reference package itself cannot be imported here:
astropy / pyuvdata are absent) on one slice of the workload per step.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "antenna-pair×source terms/s vs plain GPU path at rel.err≤1e-6; p50/p99 latency"
UNIT = "antenna-pair×source terms/s"
SPEED_OF_LIGHT = 299792458.0


GEMM_PRECISION = {
    "fp16x3": "2-term fp16 split of the power-of-two-scaled Z (3 products)",
    "bf16x6": "3-term bf16 split (6 products)",
    "bf16x3": "2-term bf16 split (3 products)",
    "tf32x3": "2-term tf32 split (3 products)",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--gemm-mode", default="fp16x3", choices=sorted(GEMM_PRECISION))
    ap.add_argument("--k-chunk", type=int, default=None)
    ap.add_argument("--config", type=int, default=2, choices=[2, 3, 4],
                    help="2: HERA-350-like job (default); 3: 1e6 power-law sources; 4: 500k sources, 256 f x 64 LST")
    ap.add_argument("--sparse", action="store_true", help="config 3: the 5,000 seeded pairs on the VectorDot path")
    ap.add_argument("--pairs", default="all", choices=["all", "redundant"],
                    help="redundant: one pair per redundant baseline group (get_redundancies) on the VectorDot path")
    ap.add_argument("--sky", default="stokes", choices=["stokes", "pol"],
                    help="pol: a seeded polarised sky (coherency fluxes) instead of Stokes I")
    ap.add_argument("--rotation", default="lst", choices=["lst", "erfa"],
                    help="erfa: the apparent-place rotation from per-time astrometry parameters (refreshed every step)")
    ap.add_argument("--beam", default="grid", choices=["grid", "fits"],
                    help="fits: config 2's beam written to and read from a beamfits file at 100 and 200 MHz (a "
                         "chromatic beam: simulate_vis runs one job per frequency); times simulate_vis end to end")
    ap.add_argument("--pair-kernel", default="auto", choices=["auto", "vecdot", "herk"],
                    help="--sparse: per-pair sums, the Hermitian product with a pair gather, or the cost model's choice")
    ap.add_argument("--nsrc", type=int, default=None, help="source count (configs 3 and 4)")
    ap.add_argument("--nfreq", type=int, default=None, help="default 64 (config 2), 1 (config 3), 256 (config 4)")
    ap.add_argument("--ntimes", type=int, default=None, help="default 16 (config 2), 1 (config 3), 64 (config 4)")
    ap.add_argument("--nside", type=int, default=128, help="config-2 sky pixelisation (128: 196,608 sources)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--serve", action="store_true", help="served form: Poisson job stream, p50/p99 latency")
    ap.add_argument("--serve-jobs", type=int, default=2000)
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-nsrc-max", type=int, default=500_000)
    ap.add_argument("--serve-max-active", type=int, default=32)
    ap.add_argument("--serve-turns-ahead", type=int, default=2,
                    help="served form: turns enqueued ahead of the GPU (0: no bound)")
    ap.add_argument("--serve-hbm-frac", type=float, default=0.75,
                    help="served form: admission budget as a fraction of the free device memory")
    ap.add_argument("--serve-turn-terms", type=float, default=2e11,
                    help="served form: terms per turn, least work left first (0: every job every turn)")
    ap.add_argument("--serve-small-terms", type=float, default=2e11,
                    help="jobs of at most this many terms are the server's priority class (0: none)")
    return ap.parse_args()


# ----------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.path is None or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def load_config(args, host_only: bool = False) -> tuple[dict, str]:
    """The workload named by --config, with its description.  ``host_only``: build
    it without the GPU library (the reference arm; redundant pairs then come from
    the oracle's restatement of get_redundancies)."""
    from matvis_b200 import workloads as wl

    if args.config == 2:
        cfg = wl.config2(nfreq=args.nfreq or 64, ntimes=args.ntimes or 16, nside=args.nside)
        desc = (f"config2 HERA-350-like: 350 ant x {len(cfg['ra'])} src x {len(cfg['freqs'])} freq x "
                f"{len(cfg['lsts'])} LST, polarised 2x2, 4 gridded beams + beam_idx; one job per step")
    elif args.config == 3:
        cfg = wl.config3(nsrc=args.nsrc or 1_000_000, nfreq=args.nfreq or 1, ntimes=args.ntimes or 1)
        if not args.sparse:
            cfg["antpairs"] = None
        desc = (f"config3: 350 ant x {len(cfg['ra'])} isotropic power-law src x {len(cfg['freqs'])} freq x "
                f"{len(cfg['lsts'])} LST, polarised 2x2, 4 gridded beams; "
                + (f"{len(cfg['antpairs'])} seeded pairs on the VectorDot path" if args.sparse else "all pairs")
                + "; one job per step")
    else:
        cfg = wl.config4(nsrc=args.nsrc or 500_000, nfreq=args.nfreq or 256, ntimes=args.ntimes or 64)
        desc = (f"config4: 350 ant x {len(cfg['ra'])} isotropic power-law src x {len(cfg['freqs'])} freq x "
                f"{len(cfg['lsts'])} LST over 6 h, polarised 2x2, 4 gridded beams; one job per step")
    if args.sparse and args.config != 3:
        raise SystemExit("--sparse applies to config 3")
    if args.pairs == "redundant":
        if host_only:
            from oracle.oracle import redundant_antpairs
        else:
            from matvis_b200.pairs import redundant_antpairs

        cfg["antpairs"] = redundant_antpairs(cfg["antpos"])
        desc += f"; {len(cfg['antpairs'])} redundant-baseline pairs on the VectorDot path"
    return cfg, desc


def terms_per_job(cfg, astrom=None) -> tuple[float, np.ndarray]:
    """Npairs * sum_t n_t * Nf (Npairs = Nant^2, or the listed pairs), with n_t from
    the same FP64 fixed-order rotation as the kernels (for the ERFA rotation its
    rigid part, BPN then CIRS -> ENU: aberration and light deflection, ~1e-4 rad,
    change the count by ~1e-5)."""
    from matvis_b200.coordinates import atioq_matrix, eci_to_enu_matrix, point_source_crd_eq

    eci = point_source_crd_eq(cfg["ra"], cfg["dec"])
    counts = []
    for t, lst in enumerate(cfg["lsts"]):
        R = (eci_to_enu_matrix(lst, cfg["latitude"]) if astrom is None
             else atioq_matrix(astrom[t]) @ np.asarray(astrom[t]["bpn"]).reshape(3, 3))
        z = (R[2, 0] * eci[0] + R[2, 1] * eci[1]) + R[2, 2] * eci[2]
        counts.append(int((z > 0).sum()))
    nant = len(cfg["antpos"])
    npairs = nant * nant if cfg.get("antpairs") is None else len(cfg["antpairs"])
    return float(npairs * sum(counts) * len(cfg["freqs"])), np.array(counts)


# ----------------------------------------------------------------------------- plain GPU path
def plain_gpu_sample(cfg, slices):
    """Complex64 torch restatement of the reference GPU driver (gpu/gpu.py:197-254) on
    the listed (f, t) slices: FP32 rotation, horizon gather with a host count,
    bilinear beam via grid_sample, FP32 phase, per-antenna Z loop, full complex64
    matmul (TF32 off) or, for a pair list, one matmul per pair (GPUVectorDot,
    gpu/matprod.py:66-98), device->host copy of the result per slice.  The first
    slice runs once untimed (warm-up).  Returns the rate and, per listed slice, the
    host visibilities in the reference layout (npairs, F, F)."""
    import torch
    import torch.nn.functional as Fnn

    from matvis_b200.coordinates import eci_to_enu_matrix, point_source_crd_eq

    torch.backends.cuda.matmul.allow_tf32 = False
    dev = torch.device("cuda")
    eci = torch.as_tensor(point_source_crd_eq(cfg["ra"], cfg["dec"]), dtype=torch.float32, device=dev)
    antpos = torch.as_tensor(cfg["antpos"], dtype=torch.float32, device=dev)
    beams = cfg["beams"]
    grids = torch.as_tensor(np.stack([b.data for b in beams]), dtype=torch.complex64, device=dev)  # B,X,F,za,az
    bidx = np.asarray(cfg["beam_idx"])
    nant = len(cfg["antpos"])
    pairs = None if cfg.get("antpairs") is None else [(int(i), int(j)) for i, j in cfg["antpairs"]]
    npairs = nant * nant if pairs is None else len(pairs)
    nb, X, F, nza, naz = grids.shape
    flux = torch.as_tensor(np.sqrt(0.5 * cfg["fluxes"]), dtype=torch.float32, device=dev)
    terms = 0.0
    times = []
    out = []
    for k, (f, t) in enumerate([slices[0]] + list(slices)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        R = torch.as_tensor(eci_to_enu_matrix(cfg["lsts"][t], cfg["latitude"]), dtype=torch.float32, device=dev)
        top = R @ eci
        idx = torch.nonzero(top[2] > 0).squeeze(1)
        n = int(idx.numel())  # host sync, as len(where) in the reference
        crd = top[:, idx]
        e, nn = crd[0], crd[1]
        az = torch.remainder(0.5 * np.pi - torch.atan2(e, nn), 2 * np.pi)
        za = 0.5 * np.pi - torch.asin(torch.sqrt(torch.clamp(1 - e * e - nn * nn, min=0)))
        gx = az / (2 * np.pi) * 2 - 1  # grid_sample coords in [-1, 1], align_corners=True
        gy = za / (0.5 * np.pi) * 2 - 1
        grid = torch.stack([gx, gy], -1).view(1, 1, n, 2)
        planes = torch.view_as_real(grids).permute(0, 1, 2, 5, 3, 4).reshape(1, nb * X * F * 2, nza, naz)
        bv = Fnn.grid_sample(planes, grid, mode="bilinear", align_corners=True).view(nb, X, F, 2, n)
        beam = torch.complex(bv[:, :, :, 0], bv[:, :, :, 1]).permute(0, 2, 1, 3)  # B,F,X,n
        phase = (2 * np.pi * float(cfg["freqs"][f]) / SPEED_OF_LIGHT) * (antpos @ crd)
        ext = torch.polar(torch.ones_like(phase), phase) * flux[idx, f][None, :]
        z = ext[:, None, None, :].expand(nant, F, X, n).clone()
        for a in range(nant):  # per-antenna loop of core/getz.py:95-96
            z[a] *= beam[int(bidx[a])]
        z = z.reshape(nant * F, X * n)
        if pairs is None:
            v = z.conj() @ z.T
        else:
            zz = z.view(nant, F, X * n)
            v = torch.stack([zz[aj] @ zz[ai].conj().T for ai, aj in pairs])
        vh = v.cpu()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if k > 0:  # the first pass is warm-up
            times.append(dt)
            terms += npairs * n
            if pairs is None:  # V[i F + q, j F + p] -> out[i A + j, p, q] (cpu/matprod.py:21-30)
                vh = vh.numpy().reshape(nant, F, nant, F).transpose(0, 2, 3, 1).reshape(nant * nant, F, F)
            else:
                vh = vh.numpy()
            out.append(vh)
    return {"value": terms / sum(times), "unit": UNIT, "slices": len(slices),
            "sample": f"{len(slices)} (f, t) slices of the workload, complex64, TF32 off"}, out


# ----------------------------------------------------------------------------- CPU oracle
def above_horizon(cfg, t, astrom=None) -> int:
    return int(terms_per_job(dict(cfg, lsts=np.asarray(cfg["lsts"])[t:t + 1], freqs=np.zeros(1), antpairs=None),
                             None if astrom is None else astrom[t:t + 1])[1][0])


def accuracy_slices(cfg) -> list[tuple[int, int]]:
    """Three (f, t) slices spread over the job: first, middle, last."""
    nf, nt = len(cfg["freqs"]), len(cfg["lsts"])
    out = []
    for s in [(0, 0), (nf // 2, nt // 2), (nf - 1, nt - 1)]:
        if s not in out:
            out.append(s)
    return out


def oracle_slices(cfg, slices, nsrc_sample: int | None = None):
    """FP64 oracle (the reference CPU algorithm) on the listed (f, t) slices, all
    antennas and pairs; the sky is the workload's own, or a seeded subset of
    ``nsrc_sample`` sources.  Returns (terms/s, seconds, sample text, [vis per
    slice, (nant^2, 2, 2) complex128])."""
    from oracle import oracle as orc

    from matvis_b200 import workloads as wl

    sub = cfg
    if nsrc_sample is not None and nsrc_sample < len(cfg["ra"]):
        sub = wl.subset(cfg, nsrc=nsrc_sample, seed=11)
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in sub["beams"]]
    antpos = np.asarray(sub["antpos"])
    terms = 0.0
    vis = []
    t0 = time.perf_counter()
    for f, t in slices:
        v = orc.simulate(antpos=antpos, freq=float(sub["freqs"][f]), lsts=np.asarray(sub["lsts"])[t:t + 1],
                         latitude=sub["latitude"], ra=sub["ra"], dec=sub["dec"], I_sky=sub["fluxes"][:, f],
                         beam_list=beams, polarized=True, beam_idx=sub["beam_idx"])
        vis.append(v[0])
        terms += len(antpos) ** 2 * above_horizon(sub, t)
    dt = time.perf_counter() - t0
    srcs = (f"all {len(cfg['ra'])} sources" if sub is cfg
            else f"{nsrc_sample} of {len(cfg['ra'])} sources (seeded subset)")
    return terms / dt, dt, (f"{len(slices)} (f, t) slice(s) {list(slices)} of the workload, all {len(antpos)} "
                            f"antennas and pairs, {srcs}, FP64 numpy/scipy oracle"), vis


def workload_config(args, cfg, desc, terms, counts) -> dict:
    """The ``config`` object of the JSON line, identical for both arms run with the
    same arguments (it names the workload only; how each arm computes it is
    reported elsewhere in the line)."""
    matprod = "VectorDot" if args.sparse or args.pairs != "all" else "MatMul"
    nant = len(cfg["antpos"])
    mpad = -(-2 * nant // 128) * 128
    plane_bytes = {"fp16x3": 8, "bf16x3": 8, "bf16x6": 12, "tf32x3": 16}[args.gemm_mode]
    panel_gb = mpad * 2 * int(np.max(counts)) * plane_bytes / 1e9
    return {
        "workload": desc,
        "matprod": matprod,
        "gemm_mode": args.gemm_mode,
        "terms_per_job": terms,
        "above_horizon_per_time": [int(c) for c in counts],
        "l2": f"inputs larger than L2: {len(cfg['ra'])} sources, and each (f, t) slice's Z panel is "
              f"{panel_gb:.2f} GB (126 MB L2)",
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg, desc = load_config(args, host_only=True)
    terms, counts = terms_per_job(cfg)
    # one (f, t) slice per step: all sources of config 2 (a few seconds on the host
    # cores), a 196,608-source seeded subset of the larger skies
    nsrc_sample = min(len(cfg["ra"]), 196_608)
    sl = accuracy_slices(cfg)
    for i in range(max(args.warmup, 0)):
        oracle_slices(cfg, [sl[i % len(sl)]], nsrc_sample)
    vals, dts = [], []
    for i in range(args.steps):
        v, dt, sample, _ = oracle_slices(cfg, [sl[i % len(sl)]], nsrc_sample)
        vals.append(v)
        dts.append(dt)
    value = float(np.median(vals))
    cores = os.cpu_count()
    sample = sample.replace(str([sl[(args.steps - 1) % len(sl)]]), "(one per step, cycling over %s)" % sl)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.median(dts)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, cfg, desc, terms, counts),
        "sample": sample,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference package not importable here (astropy, pyuvdata absent); its CPU algorithm is timed "
                "through the FP64 oracle restatement (oracle/oracle.py), pinned to fixtures from the reference "
                "code.  This arm loads no library of this repository.",
    }
    print(json.dumps(line), flush=True)


def herk_roofline(eng, args, dev) -> dict:
    """mvb_herk on the engine's last panel.  ``achieved`` counts the split's
    products on the upper triangle, P x 4 M (M+1) K flops per launch (P = 3 for
    fp16x3 / tf32x3 / bf16x3, 6 for bf16x6), against the tensor peak of the
    operands' precision (the measured bf16 burst; half of it for TF32, which has
    no measured peak).  Also reported: the useful flops alone (one product,
    ``useful_*``) and the flops the padded 128 x 128 tiles execute
    (``executed_tensor_*``)."""
    import torch

    from matvis_b200 import _lib

    panel = eng.zcalc.z
    M = eng.nant * eng.nfeed
    nlast = int(eng.n_above.item())
    kvalid = nlast * eng.nax
    kc = eng.k_chunk
    reps = 10
    hs = torch.cuda.Stream(device=dev)
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ws = eng.matprod.workspace(panel, kc)
    torch.cuda.synchronize()
    with torch.cuda.stream(hs):
        for r in range(reps + 2):
            if r == 2:
                h0.record(hs)
            _lib.check(_lib.lib.mvb_herk(_lib.ptr(panel.data), eng.matprod.mode, panel.Mpad, panel.Kcap,
                                         _lib.ptr(eng.n_above), 0, eng.nax, kc, eng.matprod.drain_ksteps, _lib.ptr(ws),
                                         ws.numel(),
                                         _lib.ptr(eng.status), _lib.stream_handle(hs)))
        h1.record(hs)
    torch.cuda.synchronize()
    herk_ms = h0.elapsed_time(h1) / reps
    algo_flops = 4.0 * M * (M + 1) * kvalid
    T = panel.Mpad // 128
    nprod = _lib.GEMM_PRODUCTS[_lib.GEMM_MODES[args.gemm_mode]]
    # 128 x 128 complex tiles: four real products per split product off the diagonal,
    # three on the T diagonal tiles (their imaginary half is W - W^T of one product)
    exec_flops = 2.0 * 128 * 128 * kvalid * nprod * (4 * (T * (T - 1) // 2) + 3 * T)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    peak_src = "measured" if "bf16_tflops" in peaks else "fallback"
    useful = algo_flops / (herk_ms / 1000.0) / 1e12
    achieved = nprod * useful
    tensor_peak = bf16_peak / 2 if args.gemm_mode.startswith("tf32") else bf16_peak
    # DRAM bytes per launch from an ncu capture (dram__bytes_read/write.sum) of the
    # nside-64 slice of this workload (K = 49,152, k_chunk 4096: 305.8 MB read, 24.4 MB
    # written over 12 x 21 work units), scaled by the columns read and the units written
    # (fp16x3: 4 planes x 2 B per row and column; other modes scale the panel read by their plane bytes)
    n_units = (T * (T + 1) // 2) * -(-kvalid // kc)
    plane_bytes = 2 * (3 if args.gemm_mode == "bf16x6" else 2) * (4 if args.gemm_mode.startswith("tf32") else 2)
    traffic = 305.779968e6 / 49152 * kvalid * plane_bytes / 8 + 24.417536e6 / 252 * n_units
    roofline = {
        "bound": "tensor", "achieved": achieved, "peak": tensor_peak, "unit": "TFLOP/s", "frac": achieved / tensor_peak,
        "flops_counted": f"{nprod} split products x 4 M (M+1) K (upper triangle incl. diagonal)",
        "useful_tflops": useful, "useful_frac_of_bf16": useful / bf16_peak,
        "traffic": traffic,
        "traffic_source": "ncu dram bytes of the nside-64 fp16x3 slice, scaled by columns, units and plane bytes",
        "peak_source": f"{peak_src} bf16 burst (MEASURED_PEAKS.json)"
                       + ("; TF32 counted at half of it" if args.gemm_mode.startswith("tf32") else ""),
        "kernel": f"mvb_herk {args.gemm_mode}: M={M}, K={kvalid}, k_chunk={kc}",
        "herk_ms": herk_ms,
        "algorithmic_flops_per_launch": algo_flops,
        "executed_tensor_tflops": exec_flops / (herk_ms / 1000.0) / 1e12,
        "executed_tensor_frac": exec_flops / (herk_ms / 1000.0) / 1e12 / tensor_peak,
    }
    return roofline


def vecdot_roofline(eng, dev) -> dict:
    """The pair kernel (+ its slice reduction) on the engine's last panel.
    Algorithmic bytes per launch: the Z rows of the antennas in the pair list
    read once (F rows x K x 8 B each) plus the FP64 slice partials written and
    read.  The staged kernel reads the panel from HBM once and runs from shared
    memory, so its bound is the shared-memory load rate (F x 8 B per column for
    a bundle's antenna i and for each of its 3 partners) and the FP32 pipe
    (8 F^2 flops per pair and column):
    both are reported against their nominal rates at the 1,965 MHz maximum SM
    clock (148 SMs x 128 B / clock; 148 x 128 FMA / clock)."""
    import torch

    from matvis_b200 import _lib

    panel = eng.zcalc.z
    mp = eng.matprod
    kvalid = int(eng.n_above.item()) * eng.nax
    reps = 10
    out = torch.empty_like(eng.vis[0, 0])
    hs = torch.cuda.Stream(device=dev)
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(hs):
        for r in range(reps + 2):
            if r == 2:
                h0.record(hs)
            mp.enqueue(panel, out, accumulate=False, stream=hs)
        h1.record(hs)
    torch.cuda.synchronize()
    ms = h0.elapsed_time(h1) / reps
    pairs = np.asarray(mp.antpairs)
    nrows = len(np.unique(pairs)) * eng.nfeed
    nsplit = -(-kvalid // mp.k_chunk)
    staged = mp.kernel == "staged"
    nslots = 3 * mp.nbundles if staged else len(pairs)  # pair steps computed, fillers included
    algo_bytes = nrows * kvalid * 8.0 + 2 * nsplit * nslots * eng.nfeed ** 2 * 16.0
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = algo_bytes / (ms / 1000.0) / 1e9
    name = "mvb_vecdot_staged" if staged else "mvb_vecdot"
    line = {
        "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
        "peak_source": ("measured" if "hbm_gbs" in peaks else "fallback") + " HBM copy (MEASURED_PEAKS.json)",
        "kernel": f"{name}: {len(pairs)} pairs, F={eng.nfeed}, K={kvalid}, k_chunk={mp.k_chunk}",
        "vecdot_ms": ms, "algorithmic_bytes_per_launch": algo_bytes,
    }
    fp32_tflops = 8.0 * eng.nfeed ** 2 * len(pairs) * kvalid / (ms / 1000.0) / 1e12
    nominal_fp32 = 148 * 128 * 2 * 1.965e9 / 1e12
    line["fp32_tflops"] = fp32_tflops
    line["fp32_frac_of_nominal"] = fp32_tflops / nominal_fp32
    if staged:
        smem_tbs = 4.0 * mp.nbundles * kvalid * eng.nfeed * 8 / (ms / 1000.0) / 1e12
        line["bundles"] = mp.nbundles
        line["bundle_fill"] = len(pairs) / (3.0 * mp.nbundles)
        line["smem_load_tbs"] = smem_tbs
        line["smem_frac_of_nominal"] = smem_tbs / (148 * 128 * 1.965e9 / 1e12)
    return line


# ----------------------------------------------------------------------------- B200 arm
def run_b200(args, rank, world, local_rank):
    import torch

    import matvis_b200 as mv
    from matvis_b200 import _lib
    from matvis_b200 import workloads as wl
    from matvis_b200.engine import VisEngine, job_from_arrays

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist

    cfg, desc = load_config(args)
    fluxes, rot_kw, sim_kw = cfg["fluxes"], {}, {}
    if args.sky == "pol":
        fluxes = wl.polarised_sky(cfg)
        desc += "; polarised sky (seeded Q, U, V; coherency fluxes)"
    if args.rotation == "erfa":
        time_s = 600.0 * np.arange(len(cfg["lsts"]))
        rot_kw = dict(astrom=wl.synthetic_astrom(cfg["lsts"], cfg["latitude"]), time_s=time_s, update_bcrs_every=0.0)
        sim_kw = dict(coord_method="CoordinateRotationERFA", coord_method_params=rot_kw)
        desc += "; ERFA apparent-place rotation from seeded astrometry parameters, refreshed every time step"
    if args.sky != "stokes" or args.rotation != "lst":
        args.skip_cpu = args.skip_plain = True  # the samplers restate the Stokes-I, LST-rotation path
    terms, counts = terms_per_job(cfg, rot_kw.get("astrom"))
    matprod = "VectorDot" if args.sparse or args.pairs != "all" else "MatMul"
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=fluxes, ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True, precision=1, gemm_mode=args.gemm_mode, k_chunk=args.k_chunk,
                           antpairs=cfg["antpairs"], matprod=matprod, pair_product=args.pair_kernel, **rot_kw)
    eng = VisEngine(spec, device=dev)
    eng.upload()
    eng.run()  # uncaptured run: checks status, warms caches
    eng.capture()
    stream = torch.cuda.current_stream()

    for _ in range(max(args.warmup, 0)):
        eng.run(check=False)
    torch.cuda.synchronize()
    _lib.check_status_word(eng.status, "warm-up")

    def barrier():
        if dist is not None:
            dist.barrier()

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            eng.run(check=False)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    clocks = clk.summary()
    _lib.check_status_word(eng.status, "timed run")
    ms = ev0.elapsed_time(ev1) / max(args.steps, 1)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * terms / (ms_max / 1000.0)

    # ---- roofline of the dominant kernel, timed on its own stream over the last slice's panel
    roofline = vecdot_roofline(eng, dev) if eng.method == "VectorDot" else herk_roofline(eng, args, dev)

    panel = eng.zcalc.z
    kvalid = int(eng.n_above.item()) * eng.nax
    if eng.method == "VectorDot":
        dtype, kc = "f32", eng.matprod.k_chunk
        if eng.matprod.kernel == "staged":
            product = ("complex64 Z staged in shared memory, FP32 per-pair sums per 16-column stage "
                       "(mvb_vecdot_staged), FP64 k-slice and slice sums")
        else:
            product = "complex64 Z, FP32 per-pair sums (mvb_vecdot), FP64 warp and slice sums"
    else:
        dtype = {"fp16x3": "fp16", "bf16x6": "bf16", "bf16x3": "bf16", "tf32x3": "tf32"}[args.gemm_mode]
        kc = eng.k_chunk
        product = (GEMM_PRECISION[args.gemm_mode] + " tcgen05 Hermitian product, FP32 register sums per drained "
                   "TMEM block, FP64 slice sums")
    sky = ("HEALPix nside=%d centres, lognormal flux" % args.nside if args.config == 2
           else "isotropic sources, power-law flux")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype,
        "data": f"synthetic (seeded; {sky}, HERA-350-like array, dipole-like beams)",
        "config": workload_config(args, cfg, desc, terms, counts),
        "implementation": {
            "pair_kernel": eng.pair_kernel if eng.method != "VectorDot" else f"vecdot ({eng.matprod.kernel})",
            "gemm_mode": None if eng.method == "VectorDot" else args.gemm_mode, "k_chunk": kc,
            "z_panel": "%.2f GB per slice" % (panel.data.numel() * panel.data.element_size() / 1e9 * kvalid /
                                              panel.Kcap),
            "parallelism": "replicas (one job per GPU)" if world > 1 else "1 GPU",
            "precision": "FP64 rotation/horizon/phase reduction, FP32 sincos and Z, " + product,
            "freq_group": eng.fgroup,
            "autotune": eng.tuned,
        },
        "roofline": roofline,
        "gpu_launches": eng.launches_per_run() * args.steps,
        "clocks": clocks,
    }

    slices = accuracy_slices(cfg)
    full_sky = len(cfg["ra"]) <= 196_608  # the oracle runs on the timed job's own sky
    ovis = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        # three (f, t) slices: about 10 s of FP64 work on the host cores (all sources of
        # config 2, a 196,608-source seeded subset of the larger skies)
        v, dt, sample, ovis = oracle_slices(cfg, slices, None if full_sky else 196_608)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample,
                                "seconds": dt}
        if full_sky and cfg.get("antpairs") is None and args.sky == "stokes" and args.rotation == "lst":
            from oracle.oracle import cosine_error_metric

            errs = [cosine_error_metric(eng.vis[f, t].cpu().numpy(), ref, 2) for (f, t), ref in zip(slices, ovis)]
            line["accuracy"] = {
                "max_norm_err": max(errs), "per_slice": errs, "slices": slices, "bar": 1e-6,
                "of": "the timed job's own visibilities (the last graph replay) at these (f, t) slices",
                "metric": "max over outputs of |V - V_oracle| / sqrt(|V_ii| |V_jj|), against the FP64 oracle on "
                          "all sources, antennas and pairs",
            }
    if rank == 0 and not args.skip_plain:
        try:
            extra = [((f + 7) % len(cfg["freqs"]), (t + 5) % len(cfg["lsts"])) for f, t in slices]
            pg, pvis = plain_gpu_sample(cfg, slices + extra)
            line["plain_gpu"] = pg
            line["vs_plain_gpu"] = value / world / pg["value"]
            if ovis is not None and "accuracy" in line:
                from oracle.oracle import cosine_error_metric

                perr = [cosine_error_metric(v, ref, 2) for v, ref in zip(pvis, ovis)]
                pg["max_norm_err"] = max(perr)
                pg["per_slice_err"] = perr
                line["accuracy"]["plain_gpu_max_norm_err"] = max(perr)
        except Exception as exc:  # the denominator is informative only
            line["plain_gpu"] = {"error": repr(exc)[:200]}

    if not args.skip_e2e:
        ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
        kw = dict(polarized=True, precision=1, beam_idx=cfg["beam_idx"], gemm_mode=args.gemm_mode,
                  k_chunk=args.k_chunk, device=dev, antpairs=cfg["antpairs"], matprod_method=matprod,
                  pair_product=args.pair_kernel)
        mv.simulate_vis(ants, fluxes, cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], cfg["beams"],
                        cfg["latitude"], **kw, **sim_kw)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nb_out = 0
        for _ in range(args.e2e_steps):
            out = mv.simulate_vis(ants, fluxes, cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], cfg["beams"],
                                  cfg["latitude"], **kw, **sim_kw)
            nb_out = out.nbytes
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / args.e2e_steps
        e_t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if dist is not None:
            dist.all_reduce(e_t, op=dist.ReduceOp.MAX)
        h2d = eng.h2d_bytes() + sum(b.data.nbytes for b in cfg["beams"]) + eng.antpos_host.nbytes
        line["e2e"] = {"value": world * terms / float(e_t.item()), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(nb_out), "seconds_per_step": float(e_t.item()),
                       "api": "matvis_b200.simulate_vis (host numpy in/out)", "steps": args.e2e_steps}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_beamfits(args, local_rank):
    """simulate_vis end to end with a beamfits beam (config 2's first grid beam at
    100 and 200 MHz, the second scaled by 0.9, written and read back)."""
    import torch

    import matvis_b200 as mv
    from matvis_b200.beamfits import BeamFits, read_beamfits, write_beamfits

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cfg, desc = load_config(args)
    g = cfg["beams"][0]
    data = np.stack([g.data[..., :-1], 0.9 * g.data[..., :-1]], axis=2).astype(np.complex128)  # az without 360 deg
    bf = BeamFits("efield", data, np.asarray(g.az)[:-1], np.asarray(g.za), np.array([100e6, 200e6]), ["x", "y"], [],
                  "linear")
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "beam.fits"
        write_beamfits(path, bf)
        beams = [read_beamfits(path)]
    terms, counts = terms_per_job(cfg)
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    kw = dict(polarized=True, precision=1, gemm_mode=args.gemm_mode, k_chunk=args.k_chunk, device=dev)
    for _ in range(max(args.warmup, 1)):
        mv.simulate_vis(ants, cfg["fluxes"], cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], beams, cfg["latitude"],
                        **kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = mv.simulate_vis(ants, cfg["fluxes"], cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], beams,
                              cfg["latitude"], **kw)
    torch.cuda.synchronize()
    sec = (time.perf_counter() - t0) / max(args.steps, 1)
    line = {
        "metric": METRIC, "impl": "b200", "unit": UNIT, "value": terms / sec, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * sec, "higher_is_better": True,
        "note": "end to end through simulate_vis (host arrays in and out): a chromatic beamfits beam runs one job "
                "per frequency",
        "config": {"workload": desc + "; one beamfits beam for all antennas (100 and 200 MHz, linear in frequency)",
                   "gemm_mode": args.gemm_mode, "terms_per_job": terms},
        "e2e": {"value": terms / sec, "unit": UNIT, "d2h_bytes_per_step": int(out.nbytes), "seconds_per_step": sec},
    }
    print(json.dumps(line), flush=True)


def run_serve(args, local_rank):
    """Served form (config 5): Poisson arrivals into the continuous-batching server.
    The stream is generated lazily (each job's sky is built when it arrives) and
    only latencies and term counts are kept, so host memory stays bounded."""
    import torch

    from matvis_b200 import devcache
    from matvis_b200 import workloads as wl
    from matvis_b200.serve import VisServer, latency_summary

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)

    def stream():
        for t, spec in wl.config5_stream(njobs=args.serve_jobs, rate_hz=args.serve_rate,
                                         nsrc_max=args.serve_nsrc_max):
            spec.gemm_mode = args.gemm_mode
            arrivals[0] = t
            yield t, spec

    arrivals = [0.0]
    _, first = next(wl.config5_stream(njobs=1, rate_hz=args.serve_rate, nsrc_max=args.serve_nsrc_max))
    first.gemm_mode = args.gemm_mode
    small = args.serve_small_terms or None
    ahead = args.serve_turns_ahead or None
    tt = args.serve_turn_terms or None
    warm = VisServer(device=dev, max_active=args.serve_max_active, keep_results=False, small_job_terms=small,
                     turns_ahead=ahead, turn_terms=tt)
    warm.serve_stream([(0.0, first)])  # kernel warm-up, not timed
    warm.close()
    budget = int(args.serve_hbm_frac * torch.cuda.mem_get_info(dev)[0])
    srv = VisServer(device=dev, hbm_budget=budget, max_active=args.serve_max_active, keep_results=False,
                    small_job_terms=small, turns_ahead=ahead, turn_terms=tt)
    hits0, miss0 = devcache.CACHE.hits, devcache.CACHE.misses
    t0 = time.perf_counter()
    srv.serve_stream(stream())
    wall = time.perf_counter() - t0
    srv.close()
    summ = latency_summary(srv.results)
    line = {
        "metric": "served form: job latency p50/p99 and throughput", "impl": "b200", "unit": UNIT,
        "throughput": summ["terms"] / wall, "p50_s": summ["p50_s"], "p99_s": summ["p99_s"],
        "mean_queue_s": summ["mean_queue_s"], "jobs": summ["jobs"], "errors": summ["errors"], "wall_s": wall,
        "arrival_span_s": arrivals[0], "max_concurrent": srv.max_concurrent, "peak_hbm_gb": srv.peak_in_use / 1e9,
        "launches_per_job": srv.launches / max(summ["jobs"] + summ.get("errors", 0), 1),
        "device_cache": {"hits": devcache.CACHE.hits - hits0, "misses": devcache.CACHE.misses - miss0},
        "allocator": {k: torch.cuda.memory_stats(dev).get(k) for k in ("num_alloc_retries", "num_device_alloc",
                                                                      "num_device_free")},
        "alloc_conf": os.environ.get("PYTORCH_CUDA_ALLOC_CONF"),
        "admission_oom_retries": srv.oom_retries,
        "config": {"workload": f"config5 stream: {args.serve_jobs} jobs, Poisson {args.serve_rate}/s, Nant log-U[16,512], "
                               f"Nsrc log-U[1e3,{args.serve_nsrc_max}], Nf U{{1..32}}, Nt U{{1..16}}, Gaussian or "
                               f"polarised grid beam", "gemm_mode": args.gemm_mode,
                   "max_active": args.serve_max_active, "small_job_terms": small, "turns_ahead": ahead,
                   "turn_terms": tt, "hbm_budget_gb": budget / 1e9,
                   "cuda_device_max_connections": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS")},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.serve:
        # one hardware work queue per active job's stream (set before CUDA starts)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
        run_serve(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    if args.beam == "fits":
        run_beamfits(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
