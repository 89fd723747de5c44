#!/usr/bin/env python
"""Benchmark of the B200 on-grid SHT: maps/s at nside 2048, lmax 4096.

Workload (one "step"): spin-2 (E,B) -> (Q,U) synthesis of one seeded a_lm pair and
its VJP through torch.autograd -- loss 0.5 ||S a - d||^2, gradient S^T (S a - d) --
in FP64.  ``value`` is maps/s with inputs resident in HBM; ``e2e`` is the same step
through the public API with pinned host buffers copied in and the gradient and
loss copied out every step.  Kernel time is measured live with CUDA events around
each stage launch inside the C ABI (jhtb_plan_set_timing); the FP64 roofline
denominator is measured with the in-library FMA probe.

``mixed`` is the batched mixed-precision form of the same step: B maps per step,
both Legendre stages (the synthesis and the VJP's adjoint) on the tensor cores
(split-BF16 products, FP32 accumulation folded into FP64), the recursion, the ring
transforms and the loss in FP64; it reports maps/s, the ratio to the FP64 maps/s, and
the relative error of every map and gradient against the FP64 path on the same inputs.

``configs`` (secondary lines): spin-0 analysis(niter=3) at nside 1024 / lmax 2048 (FP64
and tensor-core A0 with FP64 residuals, error vs FP64), 64 spin-0 maps S + S^T at
nside 512 / lmax 1024 (FP64 and bf16x3, per-map error), and the 16-RHS masked CG at
nside 512 / lmax 1024 (ms per iteration for both operator precisions).
``offgrid`` (secondary) times the off-grid synthesis_general and its adjoint at lmax 2048 on
10^7 seeded points.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With torchrun (N > 1) every rank transforms its own maps (independent work, no
data-path collective: weak scaling) and the slowest rank's device time counts.
``--impl reference`` times the CPU restatement of jht's algorithm (oracle/,
C + OpenMP recursion, NumPy ring FFTs) on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "maps/s at nside 2048: FP64 plain vs batched mixed-prec, rel err vs FP64"
UNIT = "maps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nside", type=int, default=2048)
    ap.add_argument("--lmax", type=int, default=4096)
    ap.add_argument("--cpu-sample-m", type=int, default=96,
                    help="orders in the CPU-baseline sample (the same sample for cpu_baseline and --impl reference)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mixed-batch", type=int, default=16, help="maps per step of the mixed-precision form (0: skip)")
    ap.add_argument("--mixed-steps", type=int, default=3)
    ap.add_argument("--no-configs", action="store_true", help="skip the analysis and 64-map batch lines")
    ap.add_argument("--cg-iters", type=int, default=100, help="CG iterations timed per precision in the CG line (0: skip)")
    ap.add_argument("--offgrid-points", type=int, default=10_000_000,
                    help="points of the secondary off-grid measurement (0: skip)")
    return ap.parse_args()


# --------------------------------------------------------------------------------------
# seeded synthetic inputs (config: E C_l = 1/(l+10)^2, B 0.1/(l+10)^2, l < 2 zero; d ~ N(0,1))
# --------------------------------------------------------------------------------------
def spectrum_alm(rng, lmax: int, amp: float) -> np.ndarray:
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    cl = amp / (ell + 10.0) ** 2
    g1 = rng.standard_normal(ell.size)
    g2 = rng.standard_normal(ell.size)
    a = np.sqrt(cl / 2.0) * (g1 + 1j * g2)
    a[: lmax + 1] = np.sqrt(cl[: lmax + 1]) * g1[: lmax + 1]
    a[ell < 2] = 0.0
    return a.astype(np.complex128)


def make_inputs(seed: int, nside: int, lmax: int):
    rng = np.random.default_rng(seed)
    alm = np.stack([spectrum_alm(rng, lmax, 1.0), spectrum_alm(rng, lmax, 0.1)])
    d = rng.standard_normal((2, 12 * nside * nside))
    return alm, d


# --------------------------------------------------------------------------------------
# clock sampling during the timed region
# --------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------------------
# CPU baseline: oracle (C + OpenMP log-renormalised recursion, NumPy ring FFTs), sampled
# --------------------------------------------------------------------------------------
def cpu_baseline(nside: int, lmax: int, n_m: int) -> dict:
    from oracle import _cref
    from oracle import jht_oracle as O

    ref = _cref.load()
    geo = O.Rings(nside)
    T = 2 * nside
    x = geo.z[:T]
    K = O.alm_size(lmax)
    rng = np.random.default_rng(0)
    alm = np.stack([spectrum_alm(rng, lmax, 1.0), spectrum_alm(rng, lmax, 0.1)])
    # blocks of consecutive orders (one per core) spread over [0, lmax]: OpenMP runs
    # the block's orders in parallel, as the full transform would
    ncores = os.cpu_count() or 1
    nblk = max(1, n_m // ncores)
    starts = np.unique(np.linspace(0, lmax + 1 - ncores, nblk).astype(int)) if lmax + 1 > ncores else np.array([0])
    ms = np.unique(np.concatenate([np.arange(s0, min(s0 + ncores, lmax + 1)) for s0 in starts]))
    work_sample = float(sum(lmax - m + 1 for m in ms))
    t_leg = 0.0
    V = [np.zeros((lmax + 1, T), np.complex128) for _ in range(4)]
    for s0 in starts:
        s1 = min(s0 + ncores, lmax + 1)
        t0 = time.perf_counter()
        ref.synth(2, lmax, x, alm, int(s0), int(s1))
        ref.adjoint(2, lmax, x, V, int(s0), int(s1))
        t_leg += time.perf_counter() - t0
    leg_full = t_leg * (K / work_sample)
    # ring stage: time the NumPy per-length FFT assembly on a sample of ring lengths
    lengths = np.unique(geo.nring)
    pick = lengths[np.linspace(0, lengths.size - 1, 16).astype(int)]
    mm = np.arange(lmax + 1)
    t_fft = 0.0
    pix_sample = 0
    for N in pick:
        rows = np.flatnonzero(geo.nring == N)
        G = (rng.standard_normal((rows.size, lmax + 1)) + 1j * rng.standard_normal((rows.size, lmax + 1)))
        t0 = time.perf_counter()
        D = np.zeros((rows.size, N), np.complex128)
        np.add.at(D, (slice(None), mm % N), G)
        np.add.at(D, (slice(None), (-mm[1:]) % N), np.conj(G[:, 1:]))
        y = np.fft.ifft(D, axis=1) * N
        W = np.fft.fft(y, axis=1)
        _ = W[:, mm % N]
        t_fft += time.perf_counter() - t0
        pix_sample += rows.size * N
    fft_full = t_fft * (geo.npix / pix_sample) * 2  # two channels (Fp, Fm / Vp, Vm)
    step = leg_full + fft_full
    return {
        "value": 1.0 / step,
        "unit": UNIT,
        "cores": os.cpu_count(),
        "kind": "port",
        "sample": (f"spin-2 synthesis+adjoint recursion/contraction for {ms.size} of {lmax + 1} orders m "
                   f"({t_leg:.1f} s) and the ring DFT stage for {pick.size} ring lengths ({t_fft:.1f} s), "
                   f"extrapolated by work (K={K}, Npix={geo.npix}) to {step:.1f} s per map"),
    }


# --------------------------------------------------------------------------------------
# distributed helpers
# --------------------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_mixed(args, jhtb, _lib, torch, dev, pg, nside, lmax, spin, rank, world, fp64_ms_per_step):
    """Batched mixed-precision step: B maps of synthesis and VJP with both Legendre stages on the tensor cores."""
    B = args.mixed_batch
    alm = np.stack([make_inputs(5000 + 97 * rank + b, nside, lmax)[0] for b in range(B)])
    rng = np.random.default_rng(77 + rank)
    a = torch.as_tensor(alm, device=dev).requires_grad_(True)
    d = torch.as_tensor(rng.standard_normal((B, 2, 12 * nside * nside)), device=dev)

    def step(prec):
        a.grad = None
        m = jhtb.synthesis_batch(a, nside, lmax, spin, precision=prec)
        loss = 0.5 * torch.nn.functional.mse_loss(m, d, reduction="sum")
        loss.backward()
        return m.detach(), a.grad.detach().clone()

    # error of every map and gradient against the FP64 path on the same inputs
    m64, g64 = step("fp64")
    mmx, gmx = step("bf16x3")
    torch.cuda.synchronize()
    den_m = torch.amax(torch.abs(m64).reshape(B, -1), dim=1)
    err_m = torch.amax(torch.abs(mmx - m64).reshape(B, -1), dim=1) / den_m
    den_g = torch.amax(torch.abs(g64).reshape(B, -1), dim=1)
    err_g = torch.amax(torch.abs(gmx - g64).reshape(B, -1), dim=1) / den_g
    del m64, g64, mmx, gmx
    plan = _lib.get_plan(nside, lmax, spin, "bf16x3", B)
    for _ in range(max(1, args.warmup - 1)):
        step("bf16x3")
    torch.cuda.synchronize()
    plan.timings(reset=True)
    if pg:
        pg.barrier()
    plan.set_timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.mixed_steps):
        step("bf16x3")
    e1.record()
    torch.cuda.synchronize()
    plan.set_timing(False)
    dev_ms = e0.elapsed_time(e1)
    stage = plan.timings(reset=True)
    if pg:
        t = torch.tensor([dev_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        dev_ms = float(t.item())
    ms_step = dev_ms / args.mixed_steps
    value = world * B / (ms_step * 1e-3)
    fp64_value = world / (fp64_ms_per_step * 1e-3)
    return {
        "value": value,
        "unit": UNIT,
        "maps_per_step_per_gpu": B,
        "ms_per_step": ms_step,
        "vs_fp64_plain": value / fp64_value,
        "precision": "synthesis and adjoint Legendre stages bf16x3 (tcgen05 split-BF16 products, FP32 block sums "
                     "folded into FP64); recursion, ring FFTs and loss FP64",
        "roofline": _tc_roofline(stage, nside, lmax, spin, B),
        "rel_err_synthesis_vs_fp64": {"max": float(err_m.max()), "per_map": [float(e) for e in err_m]},
        "rel_err_gradient_vs_fp64": {"max": float(err_g.max()), "per_map": [float(e) for e in err_g]},
        "avg_launch_ms": {k: v / max(n, 1) for k, (v, n) in stage.items()},
        "gpu_launches": sum(n for _, n in stage.values()),
    }


def _peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def _tc_roofline(stage: dict, nside: int, lmax: int, spin: int, B: int) -> dict:
    """Tensor-pipe roofline of the mixed step's Legendre kernels: split-BF16 work per launch
    = 6 products x (16 spin 2 / 4 spin 0) contraction flops per (l, m, ring pair) and map,
    over all K x 2 nside triples (the dead polar triples included), against the measured
    sustained cuBLAS bf16 rate (the kernels run inside a seconds-long step)."""
    K = (lmax + 1) * (lmax + 2) // 2
    per = (16.0 if spin else 4.0) * 6.0
    work = per * K * 2 * nside * B
    pk = _peaks()
    peak = pk.get("bf16_tflops_sustained")
    out = {"bound": "tensor", "unit": "TFLOP/s", "peak": peak,
           "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained" if peak else None,
           "flops_per_launch": work}
    for name in ("legendre_synth", "legendre_adjoint"):
        ms, n = stage[name]
        if n:
            a = work / (ms / n * 1e-3) / 1e12
            out[name] = {"achieved": a, "frac": (a / peak) if peak else None, "avg_launch_ms": ms / n}
    return out


def run_configs(jhtb, _lib, torch, dev) -> dict:
    """Secondary lines at the other configurations (device-resident inputs, CUDA events):
    spin-0 analysis(niter=3) at nside 1024 / lmax 2048, FP64 and with tensor-core A0, and
    64 spin-0 maps S + S^T at nside 512 / lmax 1024, FP64 and bf16x3 (per-map error)."""
    out = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ev[0].record()
        for _ in range(reps):
            r = fn()
        ev[1].record()
        torch.cuda.synchronize()
        return r, ev[0].elapsed_time(ev[1]) / reps

    # analysis
    nside, lmax = 1024, 2048
    rng = np.random.default_rng(11)
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)
    cl = 1.0 / (ell + 10.0) ** 2
    a = np.sqrt(cl / 2) * (rng.standard_normal(K) + 1j * rng.standard_normal(K))
    a[: lmax + 1] = np.sqrt(cl[: lmax + 1]) * rng.standard_normal(lmax + 1)
    m = jhtb.synthesis(a, nside, lmax, 0)
    ref, t64 = timed(lambda: jhtb.analysis(m, nside, lmax, 0, niter=3))
    mix, tmx = timed(lambda: jhtb.analysis(m, nside, lmax, 0, niter=3, precision="bf16x3"))
    out["analysis_n1024_l2048"] = {
        "workload": "spin-0 analysis(niter=3, ring weights), nside 1024, lmax 2048, 1 map",
        "fp64_ms": t64, "mixed_ms": tmx, "fp64_maps_per_s": 1e3 / t64, "mixed_maps_per_s": 1e3 / tmx,
        "mixed_rel_err_vs_fp64": float(torch.max(torch.abs(mix - ref)) / torch.max(torch.abs(ref))),
        "fp64_tflops": 7 * 8.0 * K * 2 * nside / (t64 * 1e-3) / 1e12,
    }
    del m, ref, mix
    # batched S + S^T
    nside, lmax, B = 512, 1024, 64
    K = jhtb.alm_size(lmax)
    ell = np.concatenate([np.arange(mm, lmax + 1) for mm in range(lmax + 1)])
    amp = 10.0 ** rng.uniform(-2, 2, size=B)
    ab = (rng.standard_normal((B, K)) + 1j * rng.standard_normal((B, K))) / (ell + 10.0) * amp[:, None]
    ab[:, : lmax + 1] = ab[:, : lmax + 1].real
    at = torch.as_tensor(ab, device=dev)

    def sst(prec):
        mm = jhtb.synthesis_batch(at, nside, lmax, 0, precision=prec)
        return mm, jhtb.adjoint_synthesis_batch(mm, nside, lmax, 0, precision=prec)

    (m64, b64), t64 = timed(lambda: sst("fp64"))
    (mmx, bmx), tmx = timed(lambda: sst("bf16x3"))
    em = torch.amax(torch.abs(mmx - m64), dim=1) / torch.amax(torch.abs(m64), dim=1)
    eb = torch.amax(torch.abs(bmx - b64), dim=1) / torch.amax(torch.abs(b64), dim=1)
    work = 2 * 8.0 * K * 2 * nside * B  # S and S^T, spin 0: 8 flops per triple and map
    pk = _peaks()
    # the same S + S^T pair through the C ABI on the tuned plan, replayed from a captured CUDA
    # graph (the autotuner's timing; eager if capture fails)
    graph_ms, graphed = None, False
    try:
        from jht_b200 import autotune

        gplan = _lib.get_plan(nside, lmax, 0, "bf16x3", B)
        m_out = torch.empty((B, 1, 12 * nside * nside), dtype=torch.float64, device=dev)
        b_out = torch.empty((B, 1, K), dtype=torch.complex128, device=dev)
        graph_ms, graphed = autotune._time(gplan, at.reshape(B, 1, K).contiguous(), mmx.reshape(B, 1, -1).contiguous(),
                                           m_out, b_out, 3)
        del m_out, b_out
    except Exception as e:  # noqa: BLE001 - a secondary figure; the line keeps its eager timing
        graph_ms = f"unavailable: {type(e).__name__}"
    out["batch64_n512_l1024"] = {
        "mixed_graph_ms": graph_ms, "mixed_graph_captured": graphed,
        "workload": "64 spin-0 maps, synthesis + adjoint, nside 512, lmax 1024, amplitudes log-uniform 1e-2..1e2",
        "fp64_ms": t64, "mixed_ms": tmx, "fp64_maps_per_s": B * 1e3 / t64, "mixed_maps_per_s": B * 1e3 / tmx,
        "mixed_vs_fp64": t64 / tmx,
        "rel_err_synthesis_max": float(em.max()), "rel_err_adjoint_max": float(eb.max()),
        "fp64_tflops": work / (t64 * 1e-3) / 1e12,
        "mixed_tensor_tflops": 6 * 4.0 * K * 2 * nside * B * 2 / (tmx * 1e-3) / 1e12,
        "bf16_peak_sustained": pk.get("bf16_tflops_sustained"),
    }
    return out


def cg_problem(jhtb, torch, nside: int = 512, lmax: int = 1024, B: int = 16, seed: int = 16):
    """The masked CG deconvolution workload: spin 0, a |cos theta| < 0.34 cut plus 200 seeded
    1-degree discs, data S a + white noise (sigma 1e-2) for B right-hand sides, and
    eps = 1e-6 of the largest diagonal entry of T S^T (M W) S T^-1 (probed on 16 m = 0 columns)."""
    from jht_b200 import masked as MK

    npix = 12 * nside * nside
    rng = np.random.default_rng(seed)
    geo = jhtb.healpix.RingInfo(nside)
    z = np.repeat(geo.z, geo.npix_ring)
    phi = np.concatenate([geo.phi0[r] + 2 * np.pi * np.arange(n) / n for r, n in enumerate(geo.npix_ring)])
    st = np.sqrt(1 - z * z)
    mask = (np.abs(z) >= 0.34).astype(np.float64)
    cz = rng.uniform(-1, 1, 200)
    cp = rng.uniform(0, 2 * np.pi, 200)
    cs = np.sqrt(1 - cz * cz)
    cos_r = np.cos(np.radians(1.0))
    for k in range(200):
        mask[z * cz[k] + st * cs[k] * np.cos(phi - cp[k]) > cos_r] = 0.0
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    K = jhtb.alm_size(lmax)
    cl = 1.0 / (ell + 10.0) ** 2
    a = np.sqrt(cl / 2) * (rng.standard_normal((B, K)) + 1j * rng.standard_normal((B, K)))
    a[:, : lmax + 1] = np.sqrt(cl[: lmax + 1]) * rng.standard_normal((B, lmax + 1))
    gen = torch.Generator("cuda").manual_seed(seed)
    maps = jhtb.synthesis_batch(a, nside, lmax, 0)
    maps = maps + 1e-2 * torch.randn(maps.shape, dtype=torch.float64, device="cuda", generator=gen)
    w = MK._weight_pix(nside, npix, maps.device, mask=mask)
    probe = torch.zeros((16, MK.n_dof(lmax, 0)), dtype=torch.float64, device="cuda")
    cols = torch.as_tensor(np.linspace(0, lmax, 16).astype(np.int64), device="cuda")
    probe[torch.arange(16, device="cuda"), cols] = 1.0
    diag = MK._normal(probe, w, nside, lmax, 0, "fp64")[torch.arange(16, device="cuda"), cols]
    return maps, mask, 1e-6 * float(diag.max())


def run_cg(jhtb, torch, iters: int) -> dict:
    """Secondary line: the 16-RHS masked CG at nside 512 / lmax 1024, a bounded number of
    iterations per precision (the solve to relative residual 1e-8 takes thousands of
    iterations at eps = 1e-6 and runs in the GPU test suite); ms per iteration, the
    residual reached, and the per-iteration operator work S + S^T on 16 maps."""
    nside, lmax, B = 512, 1024, 16
    maps, mask, eps = cg_problem(jhtb, torch, nside, lmax, B)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {"workload": f"masked CG (|cos theta| < 0.34 cut + 200 discs of 1 deg), spin 0, nside {nside}, "
                       f"lmax {lmax}, {B} right-hand sides, eps = 1e-6 of the largest diagonal; "
                       f"{iters} iterations timed per precision", "eps": eps}
    for prec in ("fp64", "bf16x3"):
        jhtb.deconvolve_batch(maps, mask, nside, lmax, 0, tol=1e-8, reg=eps, max_iter=2, precision=prec)
        torch.cuda.synchronize()
        ev[0].record()
        _, info = jhtb.deconvolve_batch(maps, mask, nside, lmax, 0, tol=1e-8, reg=eps, max_iter=iters,
                                        return_info=True, precision=prec)
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        out[prec] = {"ms": ms, "iterations": info["iterations"], "ms_per_iteration": ms / max(info["iterations"], 1),
                     "rel_residual_max": float(info["rel_residual"].max()),
                     "fp64_residual_replacements": info.get("outer", 0)}
    out["mixed_vs_fp64_per_iteration"] = out["fp64"]["ms_per_iteration"] / out["bf16x3"]["ms_per_iteration"]
    return out


def run_offgrid(jhtb, torch, dev, npts: int, lmax: int = 2048, spin: int = 2, reps: int = 3) -> dict:
    """Secondary line: off-grid synthesis_general and its adjoint (spin 2, lmax 2048) at
    seeded uniform points, device-resident, CUDA-event timed."""
    rng = np.random.default_rng(2024)
    K = jhtb.alm_size(lmax)
    ell = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    a = (rng.standard_normal((2, K)) + 1j * rng.standard_normal((2, K))) / (ell + 10.0)
    a[:, : lmax + 1] = a[:, : lmax + 1].real
    a[:, ell < 2] = 0
    a = torch.as_tensor(a, device=dev)
    loc = torch.as_tensor(np.stack([np.arccos(rng.uniform(-1, 1, npts)), rng.uniform(0, 2 * np.pi, npts)], 1),
                          device=dev)
    v = torch.as_tensor(rng.standard_normal((2, npts)), device=dev)
    for _ in range(2):
        jhtb.synthesis_general(a, loc, spin=spin, lmax=lmax)
        jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record()
    for _ in range(reps):
        jhtb.synthesis_general(a, loc, spin=spin, lmax=lmax)
    ev[1].record()
    for _ in range(reps):
        jhtb.adjoint_synthesis_general(v, loc, spin=spin, lmax=lmax)
    ev[2].record()
    torch.cuda.synchronize()
    ts, ta = ev[0].elapsed_time(ev[1]) / reps, ev[1].elapsed_time(ev[2]) / reps
    return {"workload": f"spin-2 synthesis_general / adjoint_synthesis_general, lmax {lmax}, {npts} points "
                        "uniform on the sphere, epsilon 1e-10 (W = 14)",
            "synthesis_ms": ts, "adjoint_ms": ta, "synthesis_mpts_per_s": npts / ts / 1e3,
            "adjoint_mpts_per_s": npts / ta / 1e3}


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)

    if args.impl == "reference":
        if rank != 0:
            return
        t_total = time.perf_counter()
        vals = []
        for _ in range(args.steps):
            b = cpu_baseline(args.nside, args.lmax, args.cpu_sample_m)
            vals.append(b["value"])
        v = statistics.median(vals)
        line = {
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"spin-2 synthesis + VJP, nside {args.nside}, lmax {args.lmax}, FP64, 1 map/step",
                       "nside": args.nside, "lmax": args.lmax, "spin": 2},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": b["cores"], "kind": "port", "sample": b["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t_total,
        }
        print(json.dumps(line))
        return

    import torch

    import jht_b200 as jhtb
    from jht_b200 import _lib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
        pg = dist

    nside, lmax, spin = args.nside, args.lmax, 2
    K = jhtb.alm_size(lmax)
    npix = 12 * nside * nside
    alm_np, d_np = make_inputs(1234 + rank, nside, lmax)

    # ---- FP64 peak probe -------------------------------------------------------------
    lib = _lib.load_library()
    sink = torch.zeros(1, dtype=torch.float64, device=dev)
    best = 0.0
    import ctypes

    for _ in range(3):
        ms = ctypes.c_double()
        fl = ctypes.c_double()
        _lib.check(lib.jhtb_probe_fp64_fma(4, 2000, ctypes.c_void_p(sink.data_ptr()), ctypes.byref(ms),
                                           ctypes.byref(fl), _lib.stream_ptr()), "probe")
        best = max(best, fl.value / (ms.value * 1e-3) / 1e12)
    fp64_peak = best

    # ---- device-resident step --------------------------------------------------------
    a = torch.as_tensor(alm_np, device=dev).requires_grad_(True)
    d = torch.as_tensor(d_np, device=dev)

    def step():
        a.grad = None
        m = jhtb.synthesis(a, nside, lmax, spin)
        loss = 0.5 * torch.nn.functional.mse_loss(m, d, reduction="sum")
        loss.backward()
        return loss

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    plan = _lib.get_plan(nside, lmax, spin, "fp64", 1)
    plan.timings(reset=True)
    if pg:
        pg.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.synchronize()
    plan.set_timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    plan.set_timing(False)
    clocks = sampler.stop()
    dev_ms = e0.elapsed_time(e1)
    stage = plan.timings(reset=True)
    if pg:
        t = torch.tensor([dev_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        dev_ms = float(t.item())
        pg.barrier()
    ms_per_step = dev_ms / args.steps
    value = world * 1.0 / (ms_per_step * 1e-3)

    # ---- end-to-end through the public API with pinned host buffers -------------------
    # Every step copies its inputs in from pinned host memory and its gradient and loss
    # out; the copies run on their own stream, double-buffered, so step i+1's inputs
    # travel while step i computes and step i's gradient travels back during step i+1.
    a_host = torch.as_tensor(alm_np).pin_memory()
    d_host = torch.as_tensor(d_np).pin_memory()
    g_host = [torch.empty_like(a_host).pin_memory() for _ in range(2)]
    loss_host = [torch.empty((), dtype=torch.float64).pin_memory() for _ in range(2)]
    comp = torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(device=dev)
    bufs = [(torch.empty(a_host.shape, dtype=a_host.dtype, device=dev),
             torch.empty(d_host.shape, dtype=d_host.dtype, device=dev)) for _ in range(2)]
    h2d_done = [torch.cuda.Event() for _ in range(2)]
    comp_done = [torch.cuda.Event() for _ in range(2)]
    out_done = [None, None]

    def issue_h2d(i):
        k = i % 2
        with torch.cuda.stream(copy):
            if out_done[k] is not None:
                copy.wait_event(out_done[k])  # step i-2 is done with buffer k
            bufs[k][0].copy_(a_host, non_blocking=True)
            bufs[k][1].copy_(d_host, non_blocking=True)
            h2d_done[k].record(copy)

    def e2e_step(i):
        k = i % 2
        comp.wait_event(h2d_done[k])
        ad = bufs[k][0].detach().requires_grad_(True)
        m = jhtb.synthesis(ad, nside, lmax, spin)
        loss = 0.5 * torch.nn.functional.mse_loss(m, bufs[k][1], reduction="sum")
        loss.backward()
        grad, lo = ad.grad, loss.detach()
        comp_done[k].record(comp)
        with torch.cuda.stream(copy):
            copy.wait_event(comp_done[k])
            g_host[k].copy_(grad, non_blocking=True)
            loss_host[k].copy_(lo, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
            out_done[k] = ev
        grad.record_stream(copy)
        lo.record_stream(copy)

    def e2e_run(nsteps, start_event=None):
        if start_event is not None:
            copy.wait_event(start_event)
        issue_h2d(0)
        for i in range(nsteps):
            if i + 1 < nsteps:
                issue_h2d(i + 1)
            e2e_step(i)
        for ev in out_done:
            if ev is not None:
                comp.wait_event(ev)

    e2e_run(max(1, args.warmup // 2))
    torch.cuda.synchronize()
    out_done[0] = out_done[1] = None
    if pg:
        pg.barrier()
    e0.record(comp)
    e2e_run(args.steps, start_event=e0)
    e1.record(comp)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if pg:
        t = torch.tensor([e2e_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * args.steps / (e2e_ms * 1e-3)
    h2d = a_host.numel() * 16 + d_host.numel() * 8
    d2h = g_host[0].numel() * 16 + 8

    # ---- roofline of the dominant kernel (fused recursion + contraction) --------------
    T = 2 * nside
    flops_per_launch = 24.0 * K * T  # spin 2: 8 recursion + 16 contraction flops per (l, m, ring pair)
    leg_s_ms, leg_s_n = stage["legendre_synth"]
    leg_a_ms, leg_a_n = stage["legendre_adjoint"]
    avg_s = leg_s_ms / max(leg_s_n, 1)
    avg_a = leg_a_ms / max(leg_a_n, 1)
    achieved = flops_per_launch / (avg_a * 1e-3) / 1e12  # the adjoint is the longest launch
    traffic = None
    prof = ROOT / "profiles" / "legendre_adjoint2_n2048_l4096.md"
    if prof.exists():
        mt = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", prof.read_text())
        if mt:
            traffic = float(mt.group(1))

    # ---- batched mixed precision: both Legendre stages on the tensor cores ------------------
    mixed = None
    if args.mixed_batch > 0:
        mixed = run_mixed(args, jhtb, _lib, torch, dev, pg, nside, lmax, spin, rank, world, ms_per_step)

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    offgrid = run_offgrid(jhtb, torch, dev, args.offgrid_points) if args.offgrid_points > 0 else None
    configs = run_configs(jhtb, _lib, torch, dev) if not args.no_configs else None
    if configs is not None and args.cg_iters > 0:
        configs["cg16_n512_l1024"] = run_cg(jhtb, torch, args.cg_iters)

    cpu = None
    if not args.no_cpu_baseline:
        cpu = cpu_baseline(nside, lmax, args.cpu_sample_m)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded alm with C_l = 1/(l+10)^2 (E), 0.1/(l+10)^2 (B), l<2 zero; d ~ N(0,1)",
        "config": {
            "workload": f"spin-2 synthesis + VJP (torch.autograd), nside {nside}, lmax {lmax}, FP64 plain, "
                        "1 (Q,U) map per GPU per step",
            "nside": nside, "lmax": lmax, "spin": spin, "precision": "fp64", "maps_per_step_per_gpu": 1,
            "l2": "inputs larger than L2 (alm 268 MB, maps 805 MB)",
            "parallelism": f"independent maps per GPU x{world}",
        },
        "roofline": {
            "kernel": "legendre_adjoint (adj2_kernel: spin 2, FP64 fused recursion + ring contraction)",
            "bound": "fp64",
            "achieved": achieved,
            "peak": fp64_peak,
            "unit": "TFLOP/s",
            "frac": achieved / fp64_peak,
            "peak_source": "measured in this run: jhtb_probe_fp64_fma (FP64 FMA, 2 flop/FMA); "
                           "MEASURED_PEAKS.json holds no FP64 figure",
            "flops_per_launch": flops_per_launch,
            "traffic": traffic,
            "avg_launch_ms": {"legendre_synth": avg_s, "legendre_adjoint": avg_a,
                              "ring_synth": stage["ring_synth"][0] / max(stage["ring_synth"][1], 1),
                              "ring_adjoint": stage["ring_adjoint"][0] / max(stage["ring_adjoint"][1], 1)},
            "synthesis_frac": flops_per_launch / (avg_s * 1e-3) / 1e12 / fp64_peak,
        },
        "mixed": mixed,
        "offgrid": offgrid,
        "configs": configs,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": sum(n for _, n in stage.values()),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
