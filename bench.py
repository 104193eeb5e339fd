"""Benchmark: effective-field evaluations per second at 1024 x 1024 x 16 cells.

Workload (one "step" = one H_eff evaluation of the full mesh): 1024 x 1024 x 16
cells of 3 nm, Ms = 8.6e5 A/m, terms demag (open boundaries, zero-padded FFT
convolution) + exchange (A = 1.3e-11 J/m) + cubic anisotropy (K1 = -1e4 J/m^3,
lab axes) + a uniform Zeeman field drawn from a 50 mT ball; m uniform random on
the unit sphere.  Inputs are synthetic and seeded.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value      FP32-field form, H_eff evals/s with m resident in HBM (the field pipeline
           alone), summed over all ranks (independent replicas, "weak" scaling).
e2e        the same metric through the public C ABI with host buffers: every step
           copies m (FP32; FP64 in fp64_m_value) host->device from pinned memory
           and H (FP32) back.
fp64_form  the FP64 form on the same mesh; rel_err_fp32_vs_fp64 checks the metric's
           condition (FP32-field error <= 1e-5 relative to the FP64 form), also per
           field term and for the component of H perpendicular to m.
trajectory 5 ps of DP45 with dense output of <m> in both forms: simulated ns per
           hour and the largest <m> difference between the forms.
configs    simulated ns per hour of short runs of the strip (100x25x1) and skyrmion
           film (512x512x4) configurations.
roofline   the dominant pass: algorithmic bytes per launch / its mean CUDA-event
           duration, against the measured HBM copy bandwidth.
rel_err_vs_oracle  both forms' fields on the full mesh against the FP64 oracle (fed the
           device's tensor), whose threaded evaluation on all host cores is also timed
           as cpu_baseline.
kernels    every kernel of the field path (both forms, and the local terms alone):
           algorithmic bytes / CUDA-event time against the measured HBM peak.
rk_step    DP45 in both forms: one attempt timed kernel by kernel, and a plain
           step loop (steps/s, simulated ns per hour).
--impl reference  the FP64 CPU oracle (the reference algorithm restated in NumPy/SciPy,
           threaded) on all host cores; each step is one H_eff of the full mesh.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "magnum.af_b200", "python"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Heff evals/s at 1024²×16; FP32-field vs FP64 form, rel. err ≤1e-5 vs FP64"
NX, NY, NZ = 1024, 1024, 16  # the metric's mesh (--mesh overrides it for small profiling runs)
DX = 3e-9
MS = 8.6e5
A_EX = 1.3e-11
K1 = -1.0e4
TRAJ_T = 5e-12  # simulated time of the reported trajectory
SEED = 1234
MU0 = 4e-7 * math.pi


def workload(seed=SEED, nz=None):
    nz = NZ if nz is None else nz
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(NX, NY, nz, 3))
    m /= np.linalg.norm(m, axis=3, keepdims=True)
    # uniform in a 50 mT ball
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    r = 0.05 * rng.uniform() ** (1.0 / 3.0)
    h_ext = v * r / MU0
    return np.asfortranarray(m), h_ext


# algorithmic bytes per pass at the metric's mesh: the five-pass padded-FFT model
# (r = 4 B FP32 / 8 B FP64, c = 2r, nxh = nx+1, Py = 2 ny, tensor stored on the
# (nx+1)(ny+1)(nz+1) quadrant with 6 components)
def pass_bytes(r, nx=None, ny=None, nz=None):
    nx, ny, nz = (NX if nx is None else nx), (NY if ny is None else ny), (NZ if nz is None else nz)
    c = 2 * r
    N = nx * ny * nz
    nxh = nx + 1
    Py = 2 * ny
    T = 6 * nxh * (ny + 1) * (nz + 1) * r
    return {
        "x_fwd": 3 * N * r + 3 * nxh * ny * nz * c,
        "y_fwd": 3 * nxh * ny * nz * c + 3 * nxh * Py * nz * c,
        "z_conv": 3 * nxh * Py * nz * c + T + 3 * nxh * Py * nz * c,
        "y_inv": 3 * nxh * Py * nz * c + 3 * nxh * ny * nz * c,
        "x_inv_local": 3 * nxh * ny * nz * c + 3 * N * r + 3 * N * r,
    }


def interval_bytes(name, r, nx=None, ny=None, nz=None):
    """Algorithmic bytes of one interval of a Runge-Kutta attempt profile
    (LLGIntegrator.attempt_profile): the field passes (the x inverse with the LLG
    epilogue: spectrum + m for the stencils + the FP64 m of the cross product, k
    written in FP64), the FP32 copy of m, the stage combine m + sum a_j k_j over
    N FP64 k buffers (FP64 staged m written, plus its FP32 copy in the FP32-field
    form) and the finalize (m and N k's read, the candidate written)."""
    nx, ny, nz = (NX if nx is None else nx), (NY if ny is None else ny), (NZ if nz is None else nz)
    N = nx * ny * nz
    pb = pass_bytes(r, nx, ny, nz)
    if name in ("x_fwd", "y_fwd", "z_conv", "y_inv"):
        return pb[name]
    if name == "x_inv_local":  # LLG epilogue
        spec = 3 * (nx + 1) * ny * nz * 2 * r
        return spec + (3 * N * 4 + 3 * N * 8 if r == 4 else 3 * N * 8) + 3 * N * 8
    if name == "stage_m32":
        return 3 * N * 8 + 3 * N * 4
    if name.startswith("rk_combine_k"):
        k = int(name[len("rk_combine_k"):])
        return (k + 1) * 3 * N * 8 + 3 * N * 8 + (3 * N * 4 if r == 4 else 0)
    if name.startswith("rk_finalize_k"):
        k = int(name[len("rk_finalize_k"):])
        return (k + 1) * 3 * N * 8 + 3 * N * 8
    return None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant pass from the committed ncu summary
    (a 512x512x16 capture scaled to the full launch by the tiles processed)."""
    p = os.path.join(ROOT, "profiles", "traffic_1024x1024x16.txt")
    out = {}
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("#") or "=" not in line:
                    continue
                k, v = line.split("=", 1)
                out[k.strip()] = float(v.split()[0])
    except OSError:
        pass
    return out


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", "maf_clocks_%d_%d.csv" % (os.getpid(), gpu_index))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            # nvidia-smi needs a moment before its first sample: wait for it so
            # that the samples cover the timed region that follows
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_state(mesh_args, m_norm):
    """Oracle State over the device-normalised m (identical inputs: the oracle's own
    constructor would normalise once more)."""
    import maf_oracle as O

    om = O.Mesh(*mesh_args)
    st = O.State.__new__(O.State)
    st.mesh, st.m, st.t, st.steps = om, m_norm, 0.0, 0
    st.Ms, st.Ms_field = MS, None
    return om, st


def oracle_terms(O, demag, h_ext):
    return [demag, O.ExchangeField(A_EX), O.CubicAnisotropyField(K1), O.ExternalField(np.asarray(h_ext))]


def time_oracle_heff(terms, state, reps, warmup=0):
    """Seconds per FP64 oracle H_eff (threaded: scipy.fft workers and slabs over all
    host cores); returns (best time, threads, last field)."""
    import maf_oracle_threaded as OT

    threads = os.cpu_count() or 1
    h = None
    for _ in range(warmup):
        h = OT.heff_in_apm(terms, state, threads)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        h = OT.heff_in_apm(terms, state, threads)
        times.append(time.perf_counter() - t0)
    return min(times), threads, h


def run_reference(args):
    """--impl reference: the FP64 CPU oracle (the reference algorithm restated in
    NumPy/SciPy, threaded over all host cores) on the full 1024 x 1024 x 16 mesh,
    rank 0 only.  The oracle assembles its own demag tensor (Newell sums in a
    spawned process pool) before the timed region; each step is one full-mesh
    H_eff evaluation."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import maf_oracle as O

    threads = os.cpu_count() or 1
    O.FFT_WORKERS = threads
    mesh = O.Mesh(NX, NY, NZ, DX, DX, DX)
    m, h_ext = workload()
    state = O.State(mesh, MS, m)
    del m
    t0 = time.perf_counter()
    demag = O.DemagField(mesh, N_real=O.demag_tensor_symmetric(mesh, workers=threads))
    setup_s = time.perf_counter() - t0
    terms = oracle_terms(O, demag, h_ext)
    import maf_oracle_threaded as OT

    for _ in range(args.warmup):
        OT.heff_in_apm(terms, state, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        OT.heff_in_apm(terms, state, threads)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    value = 1.0 / dt
    sample = ("FP64 oracle H_eff (numpy/scipy restatement of the reference path; FFTs with scipy.fft workers and "
              "the tensor product and local terms on slabs, %d threads) of the full %dx%dx%d mesh per step; the "
              "reference's ArrayFire CPU backend is unavailable on this box (no ArrayFire library)" % (
                  threads, NX, NY, NZ))
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "H_eff demag+exchange+cubic+Zeeman, %dx%dx%d cells of 3 nm (FP32-field form)"
                               % (NX, NY, NZ),
                   "cells": NX * NY * NZ, "parallelism": "replicas x1",
                   "l2": "inputs larger than L2 (m 201 MB, spectra 403-806 MB per pass)",
                   "same_config": True, "tensor_setup_s": setup_s},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def rk_step_figures(M, mesh, m, terms, stream, steps, peak):
    """DP45 on the full mesh in both forms: one Runge-Kutta attempt timed kernel by
    kernel (CUDA events, mean of 3 attempts at the step size the controller has
    reached), with each kernel's algorithmic bytes / time against the HBM peak, and
    a plain LLGIntegrator.step loop (no dense output): steps/s, attempts and
    simulated ns per hour of wall time."""
    import torch

    out = {}
    for prec in ("fp32_field", "fp64"):
        r = 4 if prec == "fp32_field" else 8
        llg = M.LLGIntegrator(0.01, terms, "DP45")
        st = M.State(mesh, MS, m, precision=prec)
        st.set_stream(stream.cuda_stream)
        llg.steps(st, 3)  # warm-up; grows the first step from hmin
        torch.cuda.synchronize()
        c0 = llg.counters()
        t_sim0 = st.t
        t0 = time.perf_counter()
        llg.steps(st, steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        c1 = llg.counters()
        reps = 3
        agg = {}
        for _ in range(reps):
            for name, ms in llg.attempt_profile(st, llg.h):
                if name in ("start", "attempt"):
                    continue
                a = agg.setdefault(name, [0.0, 0])
                a[0] += ms
                a[1] += 1
        kernels = {}
        attempt_ms = 0.0
        for name, (ms, cnt) in agg.items():
            per_attempt_ms = ms / reps
            attempt_ms += per_attempt_ms
            b = interval_bytes(name, r)
            gbs = b * cnt / (ms * 1e-3) / 1e9 if b else None
            kernels[name] = {"launches_per_attempt": cnt // reps, "ms_per_attempt": per_attempt_ms,
                             "gbs": gbs, "frac": gbs / peak if gbs else None}
        rk_only = sum(v["ms_per_attempt"] for k, v in kernels.items() if k.startswith("rk_") or k == "stage_m32")
        out[prec] = {
            "steps": steps, "attempts": int((c1["accepted"] + c1["rejected"]) - (c0["accepted"] + c0["rejected"])),
            "wall_s": wall, "steps_per_s": steps / wall,
            "sim_ns_per_hour": (st.t - t_sim0) * 1e9 / wall * 3600.0, "sim_s": st.t - t_sim0,
            "attempt_ms_profiled": attempt_ms, "rk_kernels_share": rk_only / attempt_ms if attempt_ms else None,
            "kernels": kernels,
        }
        del st, llg
    out["scheme"] = "DP45, alpha 0.01, default controller (atol = rtol = 1e-6), from the random initial m"
    return out


def heun_ensemble(M, steps, fused_only=False, shapes=None):
    """The batched Langevin ensemble: 64 stochastic-Heun members at T = 300 K on
    2-D meshes whose two sides are drawn (seeded) from {64, 96, 128, 192, 256, 384,
    512} cells of 2 x 2 x 1 nm; demag + exchange (1.6e-11 J/m) + interface DMI
    (3e-3 J/m^2) + uniaxial Ku 1e6 J/m^3 along z, Ms 1.1e6 A/m, alpha 0.1, dt 5 fs,
    FP32 field / FP64 state, each member with its own noise stream.  Timed on the
    host around StochasticBatch.steps (each call synchronises): the batched passes
    (one launch per pass for all members, one CUDA graph per two steps), the
    per-member graph on forked streams, and (a few steps) the members stepped one
    after another."""
    import torch

    rng = np.random.default_rng(SEED + 7)
    sides = [64, 96, 128, 192, 256, 384, 512]
    if shapes is None:
        shapes = [(int(rng.choice(sides)), int(rng.choice(sides))) for _ in range(64)]

    def build():
        out = []
        for i, (nx, ny) in enumerate(shapes):
            mesh = M.Mesh(nx, ny, 1, 2e-9, 2e-9, 1e-9)
            terms = [M.DemagField(mesh), M.ExchangeField(1.6e-11), M.DmiField(3e-3), M.UniaxialAnisotropyField(1e6)]
            m = np.zeros((nx, ny, 1, 3))
            m[..., 2] = 1.0
            st = M.State(mesh, 1.1e6, m, precision="fp32_field")
            it = M.Stochastic_LLG(0.1, 300.0, 5e-15, st, terms, "Heun", seed=SEED, member=i)
            out.append((it, st, terms))
        return out

    def run(batch, n):
        batch.steps(3)  # the eager step, then a capture
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batch.steps(n)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    cells = sum(nx * ny for nx, ny in shapes)
    res = {"members": len(shapes), "cells": cells, "steps": steps,
           "config": "%d stochastic-Heun members, sides %s (2-D), T 300 K, FP32 field / FP64 state" % (
               len(shapes), "from {64..512}" if len(set(shapes)) > 1 else "%dx%d" % shapes[0])}
    mem = build()
    fb = M.StochasticBatch([(it, st) for it, st, _ in mem], fused=True)
    t = run(fb, steps)
    res["fused"] = {"active": fb.fused_active, "s": t, "ensemble_steps_per_s": steps / t,
                    "member_steps_per_s": len(shapes) * steps / t, "cell_steps_per_s": cells * steps / t}
    del fb, mem
    if not fused_only:
        mem = build()
        gb = M.StochasticBatch([(it, st) for it, st, _ in mem], fused=False)
        t = run(gb, steps)
        res["graph_of_streams"] = {"s": t, "ensemble_steps_per_s": steps / t}
        del gb
        nser = max(2, min(steps, 20))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for it, st, _ in mem:
            it.steps(st, nser)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        res["one_after_another"] = {"s": t, "steps": nser, "ensemble_steps_per_s": nser / t}
        res["fused_speedup_vs_serial"] = res["fused"]["ensemble_steps_per_s"] / res["one_after_another"][
            "ensemble_steps_per_s"]
        res["fused_speedup_vs_streams"] = res["fused"]["ensemble_steps_per_s"] / res["graph_of_streams"][
            "ensemble_steps_per_s"]
        del mem
    return res


def other_configs(M, stream, film_steps=10000):
    """Simulated ns per hour of wall time on the two other single-mesh
    configurations (short runs, seeded inputs):
    strip   100x25x1 cells of 5x5x3 nm, demag + exchange, Ms 8e5, A 1.3e-11,
            m = x + U(-0.1, 0.1)^3 renormalised, alpha 1, DP45 (atol = rtol = 1e-6),
            <m> sampled every 10 ps for 0.2 ns (FP64 form, the configuration's);
    film    512x512x4 cells of 2x2x1 nm, demag + exchange (1.6e-11) + interface DMI
            (3e-3) + uniaxial Ku 1e6 along z, Ms 1.1e6, alpha 0.1, m = +z with 20
            reversed discs of radius 5-15 cells, RKF45, film_steps steps in both forms (10^4, the
            configuration's run length, by default)."""
    import torch

    rng = np.random.default_rng(SEED + 1)
    out = {}
    mesh = M.Mesh(100, 25, 1, 5e-9, 5e-9, 3e-9)
    m = np.zeros((100, 25, 1, 3))
    m[..., 0] = 1.0
    m += rng.uniform(-0.1, 0.1, size=m.shape)
    st = M.State(mesh, 8e5, m)
    st.set_stream(stream.cuda_stream)
    llg = M.LLGIntegrator(1.0, [M.DemagField(mesh), M.ExchangeField(1.3e-11)], "DP45", atol=1e-6, rtol=1e-6)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    llg.integrate_dense(st, 2e-10, 1e-11)
    wall = time.perf_counter() - t0
    out["strip_100x25x1"] = {"sim_ns_per_hour": 0.2 / wall * 3600.0, "steps": st.steps, "wall_s": wall,
                             "form": "fp64"}
    del st, llg
    n, nz = 512, 4
    mesh = M.Mesh(n, n, nz, 2e-9, 2e-9, 1e-9)
    m = np.zeros((n, n, nz, 3))
    m[..., 2] = 1.0
    yy, xx = np.meshgrid(np.arange(n), np.arange(n))
    for _ in range(20):
        r = rng.integers(5, 16)
        cx, cy = rng.uniform(0, n, size=2)
        m[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r, :, 2] = -1.0
    terms = [M.DemagField(mesh), M.ExchangeField(1.6e-11), M.DmiField(3e-3), M.UniaxialAnisotropyField(1e6)]
    llg = M.LLGIntegrator(0.1, terms, "RKF45")
    for prec in ("fp32_field", "fp64"):
        st = M.State(mesh, 1.1e6, m, precision=prec)
        st.set_stream(stream.cuda_stream)
        llg.steps(st, 5)  # warm-up
        torch.cuda.synchronize()
        t_start = st.t
        t0 = time.perf_counter()
        llg.steps(st, film_steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out["film_512x512x4_" + prec] = {"sim_ns_per_hour": (st.t - t_start) * 1e9 / wall * 3600.0,
                                         "steps": film_steps, "steps_per_s": film_steps / wall,
                                         "sim_s": st.t - t_start}
        del st
    return out


def kernel_sweep(args):
    """--kernel-sweep: a few launches of every kernel family of the path on the
    --mesh mesh, for profiler captures (nothing is timed or printed but a
    summary line): the field passes in both forms, the local terms alone, one
    DP45 attempt per form (combine, finalize, FP32 copy of m), two Heun steps of
    a 2-D film and a few LBFGS iterations (its vector kernels and energy
    partials) on a 128 x 128 film."""
    import torch

    import magnumaf as M

    mesh = M.Mesh(NX, NY, NZ, DX, DX, DX)
    m, h_ext = workload()
    terms = [M.DemagField(mesh), M.ExchangeField(A_EX), M.CubicAnisotropyField(K1), M.ExternalField.uniform(*h_ext)]
    llg = M.LLGIntegrator(0.01, terms, "DP45")
    loc = M.LLGIntegrator(0.01, terms[1:], "DP45")
    for prec in ("fp32_field", "fp64"):
        st = M.State(mesh, MS, m, precision=prec)
        llg.H_in_Apm_f32(st) if prec == "fp32_field" else llg.H_in_Apm(st)
        loc.H_in_Apm_f32(st) if prec == "fp32_field" else loc.H_in_Apm(st)
        llg.attempt_profile(st, 1e-14)
        del st
    film = M.Mesh(256, 256, 1, 2e-9, 2e-9, 1e-9)
    fst = M.State(film, 1.1e6, np.broadcast_to(np.array([0.0, 0.0, 1.0]), (256, 256, 1, 3)).copy(),
                  precision="fp32_field")
    heun = M.Stochastic_LLG(0.1, 300.0, 5e-15, fst, [M.DemagField(film), M.ExchangeField(1.6e-11),
                                                        M.UniaxialAnisotropyField(1e6)], "Heun", seed=1)
    heun.steps(fst, 2)
    small = M.Mesh(128, 128, 1, 2e-9, 2e-9, 2e-9)
    rng = np.random.default_rng(5)
    ms = rng.normal(size=(128, 128, 1, 3))
    sst = M.State(small, 8e5, ms / np.linalg.norm(ms, axis=3, keepdims=True))
    mini = M.LBFGS_Minimizer([M.ExchangeField(1.3e-11), M.DmiField(3e-3), M.UniaxialAnisotropyField(8e5)], tol=1e-6,
                             maxiter=5)
    mini.minimize(sst)
    torch.cuda.synchronize()
    print(json.dumps({"kernel_sweep": "%dx%dx%d" % (NX, NY, NZ)}), flush=True)


def run_ours(args):
    import ctypes as C

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import magnumaf as M

    lib = M.lib
    dev = torch.device("cuda", local)
    mesh = M.Mesh(NX, NY, NZ, DX, DX, DX)
    m, h_ext = workload(seed=SEED + rank)
    stream = torch.cuda.Stream(device=dev)
    demag = M.DemagField(mesh)
    terms = [demag, M.ExchangeField(A_EX), M.CubicAnisotropyField(K1), M.ExternalField.uniform(*h_ext)]
    llg = M.LLGIntegrator(0.01, terms, "DP45")
    s32 = M.State(mesh, MS, m, precision="fp32_field")
    s64 = M.State(mesh, MS, m, precision="fp64")
    s32.set_stream(stream.cuda_stream)
    s64.set_stream(stream.cuda_stream)
    n3 = 3 * NX * NY * NZ
    m_norm = np.asarray(s64.m, order="F").ravel(order="F")  # normalised m, [3][nz][ny][nx]
    m64_dev = torch.from_numpy(m_norm).to(dev)
    m32_dev = m64_dev.float()
    H32 = torch.empty(n3, dtype=torch.float32, device=dev)
    H64 = torch.empty(n3, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fn()
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        with torch.cuda.stream(stream):
            for _ in range(steps):
                fn()
        ev1.record(stream)
        ev1.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        if dist:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    tune = None
    if not args.no_autotune:  # kernel variants per pass, measured on this mesh (FP32-field form)
        tune = llg.autotune_ex(s32, reps=3)

    f32 = lambda: llg.heff_device(s32, m32_dev.data_ptr(), H32.data_ptr())
    f64 = lambda: llg.heff_device(s64, m64_dev.data_ptr(), H64.data_ptr())

    clk = ClockSampler(local)
    clk.start()
    ms32 = timed(f32, args.steps, args.warmup)
    ms64 = timed(f64, args.steps, args.warmup)
    clocks = clk.stop()

    # accuracy of the FP32-field form against the FP64 form on the full mesh
    f32()
    f64()
    torch.cuda.synchronize()
    d = (H32.double() - H64)
    rel_err = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(H64))
    rel_max = float(d.abs().max() / H64.abs().max())

    # the same error per field term (each term alone), and for the torque-relevant
    # component of H perpendicular to m (the exchange self term, parallel to m,
    # inflates |H| but exerts no torque)
    per_term = {}
    m3 = m64_dev.view(3, -1)
    for name, term in zip(("demag", "exchange", "cubic", "zeeman"), terms):
        one = M.LLGIntegrator(0.01, [term], "DP45")
        with torch.cuda.stream(stream):
            one.heff_device(s32, m32_dev.data_ptr(), H32.data_ptr())
            one.heff_device(s64, m64_dev.data_ptr(), H64.data_ptr())
        torch.cuda.synchronize()
        h32, h64 = H32.double().view(3, -1), H64.view(3, -1)
        p32 = h32 - (h32 * m3).sum(0, keepdim=True) * m3
        p64 = h64 - (h64 * m3).sum(0, keepdim=True) * m3
        nrm = float(torch.linalg.vector_norm(h64))
        per_term[name] = {
            "l2": float(torch.linalg.vector_norm(h32 - h64)) / nrm if nrm else 0.0,
            "torque_l2": float(torch.linalg.vector_norm(p32 - p64) / torch.linalg.vector_norm(p64)),
        }
        del one

    # a short trajectory in both forms: DP45 with dense output of <m> (RKF45
    # back-steps), simulated ns per hour of wall time and the largest <m>
    # difference between the forms over the samples
    traj = {}
    if not args.no_trajectory:
        rows = {}
        for prec in ("fp32_field", "fp64"):
            st = M.State(mesh, MS, m, precision=prec)
            st.set_stream(stream.cuda_stream)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rows[prec] = llg.integrate_dense(st, TRAJ_T, TRAJ_T / 10)
            wall = time.perf_counter() - t0
            traj[prec] = {"sim_ns_per_hour": TRAJ_T * 1e9 / wall * 3600.0, "wall_s": wall, "steps": st.steps}
            del st
        n_rows = min(len(rows["fp32_field"]), len(rows["fp64"]))
        traj["mean_m_max_abs_diff"] = float(np.abs(rows["fp32_field"][:n_rows, 1:]
                                                   - rows["fp64"][:n_rows, 1:]).max())
        traj["t_sim_s"] = TRAJ_T
        traj["scheme"] = "DP45 (alpha 0.01, default controller), <m> sampled every %g s" % (TRAJ_T / 10)

    # the other single-mesh configurations, short runs: simulated ns per hour
    cfgs = {} if args.no_trajectory else other_configs(M, stream, args.film_steps)
    if not args.no_trajectory and args.heun_steps > 0:
        cfgs["heun_ensemble_64"] = heun_ensemble(M, args.heun_steps)
        # the same with 64 small members (64 x 64): launch-bound, where one launch per pass pays
        cfgs["heun_ensemble_64_small"] = heun_ensemble(M, args.heun_steps, shapes=[(64, 64)] * 64)
    if not args.no_trajectory and args.warm_start_samples > 0:
        # the learned warm start: plain against warm-started LBFGS on fresh samples of the
        # 128 x 128 configuration with the pretrained U-net (seeds never used in training)
        from magnumaf import warmstart as WS

        ws = WS.gain(WS.pretrained_unet(), args.warm_start_samples, 128, 128, seed=30_000)
        ws["config"] = ("128x128x1 cells of 2 nm, exchange + interface DMI + uniaxial + z field, parameters uniform "
                        "per sample, initial m random on the sphere per cell; LBFGS tol 1e-6, maxiter 2000")
        cfgs["warm_start_128"] = ws

    # per-pass timing (CUDA events between the pass kernels on the launching stream)
    passes = {}
    nprof = max(3, min(args.steps, 10))
    for _ in range(nprof):
        for name, ms in llg.heff_device_profile(s32, m32_dev.data_ptr(), H32.data_ptr()):
            passes.setdefault(name, []).append(ms)
    pass_ms = {k: float(np.mean(v)) for k, v in passes.items()}
    passes64 = {}
    for _ in range(nprof):
        for name, ms in llg.heff_device_profile(s64, m64_dev.data_ptr(), H64.data_ptr()):
            passes64.setdefault(name, []).append(ms)
    pass_ms64 = {k: float(np.mean(v)) for k, v in passes64.items()}
    # the local terms alone (exchange, cubic, Zeeman: the k_local_epi kernel, no demag)
    loc = M.LLGIntegrator(0.01, terms[1:], "DP45")
    loc_ms = {}
    for prec_name, st_, mp_, hp_ in (("fp32_field", s32, m32_dev, H32), ("fp64", s64, m64_dev, H64)):
        v = []
        for _ in range(nprof):
            v += [ms for _, ms in loc.heff_device_profile(st_, mp_.data_ptr(), hp_.data_ptr())]
        loc_ms[prec_name] = float(np.mean(v))
    del loc
    bytes32 = pass_bytes(4)
    dominant = max(pass_ms, key=pass_ms.get)
    peak, peak_kind = peaks()
    achieved = bytes32[dominant] / (pass_ms[dominant] * 1e-3) / 1e9
    traffic = ncu_traffic().get(dominant)
    eval_bytes = sum(bytes32.values())
    eval_gbs = eval_bytes / (ms32 / args.steps * 1e-3) / 1e9
    # every kernel of the field path: algorithmic bytes / CUDA-event time against the peak
    bytes64 = pass_bytes(8)
    N = NX * NY * NZ
    kernels = {}
    for form, pm, by, r in (("fp32_field", pass_ms, bytes32, 4), ("fp64", pass_ms64, bytes64, 8)):
        for name, ms in pm.items():
            gbs = by[name] / (ms * 1e-3) / 1e9
            kernels["%s/%s" % (form, name)] = {"ms": ms, "bytes": by[name], "gbs": gbs, "frac": gbs / peak}
        lb = 2 * 3 * N * r  # m read, H written (neighbours from cache)
        gbs = lb / (loc_ms[form] * 1e-3) / 1e9
        kernels["%s/local_terms" % form] = {"ms": loc_ms[form], "bytes": lb, "gbs": gbs, "frac": gbs / peak}

    # the time step: DP45 attempt split by kernel, and a plain step loop in both forms
    rk = None
    if not args.no_trajectory and args.rk_steps > 0:
        rk = rk_step_figures(M, mesh, m, terms, stream, args.rk_steps, peak)

    # end to end through the C ABI with pinned host buffers
    m_host = torch.from_numpy(m_norm.copy()).pin_memory()
    H_host = torch.empty(n3, dtype=torch.float32).pin_memory()
    mp = C.cast(C.c_void_p(m_host.data_ptr()), C.POINTER(C.c_double))
    hp = C.cast(C.c_void_p(H_host.data_ptr()), C.POINTER(C.c_float))

    def e2e_step():
        M._ck(lib.maf_state_set_m(s32._h, mp))
        M._ck(lib.maf_llg_heff_f32(llg._h, s32._h, hp))

    e2e_steps = max(1, min(args.steps, 20))
    ms_e2e_serial = timed(e2e_step, e2e_steps, max(1, min(args.warmup, 3)))

    # the same through the pipelined call: every step still copies its m in from
    # pinned memory and its H out, overlapped with the neighbouring evaluations.
    # The headline e2e passes m in FP32 (the field form's input precision; the
    # reference's f32 State path), the FP64-input figure is reported beside it.
    H_bufs = [H_host, torch.empty(n3, dtype=torch.float32).pin_memory()]
    m_bufs64 = [m_host, torch.from_numpy(m_norm.copy()).pin_memory()]
    m_bufs32 = [torch.from_numpy(m_norm.astype(np.float32)).pin_memory() for _ in range(2)]

    def pipe(n, f32_in):
        bufs = m_bufs32 if f32_in else m_bufs64
        llg.heff_pipeline(s32, [bufs[i % 2].data_ptr() for i in range(n)],
                          [H_bufs[i % 2].data_ptr() for i in range(n)], m_float32=f32_in)

    def timed_pipe(f32_in):
        pipe(2, f32_in)  # allocates the double buffers
        barrier()
        t0 = time.perf_counter()
        pipe(e2e_steps, f32_in)
        ms = (time.perf_counter() - t0) * 1e3
        if dist:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    ms_e2e = timed_pipe(True)
    ms_e2e64 = timed_pipe(False)

    npass = len(pass_ms)
    value = world * args.steps / (ms32 * 1e-3)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms32 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded random m on the unit sphere, random 50 mT-ball Zeeman field)",
        "config": {"workload": "H_eff demag+exchange+cubic+Zeeman, %dx%dx%d cells of 3 nm (FP32-field form)"
                               % (NX, NY, NZ),
                   "cells": NX * NY * NZ, "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2 (m 201 MB, spectra 403-806 MB per pass)",
                   "tune": None if tune is None else {k: tune[k] for k in ("cols_wide", "convz_reg", "xinv_run",
                                                                          "cols_pipe", "cols_plan")}},
        "fp64_form": {"value": world * args.steps / (ms64 * 1e-3), "ms_per_step": ms64 / args.steps,
                      "fp32_speedup": ms64 / ms32},
        "rel_err_fp32_vs_fp64": {"l2": rel_err, "max": rel_max, "per_term": per_term},
        "trajectory": traj,
        "configs": cfgs,
        "passes_ms": pass_ms,
        "passes_ms_fp64": pass_ms64,
        "kernels": kernels,
        "rk_step": rk,
        "eval_roofline": {"bytes": eval_bytes, "achieved_gbs": eval_gbs, "frac": eval_gbs / peak},
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_source": "profiles/traffic_1024x1024x16.txt: ncu dram bytes of a 512x512x16 launch "
                                       "of the same kernel, scaled by the tiles processed (not measured in this run)",
                     "algorithmic_bytes": bytes32[dominant]},
        "e2e": {"value": world * e2e_steps / (ms_e2e * 1e-3), "unit": "evals/s", "h2d_bytes_per_step": n3 * 4,
                "d2h_bytes_per_step": n3 * 4,
                "path": "LLGIntegrator.heff_pipeline(m_float32=True) over pinned host buffers (copies overlapped)",
                "fp64_m_value": world * e2e_steps / (ms_e2e64 * 1e-3), "fp64_m_h2d_bytes_per_step": n3 * 8,
                "serial_value": world * e2e_steps / (ms_e2e_serial * 1e-3)},
        "gpu_launches": npass * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # The FP64 oracle on the full mesh, on all host cores: its time is the CPU
        # baseline, its field the parity check of both forms at the metric's size.
        # The oracle is fed the device's tensor (identical inputs: independently
        # assembled Newell sums differ at their rounding noise, ~1e-5 at this size);
        # tensor assembly is outside the timed region either way.
        import maf_oracle as O

        O.FFT_WORKERS = os.cpu_count() or 1
        with torch.cuda.stream(stream):
            f32()
            f64()
        torch.cuda.synchronize()
        to_xyz = lambda flat: flat.reshape(3, NZ, NY, NX).transpose(3, 2, 1, 0)
        h64 = to_xyz(H64.cpu().numpy())
        h32 = to_xyz(H32.cpu().numpy().astype(np.float64))
        om, ost = oracle_state((NX, NY, NZ, DX, DX, DX), np.ascontiguousarray(to_xyz(m_norm)))
        od = O.DemagField(om, N_real=demag.get_N(symmetric=True))
        t, threads, href = time_oracle_heff(oracle_terms(O, od, h_ext), ost, reps=2)
        del od
        nref, mref = float(np.linalg.norm(href)), float(np.abs(href).max())

        def errs(h):
            dd = h - href
            return {"l2": float(np.linalg.norm(dd)) / nref, "max": float(np.abs(dd).max()) / mref}

        line["rel_err_vs_oracle"] = {
            "mesh": "%dx%dx%d (the metric's mesh)" % (NX, NY, NZ), "tensor": "device tensor fed to the oracle",
            "fp64": errs(h64), "fp32_field": errs(h32), "tolerance": {"fp64": 1e-12, "fp32_field": 1e-5}}
        line["cpu_baseline"] = {
            "value": 1.0 / t, "unit": "evals/s", "cores": threads, "kind": "port",
            "sample": "FP64 oracle H_eff of the full %dx%dx%d mesh (numpy/scipy restatement of the reference path, "
                      "FFTs with scipy.fft workers, tensor product and local terms on slabs; %d threads), best of 2; "
                      "the reference's ArrayFire CPU backend is unavailable on this box" % (NX, NY, NZ, threads)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del s32, s64
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--no-trajectory", action="store_true", help="skip the short DP45 trajectory")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default kernel variants")
    ap.add_argument("--rk-steps", type=int, default=1000, help="DP45 steps of the plain step loop per form")
    ap.add_argument("--film-steps", type=int, default=10000, help="RKF45 steps of the 512x512x4 film per form")
    ap.add_argument("--heun-steps", type=int, default=1000, help="steps of the 64-member Heun ensemble")
    ap.add_argument("--warm-start-samples", type=int, default=16, help="held-out samples of the warm-start gain")
    ap.add_argument("--kernel-sweep", action="store_true",
                    help="launch every kernel family once or twice (for profiler captures) and exit")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="time only the batched 64-member Heun ensemble (--heun-steps steps; for profiler captures)")
    ap.add_argument("--mesh", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="smaller mesh for profiling captures (the reported metric is defined at 1024 1024 16)")
    args = ap.parse_args()
    if args.mesh:
        global NX, NY, NZ
        NX, NY, NZ = args.mesh
    if args.impl == "reference":
        run_reference(args)
    elif args.kernel_sweep:
        kernel_sweep(args)
    elif args.ensemble_only:
        import magnumaf as M

        print(json.dumps({"heun_ensemble_64": heun_ensemble(M, args.heun_steps, fused_only=True)}), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
