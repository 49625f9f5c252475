"""Benchmark of the batched mixed-precision stochastic-Hamiltonian propagator.

Workload (one "step" = one time step of every trajectory of the batch):
cylindrical tube 60 x 500 = 30,000 sites, point-dipole couplings within 25 A
(~28 per row), static disorder 150 cm^-1, OU noise 250 cm^-1 / 50 fs,
dt = 0.5 fs, Lanczos m = 20, 256 trajectories per GPU, complex64 vectors with
FP64 Lanczos scalars and FP64 Padé.  Synthetic, seeded input (the
reference's Hamiltonian file is not distributed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  Multi-GPU: one process per GPU (torchrun);
rank r propagates trajectories [r B, (r+1) B) of one ensemble of N B (Philox
keys by global trajectory index), with no exchange while stepping (weak
scaling); the end-to-end leg ends with one NCCL all-reduce of the observable
sums, the ensemble average every rank then reports.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="tube60x500_B256_m20", around=60, along=500, cutoff=25.0, m=20, B=256, dt=0.5,
                sigma_static=150.0, sigma=250.0, tau=50.0, seed=2024)
METRIC = "traj-steps/s (batched mixed vs plain FP64, pop err<=1e-6); backward/forward time"
# CUDA device of this rank (LOCAL_RANK under torchrun); every context of the run is created on it
DEVICE = 0


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """SM clock and throttle reasons sampled DURING the timed region.

    A thread reads NVML every 5 ms (read-only queries of the device this rank
    runs on, found by its PCI bus id), so even a timed region of tens of
    milliseconds gets samples; `nvidia-smi --query-gpu ... -lms 200` runs beside
    it as a second record for longer regions.  Raw samples go to
    $DQ_CLOCKS_DIR (else the temporary directory); the JSON line carries the
    median, maximum and the reasons seen."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits (nvmlClocksEventReason*)
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.thread = None
        self.samples = []
        d = os.environ.get("DQ_CLOCKS_DIR", tempfile.gettempdir())
        self.path = os.path.join(d, f"clocks_bench_{os.getpid()}.csv")

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self):
        nv, h = self.nv, self.h
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), sm, mx, rs))
            except Exception:
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        import threading
        try:
            self.nv, self.h = self._handle()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
        if self.samples:
            with open(self.path.replace(".csv", "_nvml.csv"), "w") as f:
                for t, sm, mx, rs in self.samples:
                    f.write(f"{t:.4f},{sm},{mx},{rs:#x}\n")

    def _smi(self):
        sm, mx, reasons = [], [], set()
        if not self.proc or not os.path.exists(self.path):
            return sm, mx, reasons
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return sm, mx, reasons

    def summary(self):
        if self.samples:
            sm = [x[1] for x in self.samples]
            reasons = sorted(nm for nm, b in self.BITS.items() if any(x[3] & b for x in self.samples))
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(x[2] for x in self.samples),
                    "reasons": reasons, "samples": len(sm), "source": "nvml every 5 ms"}
        sm, mx, reasons = self._smi()
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi every 200 ms"}


def build_system():
    from dynaquant_b200 import systems
    w = WORKLOAD
    return systems.tube(w["around"], w["along"], cutoff=w["cutoff"])


def make_prop(s, B, precision, seed, max_steps, pop_every=16, reorth=0):
    import dynaquant_b200 as dq
    w = WORKLOAD
    p = dq.Propagator(s.n, m=w["m"], n_traj=B, dt=w["dt"], noise=dq.NOISE_OU, sigma_static=w["sigma_static"],
                      seed=seed, dot=dq.DOT_HERMITIAN, precision=precision, pop_every=pop_every,
                      max_steps=max_steps, reorth=reorth, device=DEVICE)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, w["sigma"]), np.full(s.n, w["tau"]))
    p.set_initial_state(s.bright_state())
    return p


def plain_roofline(s, value):
    """HBM roofline of the plain FP64 per-trajectory path: algorithmic bytes per trajectory-step
    48 m N + 16 (m+1) N + 16 N + m (20 (z+1) N + 4 (N+1)) (complex128 vectors, the reference's
    complex128 CSR values re-read by every SpMV) at the measured rate."""
    w = WORKLOAD
    m, n = w["m"], s.n
    z = (s.nnz - s.n) / s.n
    per = 48.0 * m * n + 16.0 * (m + 1) * n + 16.0 * n + m * (20.0 * (z + 1) * n + 4.0 * (n + 1))
    peak, kind = _peaks()
    gbs = value * per / 1e9
    return {"bytes_per_traj_step": per, "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "peak_kind": kind, "note": "about 45 launches per trajectory-step, one trajectory at a time: "
                                       "launch-latency bound, not HBM bound"}


def dominant_kernel(s, B, m, staged, prof):
    """(algorithmic bytes per launch, mean ms per launch, achieved GB/s) of the step's dominant
    kernel under tiling form `staged`, from profile_step's per-kind launch times."""
    ms = prof["spmm_alpha"][0]
    if staged in (2, 4, 8, 11):
        # fused forms: the dominant launch is the whole iteration
        ms = prof["fused_iter"][0]
    b = spmm_bytes(s, B)
    if staged in (0, 5, 9, 10, 11, 12):
        # the L1 forms also read q_{j-1} (8 B per site-trajectory) in m - 1 of the step's m launches
        b += 8.0 * s.n * B * (m - 1) / m
    if staged in (2, 4):
        b += 24.0 * s.n * B   # + r_j, r_{j-1} reads and the r_{j+1} write
    if staged == 11:
        # SpMM launch bytes plus the axpy's (w and q_j read, r_{j+1} written) in the same launch
        b += 24.0 * s.n * B
    if staged == 8:
        # p-form launch j (2 < j <= m): reads p_j, q_{j-1}, q_{j-2} and d, writes q_j and p_{j+1}
        b = 44.0 * s.n * B + 8.0 * (s.nnz - s.n) + 4.0 * (s.n + 1)
    return b, ms, b / (ms / 1e3) / 1e9


def gather_floor_ms(p, reps=20):
    """Device ms of the gathers alone of the context's packed coupling blocks (dq_time_gather_floor), or
    None for a tiling without them."""
    import dynaquant_b200 as dq
    try:
        return p.time_gather_floor(reps)
    except dq.DQError:
        return None


def spmm_bytes(s, B):
    """Algorithmic HBM bytes of one SpMM+alpha launch (complex64 path):
    read q_j (8 B) and the diagonal (4 B), write w (8 B) per site-trajectory,
    plus the shared CSR once (4 B value + 4 B column per coupling, 4 B per row
    pointer)."""
    nnz_off = s.nnz - s.n
    return 20.0 * s.n * B + 8.0 * nnz_off + 4.0 * (s.n + 1)


# SpMM form per tiling `staged` value: kernel name and the committed ncu summary of it
SPMM_FORMS = {0: ("k_spmm_blk (L1 gathers + alpha, minus beta q_{j-1})", None),
              2: ("k_lanczos_fused (r_{j+1} + SpMM + alpha, beta)", None),
              3: ("k_spmm_warp (L1 gathers, warp per block + alpha)", None),
              4: ("k_lanczos_fw (fused, warp-owned blocks)", None),
              5: ("k_spmm_blk, 512-thread CTAs (L1 gathers + alpha, minus beta q_{j-1})",
                  "k_spmm_blk512_tube60x500.md"),
              6: ("k_spmm_ring (TMA ring gathers + alpha)", "k_spmm_ring_tube60x500.md"),
              7: ("k_spmm_ring, 4 trajectories per lane (TMA ring gathers + alpha)", None),
              8: ("k_lanczos_p (one launch per iteration: gathers p_j, writes q_j and p_{j+1}, alpha and beta)",
                  None),
              9: ("k_spmm_cpa (gathers as asynchronous copies into shared memory + alpha, minus beta q_{j-1})",
                  None),
              10: ("k_spmm_wg (warp per row block, eight gathers in flight + alpha, minus beta q_{j-1})", None),
              11: ("k_spmm_wg with the axpy (one cooperative launch per iteration: SpMM + alpha, wait, r_{j+1}, beta)",
                   "k_spmm_wg_tube60x500.md"),
              12: ("k_spmm_lean (L1 gathers at 32 warps per SM, 64 registers + alpha, minus beta q_{j-1})",
                   "k_spmm_lean_tube60x500.md")}


def measured_traffic(staged):
    """DRAM bytes per launch of the chosen SpMM kernel from its committed ncu summary
    (dram__bytes_read.sum + dram__bytes_write.sum of one capture), and the file, or (None, None)."""
    name = SPMM_FORMS.get(staged, (None, None))[1]
    if not name:
        return None, None
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1]), "profiles/" + name
    except OSError:
        pass
    return None, None


def cpu_baseline_sample(s, threads, target_s=12.0):
    """Times the FP64 oracle (C, OpenMP over trajectories) on a bounded
    sample of the same workload; returns traj-steps/s and the sample."""
    from oracle import oracle as O
    O.build()
    w = WORKLOAD
    rp, col, val, diag = s.off_diagonal()
    S = O.System(rp, col, val, diag, m=w["m"], dt=w["dt"], dot_mode=O.DOT_HERMITIAN, noise=O.NOISE_OU,
                 sigma=w["sigma"], tau=w["tau"], sigma_static=w["sigma_static"], seed=w["seed"])
    psi0 = s.bright_state()
    t0 = time.perf_counter()
    S.run(threads, 1, psi0, pop_every=1, threads=threads)
    t1 = time.perf_counter() - t0
    steps = max(1, min(50, int(target_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    S.run(threads, steps, psi0, pop_every=steps, threads=threads)
    dt = time.perf_counter() - t0
    return threads * steps / dt, f"{threads} trajectories x {steps} steps of the same tube workload, FP64 oracle"


def run_reference(args, rank, world):
    """--impl reference: the CPU implementation of the path (the FP64 oracle
    port; the reference itself does not build here) on all host cores."""
    if rank != 0:
        return
    s = build_system()
    threads = os.cpu_count() or 1
    from oracle import oracle as O
    O.build()
    w = WORKLOAD
    rp, col, val, diag = s.off_diagonal()
    S = O.System(rp, col, val, diag, m=w["m"], dt=w["dt"], dot_mode=O.DOT_HERMITIAN, noise=O.NOISE_OU,
                 sigma=w["sigma"], tau=w["tau"], sigma_static=w["sigma_static"], seed=w["seed"])
    psi0 = s.bright_state()
    per_step = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        S.run(threads, 1, psi0, pop_every=1, traj0=k * threads, threads=threads)
        if k >= args.warmup:
            per_step.append(time.perf_counter() - t0)
    tot = sum(per_step)
    value = threads * len(per_step) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "traj-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(per_step),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded tube generator)",
        "config": {"workload": w["name"], "n_sites": s.n, "m": w["m"], "trajectories_per_step": threads,
                   "note": "each step = one time step of `threads` trajectories, FP64 oracle on host cores"},
        "cpu_baseline": {"value": value, "unit": "traj-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{threads} trajectories x 1 step per timed step"},
        "e2e": {"value": value, "unit": "traj-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


AGG = dict(name="tubes60xL_8aggregates_B512_adaptive_m8-32", around=60, Ls=(34, 68, 135, 270, 405, 540, 810, 1000),
           B=(240, 120, 64, 32, 24, 16, 8, 8), m=32, m_min=8, m_tol=1e-7, dt=0.5, steps=2000)


def zz_leg(s, tiling):
    """The ZZ real-noise model (the reference's own example uses it) on the bench tube: 253 oscillators
    of a synthetic Ohmic spectral density on the reference's frequency grid (dOmega = 8.1357 cm^-1,
    T = 77 K) standing in for its spectral-density file; 256 trajectories, mixed precision, the bench's
    tiling; device time of 48 graph-captured steps (three 16-step noise blocks)."""
    import torch
    import dynaquant_b200 as dq
    w = WORKLOAD
    B, K = 256, 48
    p = dq.Propagator(s.n, m=w["m"], n_traj=B, dt=w["dt"], noise=dq.NOISE_ZZ, sigma_static=w["sigma_static"],
                      seed=w["seed"], dot=dq.DOT_HERMITIAN, precision=dq.PREC_MIXED, pop_every=16,
                      max_steps=K + 32, device=DEVICE)
    p.set_system(s)
    om = 8.1357 * np.arange(1, 254)
    p.set_zz_spectral_density(om, 60.0 * (om / 120.0) * np.exp(-om / 120.0), 8.1357, 77.0)
    p.set_initial_state(s.bright_state())
    p.set_tiling(tiling["traj_chunk"], tiling["vec"], tiling["ctas_per_sm"], tiling["rows_per_block"],
                 tiling["staged"], tiling["groups"])
    p.reset()
    p.run(16)
    st = torch.cuda.ExternalStream(p.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    p.run(K)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    p.close()
    return {"workload": "tube60x500_B256_m20_ZZ253", "value": B / (ms / 1e3), "unit": "traj-steps/s",
            "ms_per_step": ms, "note": "noise sums computed 16 steps at a time; synthetic Ohmic density"}


def large_leg():
    """The largest workload: tube 120 x 1000 = 120,000 sites, 40 A cutoff, 1024 trajectories, m = 24,
    dt 0.5 fs, mixed precision, autotuned tiling; device time of 8 graph-captured steps after 2 warm-up
    steps (parity with the FP64 path at this size is a GPU test)."""
    import torch
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    w = WORKLOAD
    s = systems.tube(120, 1000, cutoff=40.0)
    B, K, W = 1024, 8, 2
    p = dq.Propagator(s.n, m=24, n_traj=B, dt=w["dt"], noise=dq.NOISE_OU, sigma_static=w["sigma_static"],
                      seed=w["seed"], dot=dq.DOT_HERMITIAN, precision=dq.PREC_MIXED, pop_every=16,
                      max_steps=W + K + 4, device=DEVICE)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, w["sigma"]), np.full(s.n, w["tau"]))
    p.set_initial_state(s.bright_state())
    tiling = p.autotune()
    p.reset()
    p.run(W)
    st = torch.cuda.ExternalStream(p.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    p.run(K)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    prof = p.profile_step(1)
    gather_floor = gather_floor_ms(p)
    p.close()
    # with chunk groups each launch covers B / groups trajectories
    b, kms, achieved = dominant_kernel(s, B // tiling.get("groups", 1), 24, tiling["staged"], prof)
    peak, peak_kind = _peaks()
    return {"workload": "tube120x1000_B1024_m24", "n_sites": s.n, "nnz_per_row": (s.nnz - s.n) / s.n,
            "value": B / (ms / 1e3), "unit": "traj-steps/s", "ms_per_step": ms,
            "tiling": {k: tiling[k] for k in ("traj_chunk", "vec", "ctas_per_sm", "rows_per_block", "staged", "groups")},
            "roofline": {"bound": "hbm", "kernel": SPMM_FORMS.get(tiling["staged"], ("SpMM + alpha",))[0],
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": b, "ms_per_launch": kms,
                         "gather_floor_ms": gather_floor,
                         "frac_of_gather_floor": (gather_floor / kms) if gather_floor else None},
            "kernels_ms_per_launch": {k: v[0] for k, v in prof.items()}}


def aggregates_leg():
    """Eight tubes 60 x L with 512 trajectories split about as 1/L (multiples of 8), adaptive Krylov
    dimension 8..32 at tolerance 1e-7, dt 0.5 fs, 2000 steps: every member's tiling from the project's
    autotuner (cached per GPU model and size class), then all aggregates in one graph per step
    (dq_group_run_timed: device time of the step launches, capture excluded) against the same aggregates
    run one after another (dq_run each, device time on each member's stream)."""
    import torch
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    a = AGG
    w = WORKLOAD

    def members(seed0):
        out = []
        for i, (L, B) in enumerate(zip(a["Ls"], a["B"])):
            s = systems.tube(a["around"], L, cutoff=w["cutoff"])
            p = dq.Propagator(s.n, m=a["m"], n_traj=B, dt=a["dt"], noise=dq.NOISE_OU, sigma_static=w["sigma_static"],
                              seed=seed0 + i, dot=dq.DOT_HERMITIAN, precision=dq.PREC_MIXED, pop_every=50,
                              max_steps=a["steps"] + 8, m_min=a["m_min"], m_tol=a["m_tol"],
                              device=DEVICE)
            p.set_system(s)
            p.set_noise_params(np.full(s.n, w["sigma"]), np.full(s.n, w["tau"]))
            p.set_initial_state(s.bright_state())
            out.append(p)
        return out

    ms = members(500)
    tilings = []
    for p in ms:
        t = p.autotune()
        tilings.append({k: t[k] for k in ("traj_chunk", "vec", "ctas_per_sm", "rows_per_block", "staged", "groups")})
    g = dq.Group(ms)
    g.run(4)                       # warm-up (allocation, first capture)
    for p in ms:
        p.reset()
    torch.cuda.synchronize()
    t_group = g.run_timed(a["steps"]) / 1e3
    g.close()
    for p in ms:
        p.reset()
    torch.cuda.synchronize()
    t_seq = 0.0
    for p in ms:
        st = torch.cuda.ExternalStream(p.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        p.run(a["steps"])
        e1.record(st)
        torch.cuda.synchronize()
        t_seq += e0.elapsed_time(e1) / 1e3
    n_sites = [p.n for p in ms]
    for p in ms:
        p.close()
    total = sum(a["B"]) * a["steps"]
    return {"workload": a["name"], "sites": n_sites, "trajectories": list(a["B"]), "steps": a["steps"],
            "value": total / t_group, "unit": "traj-steps/s", "sequential_value": total / t_seq,
            "group_over_sequential": t_seq / t_group, "tilings": tilings,
            "note": "device time (CUDA events) of the group's step launches, graph capture excluded, against the "
                    "sum of the eight dq_run device times; tilings from the autotuner per member"}


ADJ = dict(name="lattice64x64_B128_T2000_m16", L=64, J_nn=-250.0, J_nnn=40.0, B=128, dt=1.0, steps=2000, m=16,
           checkpoint_every=50, fft_len=4096, sigma=200.0, tau=100.0, eps_sigma=100.0, target_shift=30.0, seed=77)


def adjoint_leg():
    """Spectrum-loss gradient on the 64x64 lattice (4096 site energies + 2 coupling scales, 128
    trajectories, 2000 steps, checkpoints every 50): backward/forward time ratio in mixed precision,
    and the FP64 gradient against central finite differences on a few parameters."""
    import torch
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    a = ADJ
    lat = systems.lattice2d(a["L"], J_nn=a["J_nn"], J_nnn=a["J_nnn"], seed=0)
    n, T, L = lat.n, a["steps"], a["fft_len"]
    eps = np.random.default_rng(0).normal(0.0, a["eps_sigma"], n)
    eps_t = eps + np.random.default_rng(1).normal(0.0, a["target_shift"], n)

    def make(prec, e, scales=(1.0, 1.0)):
        p = dq.Propagator(n, m=a["m"], n_traj=a["B"], dt=a["dt"], noise=dq.NOISE_OU, seed=a["seed"],
                          dot=dq.DOT_HERMITIAN, precision=prec, max_steps=T, device=DEVICE)
        p.set_system(lat)
        p.set_coupling_classes(lat.cls_off, list(scales))
        p.set_noise_params(np.full(n, a["sigma"]), np.full(n, a["tau"]))
        p.set_static_energies(e)
        p.set_initial_state(lat.bright_state((1.0, 0.0, 0.0)))
        return p

    out = {"workload": a["name"], "params": n + 2, "loss": "L2 between scale*Re(IDFT_4096(Cbar)) and the same "
           "spectrum from site energies shifted by N(0, 30 cm^-1)"}
    for prec, tag in ((dq.PREC_MIXED, "mixed"), (dq.PREC_FP64, "fp64")):
        p = make(prec, eps_t)
        tiling = p.autotune(use_cache=False)
        p.reset()
        p.run(T)
        target = (1.0 / T) * p.spectrum(L).real
        p.close()
        p = make(prec, eps)
        p.set_tiling(tiling["traj_chunk"], tiling["vec"], tiling["ctas_per_sm"], tiling["rows_per_block"],
                     tiling["staged"], tiling["groups"])
        p.adjoint_setup(T, L, 1.0 / T, target, checkpoint_every=a["checkpoint_every"])
        p.forward()
        p.backward()             # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = p.forward()
        t1 = time.perf_counter()
        gs, gc = p.backward()
        t2 = time.perf_counter()
        r = {"forward_s": t1 - t0, "backward_s": t2 - t1, "backward_over_forward": (t2 - t1) / (t1 - t0),
             "loss": loss, "grad_scales": [float(v) for v in gc]}
        if tag == "fp64":
            # central differences, h = 1e-3 cm^-1 on the two largest site gradients, 1e-5 on the scales
            fd = []
            for i in np.argsort(-np.abs(gs))[:2]:
                e1, e2 = eps.copy(), eps.copy()
                e1[i] += 1e-3
                e2[i] -= 1e-3
                p.set_static_energies(e1)
                f1 = p.forward()
                p.set_static_energies(e2)
                f2 = p.forward()
                d = (f1 - f2) / 2e-3
                fd.append({"param": f"eps[{int(i)}]", "adjoint": float(gs[i]), "fd": d,
                           "rel_err": abs(gs[i] - d) / abs(d)})
            p.set_static_energies(eps)
            for q in range(2):
                vals = []
                for sgn in (1, -1):
                    sc = [1.0, 1.0]
                    sc[q] += sgn * 1e-5
                    p.set_coupling_classes(lat.cls_off, sc)
                    vals.append(p.forward())
                d = (vals[0] - vals[1]) / 2e-5
                fd.append({"param": f"scale[{q}]", "adjoint": float(gc[q]), "fd": d, "rel_err": abs(gc[q] - d) / abs(d)})
            r["finite_differences"] = fd
            r["fd_max_rel_err"] = max(f["rel_err"] for f in fd)
        p.close()
        out[tag] = r
    out["note"] = ("host wall clock around dq_forward / dq_backward (each ends in a device sync), after one "
                   "warm-up pair; the backward recomputes every 50-step segment from its checkpoint")
    return out


def secondary_legs(s, B, seed, tiling, value):
    """The N = 1 extras of the JSON line: the plain FP64 path, the population error against the oracle,
    full reorthogonalisation, the adjoint, the aggregates, ZZ noise, the large tube and the CPU baseline."""
    import torch
    import dynaquant_b200 as dq
    w = WORKLOAD
    # ---- plain FP64 per-trajectory GPU path on the same workload ---------------
    pp = make_prop(s, 2, dq.PREC_FP64, seed, max_steps=64)
    plain_steps = 20
    pp.run_plain(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pp.run_plain(plain_steps)
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    pp.close()
    plain = 2 * plain_steps / plain_s
    # ---- population error of the mixed path: vs the FP64 oracle (a short run of a few
    # trajectories) and vs the oracle-pinned batched FP64 path over the configuration's own
    # 4096 steps for all 256 trajectories -------------------------------------------------
    pop_err = {}
    try:
        from oracle import oracle as O
        O.build()
        rp, col, val, diag = s.off_diagonal()
        S = O.System(rp, col, val, diag, m=w["m"], dt=w["dt"], dot_mode=O.DOT_HERMITIAN, noise=O.NOISE_OU,
                     sigma=w["sigma"], tau=w["tau"], sigma_static=w["sigma_static"], seed=seed)
        nT, nS = 4, 64
        ref = S.run(nT, nS, s.bright_state(), pop_every=16, threads=os.cpu_count() or 1)
        pm = make_prop(s, nT, dq.PREC_MIXED, seed, max_steps=nS, pop_every=16)
        pm.run(nS)
        d = np.abs(pm.populations() - ref["pops"]).max()
        pop_err["vs_oracle"] = {"abs": float(d), "rel": float(d / ref["pops"].max()), "trajectories": nT,
                                "steps": nS}
        pm.close()
    except Exception as e:  # pragma: no cover - reported, not hidden
        pop_err["vs_oracle"] = f"unavailable: {e}"
    T_long = 4096
    res = {}
    for prec in (dq.PREC_FP64, dq.PREC_MIXED):
        pl = make_prop(s, B, prec, seed, max_steps=T_long, pop_every=16)
        if prec == dq.PREC_MIXED:
            pl.set_tiling(tiling["traj_chunk"], tiling["vec"], tiling["ctas_per_sm"], tiling["rows_per_block"],
                          tiling["staged"], tiling["groups"])
        else:
            pl.autotune()
        pl.reset()
        pl.run(T_long)
        res[prec] = pl.populations()
        pl.close()
    d_abs = np.abs(res[dq.PREC_MIXED] - res[dq.PREC_FP64]).max(axis=1)
    d_rel = d_abs / res[dq.PREC_FP64].max(axis=1)
    recs = [k for k in (1, 4, 16, 64, 128, 256) if k < len(d_abs)]
    pop_err["vs_fp64_ensemble"] = {
        "abs": float(d_abs.max()), "rel": float(d_rel.max()), "trajectories": B, "steps": T_long,
        "by_step": {str(16 * k): [float(d_abs[k]), float(d_rel[k])] for k in recs},
        "note": "max over sites and records of |p_mixed - p_fp64| (rel: / max p of the record); the batched FP64 "
                "path matches the oracle to 1e-10 (tests)"}
    # ---- the same step with full FP64 reorthogonalisation ------------------------
    # the reorthogonalisation passes favour a different trajectory chunk than the plain iteration, so
    # two tilings are timed (the autotuner times one iteration without them)
    cands = [(32, 2, 1, 3, 5, 1)]
    if tiling["staged"] not in (2, 4, 8):   # the fused forms cannot reorthogonalise between iterations
        cands.insert(0, (tiling["traj_chunk"], tiling["vec"], tiling["ctas_per_sm"], tiling["rows_per_block"],
                         tiling["staged"], tiling["groups"]))
    reorth_runs = []
    for til in cands:
        pr = make_prop(s, B, dq.PREC_MIXED, seed, max_steps=16, reorth=1)
        pr.set_tiling(*til)
        pr.reset()
        pr.run(2)
        rs = torch.cuda.ExternalStream(pr.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(rs)
        pr.run(8)
        e1.record(rs)
        torch.cuda.synchronize()
        reorth_runs.append((e0.elapsed_time(e1) / 8, til))
        pr.close()
    reorth_ms, reorth_til = min(reorth_runs)
    with_reorth = {"value": B / (reorth_ms / 1e3), "unit": "traj-steps/s", "ms_per_step": reorth_ms,
                   "tiling": list(reorth_til), "speedup_over_plain": B / (reorth_ms / 1e3) / plain,
                   "tilings_timed": {",".join(map(str, t)): m for m, t in reorth_runs},
                   "note": "classical Gram-Schmidt against q_1..q_j after every iteration (all h_k in one launch), "
                           "FP64 sums; 8 steps"}
    adjoint = adjoint_leg()
    aggregates = aggregates_leg()
    zz = zz_leg(s, tiling)
    large = large_leg()
    cpu_v, cpu_sample = cpu_baseline_sample(s, os.cpu_count() or 1)
    return {
        "plain_fp64": {"value": plain, "unit": "traj-steps/s", "speedup_batched_mixed": value / plain,
                       "sample": f"2 trajectories x {plain_steps} steps, dq_run_plain",
                       "roofline": plain_roofline(s, plain)},
        "pop_err_vs_fp64_oracle": pop_err,
        "with_reorth": with_reorth,
        "adjoint": adjoint,
        "aggregates": aggregates,
        "zz_noise": zz,
        "large_tube": large,
        "cpu_baseline": {"value": cpu_v, "unit": "traj-steps/s", "cores": os.cpu_count() or 1, "kind": "port",
                         "sample": cpu_sample},
    }


def run_ours(args, rank, world, local_rank):
    import torch
    import dynaquant_b200 as dq
    global DEVICE
    torch.cuda.set_device(local_rank)
    dev = DEVICE = local_rank
    w = WORKLOAD
    B = w["B"]
    s = build_system()
    K, W = args.steps, args.warmup
    seed = w["seed"]
    # ---- device-resident throughput ----------------------------------------
    # rank r runs trajectories [r B, (r+1) B) of one ensemble of world x B (no exchange while stepping)
    p = make_prop(s, B, dq.PREC_MIXED, seed, max_steps=W + K + 8)
    p.set_trajectory_offset(rank * B)
    tiling = p.autotune()
    p.reset()
    p.run(W)
    stream = torch.cuda.ExternalStream(p.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(dev) as clk:
        ev0.record(stream)
        p.run(K)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = B * K * world / (ms / 1e3)
    # ---- per-kernel times (eager, events between kernels) ------------------
    prof = p.profile_step(2)
    gather_floor = gather_floor_ms(p)
    p.close()
    peak, peak_kind = _peaks()
    bytes_spmm, spmm_ms, achieved = dominant_kernel(s, B // tiling.get("groups", 1), w["m"], tiling["staged"], prof)
    step_ms_eager = sum(v[0] * v[1] for v in prof.values()) / 2
    kernels_per_step = sum(v[1] for v in prof.values()) // 2
    # ---- end to end through the C ABI with host buffers --------------------
    # each phase ends in a device synchronisation so the host clock attributes its work
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    marks = []

    def mark(name):
        torch.cuda.synchronize()
        marks.append((name, time.perf_counter()))

    mark("start")
    p2 = dq.Propagator(s.n, m=w["m"], n_traj=B, dt=w["dt"], noise=dq.NOISE_OU, sigma_static=w["sigma_static"],
                       seed=seed, dot=dq.DOT_HERMITIAN, precision=dq.PREC_MIXED, pop_every=16, max_steps=K + 8,
                       device=DEVICE)
    mark("create")
    p2.set_system(s)
    mark("csr_upload")
    p2.set_noise_params(np.full(s.n, w["sigma"]), np.full(s.n, w["tau"]))
    p2.set_initial_state(s.bright_state())
    p2.set_trajectory_offset(rank * B)
    mark("noise_params_and_psi0")
    p2.set_tiling(tiling["traj_chunk"], tiling["vec"], tiling["ctas_per_sm"], tiling["rows_per_block"],
                  tiling["staged"], tiling["groups"])
    mark("workspace_and_block_format")
    p2.reset()
    mark("reset")
    p2.run(1)
    mark("capture_and_first_step")
    p2.run(K - 1)
    mark("steps")
    if world > 1:
        # the ensemble's one exchange: observable sums all-reduced over the ranks (NCCL)
        from dynaquant_b200.ensemble import allreduce_observables
        allreduce_observables(p2, B * world)
        mark("allreduce")
    pops = p2.populations()
    corr = p2.correlation()
    mark("download")
    e2e_s = marks[-1][1] - marks[0][1]
    breakdown = {marks[i][0]: 1e3 * (marks[i][1] - marks[i - 1][1]) for i in range(1, len(marks))}
    p2.close()
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = s.nnz * 12 + (s.n + 1) * 4 + s.n * 16 * 2 + s.n * 16
    d2h = pops.nbytes + corr.nbytes
    e2e = {"value": B * K * world / e2e_s, "unit": "traj-steps/s", "h2d_bytes_per_step": h2d / K,
           "d2h_bytes_per_step": d2h / K, "breakdown_ms": breakdown,
           "note": "whole job through the C ABI from host arrays: context, CSR/noise/psi0 upload, ensemble "
                   "workspace, reset, K steps (the first one captures the step graph), (N > 1: all-reduce of the "
                   "observable sums), populations + correlation download; host clock, a device sync after each "
                   "phase"}
    if rank != 0:
        return
    traffic, traffic_src = measured_traffic(tiling["staged"])
    cpu_v, cpu_sample = cpu_baseline_sample(s, os.cpu_count() or 1)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "traj-steps/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (seeded tube generator)",
        "config": {"workload": w["name"], "n_sites": s.n, "nnz_per_row": (s.nnz - s.n) / s.n, "m": w["m"],
                   "trajectories_per_gpu": B, "dt_fs": w["dt"], "noise": "OU 250/50 fs + static 150",
                   "l2": "inputs larger than L2 (Krylov slabs %.1f GB)" % (8.0 * s.n * B * (w["m"] + 2) / 1e9),
                   "parallelism": (f"ensemble shards x{world}: trajectory ranges per GPU, one NCCL all-reduce of "
                                   "the observables at the end of the e2e run") if world > 1 else "1 GPU",
                   "tiling": {k: tiling[k] for k in ("traj_chunk", "vec", "ctas_per_sm", "rows_per_block", "staged",
                                                    "groups", "ms_per_iter")}},
        "e2e": e2e,
        "gpu_launches": int(kernels_per_step * K),
        "roofline": {"bound": "hbm", "kernel": SPMM_FORMS.get(tiling["staged"], ("SpMM + alpha",))[0],
                     "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": bytes_spmm, "ms_per_launch": spmm_ms,
                     "traffic": traffic,
                     "traffic_source": (traffic_src + " (ncu dram bytes, one launch)") if traffic_src else None,
                     "gather_floor_ms": gather_floor,
                     "frac_of_gather_floor": (gather_floor / spmm_ms) if gather_floor else None,
                     "gather_floor_note": "dq_time_gather_floor: the same row-block walk, records and 16-byte "
                                          "gathers without the FMAs, diagonal, q_{j-1}, alpha and all but one "
                                          "store per block"},
        "kernels_ms_per_launch": {k: v[0] for k, v in prof.items()},
        "eager_step_ms": step_ms_eager,
        "clocks": clocks,
    }
    if world == 1:
        line.update(secondary_legs(s, B, seed, tiling, value))
    else:
        line["note"] = ("the secondary legs (plain FP64, oracle error, reorthogonalisation, adjoint, aggregates, "
                        "ZZ, large tube) and the CPU baseline run at N = 1 only")
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
