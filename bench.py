"""Benchmark: FP64 scan energies/sec of the per-energy scattering path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config h2o_like|h2_like|h2o_mixed|c8f8_like] [--slots S] [--groups G]
                    [--graphs 0|1] [--autotune 0|1]

Workload (default): the H2O-like system -- O + 2 H, five doubly occupied
orbitals, l_cont = 20 (441 continuum + 605 exchange channels, N_t = 1046),
dr = 0.005 bohr, 12001 radial points, momenta k = 0.05 .. 2.0 (200 energies).
Inputs are seeded synthetic data of those shapes (no molecular file exists
here).  The energies stream through the library's scan (scatt_scan_*): S
device slots in G phase groups started a fraction 1/G of the radial sweep
apart; a step is one group finishing -- S/G energies solved end to end
(Schur inverses, R-ratio recurrence, K, asymptotic fit, dipoles) while the
other groups advance by 1/G of their sweep -- and the finished slots take the
next energies of the k grid at once.  Under torchrun each rank streams its
own contiguous block of the k grid (energies are independent: weak scaling,
no data-path collective).

value      energies/s of the whole job over the timed steps, device time
           (CUDA events on the library's stream), max over ranks;
e2e        the same steps through the C ABI with host buffers: energies
           submitted from host memory, every output of the finished energies
           read back into pinned host memory, host clock, max over ranks;
roofline   the dominant kernel group -- the batched R^-1 inversion -- as
           achieved FP64 TF/s (2 n^3 per matrix, over the sampled inversions)
           against the cuBLAS DGEMM peak measured on this GPU in the same run;
cpu_baseline  the oracle port timed on a bounded sample of the same workload
           on this host's cores, extrapolated to energies/s.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "spion-emol_b200", "python"))

import numpy as np  # noqa: E402

CONFIGS = {
    "h2o_like": dict(builder="h2o_like", kw=dict(Nr=12001, dr=0.005, l_cont=20, lmax_orb=40, n_orb=5),
                     ks=lambda: np.linspace(0.05, 2.0, 200), slots=128, groups=16, graphs=0),
    "h2_like": dict(builder="h2_like", kw=dict(Nr=4001, dr=0.01, l_cont=8),
                    ks=lambda: np.arange(1, 21) * 0.1, slots=20, groups=4, graphs=1),
    # the batched scan of mixed continuum cutoffs: 256 energies, l_cont 12 / 16 / 20 in turn
    "h2o_mixed": dict(builder="h2o_like", kw=dict(Nr=12001, dr=0.005, l_cont=20, lmax_orb=40, n_orb=5),
                      ks=lambda: np.linspace(0.05, 2.0, 256), slots=128, groups=16, graphs=0,
                      l_conts=(12, 16, 20)),
    # C8F8-like production shape: 36 occupied orbitals (N_f = 36 x 121 = 4356) and
    # l_cont = 30 (961 continuum channels, the size of the ~950-channel symmetry
    # block), N_t = 5317; 10001 points at dr = 0.01; one energy in flight
    "c8f8_like": dict(builder="c8f8_like", kw=dict(Nr=10001, dr=0.01, l_cont=30, lmax_orb=40, n_orb=36),
                      ks=lambda: np.linspace(0.1, 2.0, 50), slots=1, groups=1, graphs=0),
}

SEEDS = {"h2_like": 0, "h2o_like": 1, "c8f8_like": 4}
DATA = {"h2_like": "synthetic (seeded H2-like inputs of the benchmark shapes)",
        "h2o_like": "synthetic (seeded H2O-like inputs of the benchmark shapes)",
        "c8f8_like": "synthetic (seeded C8F8-like inputs of the benchmark shapes)"}


# DRAM bytes (read + write) of the trailing updates of one sampled R^-1
# inversion of the scan, keyed by (config, slots, groups).  From one ncu
# capture of gj3_trail128_kernel on 32 matrices of order 1046 (452.7 MB for
# 15 of the 17 column tiles of one 128-column window), scaled to 17 tiles,
# 128 matrices and the call's 9 windows: the C tiles are read and written
# once per window, so the traffic grows with the tiles and matrices.
INVERSE_TRAFFIC: dict = {("h2o_like", 128, 16): 452.7e6 * 17 / 15 * 4 * 9}


# Device seconds of one chunk (8 radial steps) with every slot busy, as
# fixed + per-slot parts: the inverse's pivot chain is one CTA per matrix and
# costs the same for any batch, the trailing updates and GEMMs grow with the
# slots.  Measured on one B200 in FP64: H2O-like 57.3 ms per chunk at 32 slots
# and 200 ms at 128 slots (8 x 3.6 ms of it the chain); H2-like 3.2 ms at 20
# slots (launch-bound).
CHUNK_S = {"h2o_like": (0.0288, 0.00134), "h2_like": (0.0016, 0.00008), "h2o_mixed": (0.0288, 0.00134),
           "c8f8_like": (0.0, 0.28)}


def plan(config: str, slots: int, groups: int, steps: int, warmup: int) -> dict:
    """Chunks of 8 radial steps the bench runs.  The first step ends when
    group 0 has swept the whole grid (the later groups start 1/groups of a
    sweep apart); every later step is one group finishing, 1/groups of a
    sweep.  Warm-up steps come first."""
    Nr = CONFIGS[config]["kw"]["Nr"]
    cps = -(-Nr // 8)                        # a sweep covers n = 0 .. N = Nr - 1
    per_step = -(-cps // groups)
    n_steps = warmup + steps
    total = (cps + (n_steps - 1) * per_step) if n_steps > 0 else 0
    return {"chunks_per_sweep": cps, "chunks_first_step": cps, "chunks_per_step": per_step,
            "chunks_total": total, "chunks_timed": steps * per_step if warmup > 0 else total}


def predict_seconds(config: str, slots: int, groups: int, steps: int, warmup: int, setup_s: float = 120.0,
                    cpu_s: float = 30.0) -> float:
    """Wall time of `bench.py --config C --steps K --warmup W`: the chunks at
    the measured cost per chunk (post stages included in it), plus setup
    (upload, cuBLAS peak, autotune) and the CPU baseline."""
    fixed, per_slot = CHUNK_S[config]
    return setup_s + cpu_s + plan(config, slots, groups, steps, warmup)["chunks_total"] * (fixed + per_slot * slots)


def job_grid(config: str, world: int) -> np.ndarray:
    """The k grid of the whole job: the workload's grid at one GPU; at N
    ranks the same k range with N times the points, so that every rank
    streams as many energies as one GPU does (weak scaling: the per-rank
    work is fixed as N grows)."""
    ks = CONFIGS[config]["ks"]()
    if world <= 1:
        return ks
    return np.linspace(ks[0], ks[-1], ks.size * world)


def rank_block(config: str, world: int, rank: int, n_f: int):
    """This rank's contiguous, cost-balanced block of the job's k grid: the
    momenta and each energy's continuum cutoff."""
    from scatt_b200 import shard
    cfg = CONFIGS[config]
    ks = job_grid(config, world)
    lcs = cfg.get("l_conts")
    lc_all = (np.array([lcs[i % len(lcs)] for i in range(ks.size)], dtype=np.int32) if lcs
              else np.full(ks.size, cfg["kw"]["l_cont"], dtype=np.int32))
    blocks = shard.partition(shard.energy_cost(lc_all, n_f), world)
    return ks[blocks[rank]], lc_all[blocks[rank]]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    r = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                        "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                    if r.returncode == 0:
                        self.samples.append([x.strip() for x in r.stdout.strip().split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cuda_dgemm_peak(torch):
    """cuBLAS DGEMM 8192^3, best of 10 (the FP64 denominator of the roofline)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def oracle_setup(inp, l_conts=None):
    """The oracle's energy-independent tables for this workload (built once,
    never timed): one setup, or one per continuum cutoff of a mixed scan."""
    from oracle import solver as O
    if l_conts:
        return [O.make_setup(inp, l_cont=lc) for lc in l_conts]
    return O.make_setup(inp)


def oracle_baseline_mix(sts, ks, budget_s=20.0):
    """oracle_baseline over the cutoffs of a mixed scan, which cycles through
    them in equal shares: the budget is split between them and the seconds
    per energy averaged."""
    if not isinstance(sts, list):
        return oracle_baseline(sts, ks, budget_s)
    parts = [oracle_baseline(st, ks, budget_s / len(sts)) for st in sts]
    t = float(np.mean([p["sec_per_energy"] for p in parts]))
    return {"value": 1.0 / t, "unit": "energies/s", "cores": parts[0]["cores"], "cpu_model": parts[0]["cpu_model"],
            "kind": "port",
            "sample": " | ".join(f"l_cont {st.l_cont}: " + p["sample"] for st, p in zip(sts, parts))
                      + "; seconds per energy averaged over the cutoffs",
            "sec_per_energy": t}


def cpu_model() -> str:
    """The host CPU's model name (first entry of /proc/cpuinfo), for the baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_baseline(st, ks, budget_s=20.0):
    """Time the CPU oracle on a bounded sample of one energy and extrapolate.

    Sample: the stage-by-stage oracle steps (Schur inverse + R-recursion step +
    backward step + W^-1 apply) over up to 200 radial points inside the
    exchange region and up to 200 outside it, each stretch with half of the
    budget, scaled to the full grid.  The asymptotic fit, K extraction and the
    dipole quadrature (once per energy) are left out, which favours the oracle.
    """
    from oracle import solver as O
    E = 0.5 * float(ks[len(ks) // 2]) ** 2
    nthreads = os.cpu_count()

    def per_step(n0, count, bud):
        prev = O.analytic_init(st, E, 1) if n0 < O.n_start(st) else np.zeros((st.Nt, st.Nt))
        Z = np.random.default_rng(0).standard_normal((st.Nt, st.n_mu))
        t = time.time()
        done = 0
        for n in range(n0, n0 + count):
            Sinv = O.sinv_at(st, E, n)
            Rinv = O.frp_step(st, n, Sinv, prev)
            prev = Rinv
            Z = Rinv @ Z                                   # BackPropagator step
            O.winv_apply(st, n, Sinv, Z)
            done += 1
            if time.time() - t > bud:
                break
        return (time.time() - t) / max(done, 1), done

    n_in = max(O.STAB_N_MAX, min(st.n_tr // 2, st.Nr - 200))
    t_in, c_in = per_step(n_in, 200, 0.5 * budget_s)
    n_out = min(st.Nr - 300, max(st.n_tr + 10, st.Nr // 2))
    t_out, c_out = per_step(n_out, 200, 0.5 * budget_s)
    inner = min(st.n_tr, st.Nr)
    t_energy = inner * t_in + (st.Nr - inner) * t_out
    return {
        "value": 1.0 / t_energy,
        "unit": "energies/s",
        "cores": nthreads,
        "cpu_model": cpu_model(),
        "kind": "port",
        "sample": (f"oracle (numpy/scipy-OpenBLAS, {nthreads} threads): {c_in} radial steps at n={n_in} "
                   f"(exchange region) and {c_out} at n={n_out} of one energy (k={np.sqrt(2 * E):.3f}); "
                   f"Schur inverse + R-ratio step + backward step each, extrapolated to {st.Nr} points "
                   f"(n_transition={st.n_tr}); K extraction, fit and dipole tails left out"),
        "sec_per_energy": t_energy,
    }


def pinned_alloc(torch):
    """Host output arrays in page-locked memory (device-to-host at full speed)."""
    keep = []

    def mk(shape, dtype=np.float64):
        t = torch.empty(shape, dtype=torch.from_numpy(np.zeros(0, dtype=dtype)).dtype, pin_memory=True)
        t.zero_()
        keep.append(t)
        return t.numpy()
    return mk, keep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="h2o_like", choices=list(CONFIGS))
    ap.add_argument("--slots", type=int, default=0)
    ap.add_argument("--groups", type=int, default=0)
    ap.add_argument("--graphs", type=int, default=-1, help="replay chunks from CUDA graphs (default: per config)")
    ap.add_argument("--keep-window", type=int, default=0,
                    help="1: keep the fit window store (fit residual diagnostics); 0: accumulate the fit forward")
    ap.add_argument("--autotune", type=int, default=1,
                    help="time the inverse's blockings for the workload's orders before the run")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="seconds of oracle work per CPU sample (the reference arm takes one per step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    a = ap.parse_args()
    ws, rank, local = dist_env()
    cfg = CONFIGS[a.config]
    from scatt_b200 import synth
    ks = job_grid(a.config, ws)
    slots = a.slots or cfg["slots"]
    groups = a.groups or cfg["groups"]
    graphs = cfg["graphs"] if a.graphs < 0 else a.graphs
    workload = {"workload": a.config, **cfg["kw"], "energies": int(len(ks)), "slots": slots, "groups": groups,
                "energies_per_step": slots // groups,
                "seed": synth.SEED_BASE + SEEDS[cfg["builder"]]}
    if cfg.get("l_conts"):
        workload["l_cont_per_energy"] = list(cfg["l_conts"])

    if a.impl == "reference":
        if rank != 0:
            return
        inp = getattr(synth, cfg["builder"])(**cfg["kw"])
        st = oracle_setup(inp, cfg.get("l_conts"))      # energy-independent tables, not timed
        steps = []
        for _ in range(a.warmup + a.steps):
            steps.append(oracle_baseline_mix(st, ks, budget_s=a.cpu_budget))
        timed = steps[a.warmup:]
        v = float(np.mean([s["value"] for s in timed]))
        line = {"impl": "reference", "metric": "FP64 scan energies/sec", "value": v, "unit": "energies/s",
                "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": workload,
                "cpu_baseline": {k: timed[-1][k] for k in ("value", "unit", "cores", "cpu_model", "kind", "sample")},
                "e2e": {"value": v, "unit": "energies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from scatt_b200 import solver as S
    from scatt_b200 import _lib

    inp = getattr(synth, cfg["builder"])(**cfg["kw"])
    t0 = time.time()
    sol = S.ScanSolver(inp, device=local)
    setup_s = time.time() - t0
    # this rank's contiguous block of the job's k grid (cost-balanced)
    k_mine, lc_mine = rank_block(a.config, ws, rank, sol.Nf)
    Es_all = 0.5 * k_mine ** 2
    if slots > len(Es_all):
        raise SystemExit(f"--slots {slots} exceeds this rank's {len(Es_all)} energies")
    gsize = slots // groups
    cursor = [0]

    def next_energies(n):
        idx = [(cursor[0] + i) % len(Es_all) for i in range(n)]
        cursor[0] += n
        return Es_all[idx], lc_mine[idx]

    tuned = []
    if a.autotune:
        # inverses of the scan's batches: R^-1 of order N_t over the slots, and the
        # Schur inverses of order Np over the slots' 8 radial steps of a chunk
        # (orders above 1280 have one blocking, the cluster panel: nothing to tune)
        for n, count in sorted({(sol.Np + sol.Nf, slots), (sol.Np, slots * 8)}):
            if n <= 1280:
                tuned.append(_lib.autotune_inverse(n, count, device=local))
    peak = cuda_dgemm_peak(torch) if rank == 0 else None
    alloc, _keep = pinned_alloc(torch)
    opts = S.default_opts(allow_closed_channels=1, timing=1, use_graphs=graphs, keep_window=a.keep_window)
    scan = sol.scan(slots=slots, groups=groups, opts=opts, alloc=alloc)
    assert (scan.slots, scan.groups) == (slots, groups)
    scan.submit(*next_energies(slots))
    for w in range(a.warmup):
        scan.submit(*next_energies(gsize))
        scan.step(results=False)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    st0 = sol.last_stats()
    clocks = ClockSampler(local)
    clocks.start()
    n_done = 0
    out_bytes = 0
    t_host = time.time()
    for k in range(a.steps):
        scan.submit(*next_energies(gsize))              # energies from host memory
        n_done += len(scan.step(results=False))         # outputs back in pinned host memory
        out_bytes += scan.last_out_bytes
    torch.cuda.synchronize()
    host_s = time.time() - t_host
    ck = clocks.stop()
    st1 = sol.last_stats()
    dev_s = st1["device_s"] - st0["device_s"]
    rinv_s = st1["rinv_s"] - st0["rinv_s"]
    rinv_flops = st1["rinv_flops"] - st0["rinv_flops"]
    launches = st1["launches"] - st0["launches"]
    if ws > 1:
        dist.barrier()
        t = torch.tensor([dev_s, host_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, host_s = float(t[0]), float(t[1])
        c = torch.tensor([n_done], dtype=torch.float64, device="cuda")
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        n_total = int(c[0])
    else:
        n_total = n_done
    scan.close()
    if rank == 0:
        Nt = sol.Np + sol.Nf
        achieved = rinv_flops / rinv_s / 1e12 if rinv_s > 0 else None
        line = {
            "metric": "FP64 scan energies/sec", "value": n_total / dev_s, "unit": "energies/s",
            "n_gpus": ws, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * dev_s / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA[cfg["builder"]],
            "config": {**workload, "parallelism": f"energy-sharded x{ws}", "cuda_graphs": bool(graphs),
                       "fit": "window store and back sweep (fit residual diagnostics)" if a.keep_window else
                              "accumulated forward, [A; B] = G_A(N-1)^T Z_N (no window store; fit residual not computed)",
                       "autotuned_inverses": tuned,
                       "l2": "inputs larger than L2 (the scan's device state, several GB, exceeds the 126 MB L2)"},
            "e2e": {"value": n_total / host_s, "unit": "energies/s", "h2d_bytes_per_step": 8 * gsize,
                    "d2h_bytes_per_step": int(out_bytes / max(a.steps, 1))},
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if (achieved and peak) else None,
                         "traffic": INVERSE_TRAFFIC.get((a.config, slots, groups)),
                         "kernel": f"batched R^-1 (Gauss-Jordan, N_t={Nt} in the exchange region, "
                                   f"{sol.Np} outside; {slots} matrices a call); "
                                   "peak = cuBLAS DGEMM 8192^3 measured in this run (FP64 of measured)"},
            "clocks": ck,
            "setup_s": setup_s,
        }
        if not a.no_cpu_baseline and ws == 1:         # the CPU baseline is an N = 1 figure
            try:
                line["cpu_baseline"] = {k: v for k, v in oracle_baseline_mix(oracle_setup(inp, cfg.get("l_conts")), ks,
                                                                             a.cpu_budget).items()
                                        if k in ("value", "unit", "cores", "cpu_model", "kind", "sample")}
            except Exception as ex:          # the baseline is reported, never required
                line["cpu_baseline"] = {"value": None, "error": str(ex)}
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
