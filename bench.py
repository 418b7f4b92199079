"""Benchmark: converged IV points per second of QUICHOTTE's order-2 SCF on B200.

Workload (one "step" = one IV point: solve_scf at the next voltage of the sweep, with
continuation from the previous one, then Current and the observables):
  helix of 10 sites/turn x 6 turns (60 sites, 120x120 complex H), E_CC = 0, t = 1.0 eV,
  SOC lambda = 0.01 eV, radius 0.7 nm, pitch 0.34 nm/turn, hand = +1, wide-band leads
  Gamma_L = Gamma_R = 0.5 eV on the first and last site, U = 1.0 eV on every site,
  2nd order, T = 300 K, mu = 0, 16384 energies on [-12, 12] eV, V from -1 to 1 V in
  steps of 0.05 V (41 voltages), Broyden: the reference's input defaults (alpha_mix 0.5,
  16-column single-precision history, tolf 1e-6, maxscf 300). Synthetic input (the model
  is analytic).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--precision both|fp64|mixed]
                  [--serve R] [--serve-rate r] [--serve-inflight k]

Default: the FP64 form, then the mixed form (the headline value), their ratio and the
error of every observable of the mixed form against the FP64 one over the points both
converged; the CPU oracle on a bounded sample of the same sweep beside the GPU on the same
sample; then a serving stream (p50/p99 latency of IV-point requests through qs_server).

N > 1 (launched with torch.distributed.run): replicas. Rank r solves its own contiguous
block of the voltage sweep; no data-path collective. value = all IV points / max over
ranks of the device time. The reference arm (--impl reference) times the CPU oracle (a
restatement of the reference's Fortran path, oracle/) on the host cores; it loads the
oracle's library only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "quichotte-and-sancho_b200"))

N_IONS, N_TURNS = 10, 6
PITCH, RADIUS = 0.34, 0.7
N_OMEGA, W_LO, W_HI = 16384, -12.0, 12.0
VOLTS = [round(-1.0 + 0.05 * k, 10) for k in range(41)]


def model_cfg1(qb, n_omega=N_OMEGA, ions=N_IONS, turns=N_TURNS):
    """Helix model with its grid exactly on [W_LO, W_HI] with n_omega points
    (omega_i = w_init + i*delta, i = 1..n; w_init = Ev_min - dw, n = int((w_fin-w_init)/delta))."""
    hel_length = PITCH * turns * (ions - 1) / ions  # dz = pitch / N_ions
    args = dict(N_ions=ions, N_turns=turns, hel_length=hel_length, hel_radius=RADIUS, hand=1.0, E_CC=0.0,
                t_hop=1.0, lamb=0.01, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0)
    probe = qb.Model.helix(dw=1.0, up=1.0, delta=0.1, **args)
    ev = np.linalg.eigvalsh(probe.H)
    delta = (W_HI - W_LO) / n_omega
    dw = ev[0] - W_LO  # w_init = W_LO, omega_n = W_LO + n delta = W_HI
    up = W_HI - ev[-1]
    m = qb.Model.helix(dw=dw, up=up, delta=delta, **args)
    if m.n_omega == n_omega - 1:  # int() truncation of (w_fin - w_init)/delta (src/quichotte.f90:246)
        up += 0.5 * delta
        m = qb.Model.helix(dw=dw, up=up, delta=delta, **args)
    assert m.n_omega == n_omega, m.n_omega
    m.alpha_mix, m.nhist, m.tolf, m.maxscf = BROYDEN["alpha_mix"], BROYDEN["nhist"], BROYDEN["tolf"], BROYDEN["maxscf"]
    m.single_history = bool(BROYDEN["single_history"])
    return m


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.samples, self.index = [], index
        self._stop = threading.Event()
        self._t = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
                for k, nm in enumerate(names):
                    if s[4 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# Broyden settings of the workload: the reference's input defaults (src/input_output.f90:
# 109-114). Both arms and every form use them.
BROYDEN = dict(alpha_mix=0.5, nhist=16, tolf=1e-6, maxscf=300, single_history=1)
# energies of the CPU sample grid (the same helix and window; see cpu_sample_sweep)
SAMPLE_N = 512


def bench_config(n_omega, ions, turns, nhist, world):
    """The static description of the workload, identical in every arm's line."""
    N = 2 * ions * turns
    b = dict(BROYDEN, nhist=nhist)
    return {"workload": f"helix {ions}x{turns} ({N}x{N} complex), {n_omega} energies on [-12,12] eV, order 2, "
                        "U=1.0 eV, lambda=0.01 eV, Gamma_L=Gamma_R=0.5 eV, T=300 K; V sweep -1..1 V step 0.05 "
                        "with continuation; the first W voltages warm up, the next K are timed",
            "broyden": {"alpha_mix": b["alpha_mix"], "nhist": b["nhist"], "history": "single" if b["single_history"]
                        else "double", "tolf": b["tolf"], "maxscf": b["maxscf"]},
            "forms": "FP64 GPU form, then the mixed form (headline)",
            "parallelism": f"replicas x{world}", "l2": "working set ~147 GB >> L2 126 MB (no flush needed)"}


def cpu_sample_sweep(volts, n_sample=SAMPLE_N, threads=None, ions=N_IONS, turns=N_TURNS):
    """The CPU oracle (oracle/oracle_py.py: the model built in numpy, only liboracle.so loaded)
    on a bounded sample of the sweep: real converged IV points of the same helix, physics,
    window and Broyden settings at the voltages `volts` (continuation from the first, fresh
    after an unconverged point, as src/quichotte.f90:125-143), on a grid of n_sample energies
    instead of 16384. Returns per-point wall times, step counts and currents."""
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    m = oracle_py.Helix(ions, turns, PITCH * turns * (ions - 1) / ions, RADIUS, 1.0, 0.0, 1.0, 0.01, 1.0, 0.5, 0.5,
                        0.5, 300.0, 0.0, W_LO, (W_HI - W_LO) / n_sample, n_sample)
    s = oracle_py.Solver(m, **BROYDEN)
    out, ok = [], False
    for k, V in enumerate(volts):
        r = s.solve_scf(V, k == 0 or not ok)
        ok = r["converged"]
        out.append(dict(V=V, converged=ok, n_iter=r["n_iter"], wall=r["wall"], J=s.current(V)))
    s.close()
    return out


def scaled_cpu_rate(points, n_sample):
    """IV points/s of the 16384-energy workload from the sample: converged sample points per
    second x n_sample/16384 (the Dyson, Keldysh and Broyden work per SCF step is linear in the
    number of energies and the FFT's n log n only slightly more, so this favours the CPU)."""
    t = sum(p["wall"] for p in points)
    conv = sum(int(p["converged"]) for p in points)
    rate = conv / t if t > 0 else 0.0
    return rate * n_sample / N_OMEGA, rate, t, conv


def cpu_baseline_line(qb, volts, n_sample, ions, turns, device):
    """cpu_baseline of the GPU arm's line: the CPU oracle on a bounded sample (the first
    timed voltages, on the sample grid), and the GPU's FP64 form on exactly the same sample
    points in the same run (device time and wall time), so that the two are compared on
    identical work as well as through the scaled figure."""
    nthr = os.cpu_count()
    pts = cpu_sample_sweep(volts, n_sample, threads=nthr, ions=ions, turns=turns)
    v, v_sample, t, conv = scaled_cpu_rate(pts, n_sample)
    ms = model_cfg1(qb, n_sample, ions, turns)
    s = qb.Solver(ms, device=device, **BROYDEN)
    gdev, gwall, gconv, giters, gJ, ok = 0.0, 0.0, 0, [], [], False
    for k, V in enumerate(volts):
        t0 = time.perf_counter()
        r = s.solve_scf(V, k == 0 or not ok)
        J = s.current(V)
        s.observables()
        gwall += time.perf_counter() - t0
        ok = r["converged"]
        gdev += r["seconds"]
        gconv += int(ok)
        giters.append(r["n_iter"])
        gJ.append(J)
    s.close()
    jc = np.array([p["J"] for p in pts])
    jg = np.array(gJ)
    return {"value": v, "unit": "IV points/s", "cores": nthr, "kind": "port",
            "sample": f"CPU oracle (OpenMP over energies, OpenBLAS zgetrf/zgetri/dposv, radix-4 FFT; oracle/) on "
                      f"{nthr} threads: real converged IV points of the same sweep at V = {volts[0]:g}..{volts[-1]:g} "
                      f"(fresh start at the first) on {n_sample} energies over [-12,12] eV; value = the sample's "
                      f"IV points/s x{n_sample}/{N_OMEGA}",
            "sample_value": v_sample, "sample_s": t, "sample_converged": conv, "sample_energies": n_sample,
            "scf_steps_per_point": [p["n_iter"] for p in pts],
            "gpu_same_sample": {"form": "fp64", "device_s": gdev, "wall_s": gwall, "converged": gconv,
                                "scf_steps_per_point": giters,
                                "value": gconv / gdev if gdev > 0 else 0.0, "e2e": gconv / gwall if gwall > 0 else 0.0,
                                "current_rel_diff_vs_cpu": float(np.max(np.abs(jg - jc)) / np.max(np.abs(jc)))}}


def observable_errors(ref_pts, pts):
    """Error of every observable of `pts` against `ref_pts` (the FP64 form), over the
    points that converged in both: currents relative to the largest |J| of the compared
    points (J crosses zero in the sweep), occupations and the spectral function relative to
    their largest magnitude at each point. Points that either form did not converge are
    excluded and counted."""
    both = [k for k in range(min(len(ref_pts), len(pts))) if ref_pts[k]["converged"] and pts[k]["converged"]]
    out = {"points_compared": len(both), "points_excluded_not_converged": len(pts) - len(both)}
    if not both:
        return out
    jr = np.array([ref_pts[k]["J"] for k in both])
    jm = np.array([pts[k]["J"] for k in both])
    out["current_rel"] = float(np.max(np.abs(jm - jr)) / np.max(np.abs(jr)))
    occ = max(float(np.max(np.abs(pts[k]["occ"] - ref_pts[k]["occ"])) / np.max(np.abs(ref_pts[k]["occ"])))
              for k in both)
    G = max(float(np.max(np.abs(pts[k]["G"] - ref_pts[k]["G"])) / np.max(np.abs(ref_pts[k]["G"]))) for k in both)
    spec = max(float(np.max(np.abs(pts[k]["dosd"] - ref_pts[k]["dosd"])) / np.max(np.abs(ref_pts[k]["dosd"])))
               for k in both)
    out.update(occupation_rel=occ, G_less_obs_rel=G, spectral_rel=spec,
               current_rel_per_point=[float(np.max(np.abs(np.array(pts[k]["J"]) - np.array(ref_pts[k]["J"])))
                                            / np.max(np.abs(jr))) for k in both])
    return out


def voltage_block(rank, world, volts=VOLTS):
    """Replica r's contiguous block of the voltage sweep (no data-path collective: each
    replica continues along its own block)."""
    per = (len(volts) + world - 1) // world
    return volts[rank * per:(rank + 1) * per] or volts[-1:]


def reduce_replicas(dev_s, wall, n_conv, device="cpu"):
    """Max over ranks of the device and wall times, sum of the converged points."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([dev_s, wall], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(n_conv)], device=device, dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), int(c[0])


def serving_requests(qb, n_req, seed=2024):
    """The serving stream: seeded random helices (sites/turn in [3,12], turns in [1,8],
    U ~ U[0.2,1.5] eV, V ~ U[-1,1] V, n_omega in {4096, 8192, 16384, 32768} on [-10,10] eV,
    t = 1 eV, lambda = 0.01 eV, Gamma = 0.5 eV, T = 300 K, 2nd order)."""
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n_req):
        ions, turns = int(rng.integers(3, 13)), int(rng.integers(1, 9))
        U, V = float(rng.uniform(0.2, 1.5)), float(rng.uniform(-1.0, 1.0))
        n = int(rng.choice([4096, 8192, 16384, 32768]))
        args = dict(N_ions=ions, N_turns=turns, hel_length=PITCH * turns * (ions - 1) / ions, hel_radius=RADIUS,
                    hand=1.0, E_CC=0.0, t_hop=1.0, lamb=0.01, U_int=U, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5,
                    T=300.0, mu=0.0, order=2)
        ev = np.linalg.eigvalsh(qb.Model.helix(dw=1.0, up=1.0, delta=0.1, **args).H)
        delta = 20.0 / n
        m = qb.Model.helix(dw=ev[0] + 10.0, up=10.0 - ev[-1] + 0.5 * delta, delta=delta, **args)
        reqs.append((k, m, V, 2 * ions * turns))
    return reqs


def run_serving(qb, n_req, rate, max_inflight, precision):
    """Requests submitted at Poisson arrival times (rate per second) to a qs_server; returns
    latency percentiles (arrival to completion) and throughput."""
    reqs = serving_requests(qb, n_req)
    settings = dict(alpha_mix=0.5, nhist=8, tolf=1e-6, maxscf=300, single_history=1)
    srv = qb.Server(max_inflight=max_inflight)
    rng = np.random.default_rng(7)
    gaps = rng.exponential(1.0 / rate, size=n_req)
    refused, results = [], []
    t0 = time.perf_counter()
    t_next = 0.0
    for (k, m, V, norb), gap in zip(reqs, gaps):
        t_next += gap
        while time.perf_counter() - t0 < t_next:
            results += srv.poll(timeout=min(0.05, max(0.0, t_next - (time.perf_counter() - t0))))
        if srv.submit(m, V, k, precision=precision, **settings) != 0:
            refused.append(k)
    results += srv.drain()
    srv.close()
    ok = [r for r in results if r["status"] == 0]
    lat = np.array([r["t_done"] - r["t_arrival"] for r in ok])
    span = max(r["t_done"] for r in ok) - min(r["t_arrival"] for r in ok) if ok else 0.0
    conv = sum(int(r["converged"]) for r in ok)
    return {"requests": n_req, "arrival_rate_per_s": rate, "max_inflight": max_inflight, "served": len(ok),
            "converged": conv, "refused_too_large": len(refused), "failed": len(results) - len(ok),
            "p50_s": float(np.percentile(lat, 50)) if ok else None, "p99_s": float(np.percentile(lat, 99)) if ok else None,
            "mean_solve_s": float(np.mean([r["solve_s"] for r in ok])) if ok else None,
            "throughput_per_s": conv / span if span > 0 else 0.0, "span_s": span,
            "orbitals": [int(x[3]) for x in reqs]}


def run_reference(args, rank, world):
    """--impl reference: the oracle (a restatement of the reference's CPU path: OpenMP
    over energies, LAPACK zgetrf/zgetri from OpenBLAS, its own FFT; oracle/) on all host
    cores. Each step is a bounded sample of the workload: one real converged IV point of the
    same sweep (same voltage, continuation, model, window and Broyden settings) on a grid of
    --ref-sample energies. The line's value scales the measured rate to the 16384-energy
    grid (scaled_cpu_rate); ms_per_step is the measured time of a sample step."""
    if rank != 0:
        return 0
    nthr = os.cpu_count()
    ions, turns = (int(v) for v in args.helix.split("x"))
    block = voltage_block(0, 1)
    seq = block[:args.warmup + args.steps]
    t0 = time.perf_counter()
    pts = cpu_sample_sweep(seq, args.ref_sample, threads=nthr, ions=ions, turns=turns)
    timed = pts[args.warmup:]
    v, v_sample, t, conv = scaled_cpu_rate(timed, args.ref_sample)
    desc = (f"CPU oracle (OpenMP over energies, OpenBLAS zgetrf/zgetri/dposv, radix-4 FFT; oracle/) on {nthr} "
            f"threads: {len(timed)} real converged IV points of the same sweep (voltages {timed[0]['V']:g}.."
            f"{timed[-1]['V']:g}, continuation after {args.warmup} warm-up points) on {args.ref_sample} energies "
            f"over [-12,12] eV: {conv} converged in {t:.1f} s = {v_sample:.4g} IV points/s; x{args.ref_sample}/"
            f"{N_OMEGA} to the 16384-energy grid")
    line = {"metric": "converged IV points/s", "value": v, "unit": "IV points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / max(len(timed), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": bench_config(args.n_omega, ions, turns, args.nhist, world),
            "cpu_baseline": {"value": v, "unit": "IV points/s", "cores": nthr, "kind": "port", "sample": desc,
                             "sample_value": v_sample, "sample_energies": args.ref_sample,
                             "scf_steps_per_point": [p["n_iter"] for p in timed],
                             "converged": [bool(p["converged"]) for p in timed]},
            "e2e": {"value": v, "unit": "IV points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "run_s": time.perf_counter() - t0}
    print(json.dumps(line), flush=True)
    return 0


def setup_timing(qb, m, repeats=3):
    """The set-up's dense linear algebra on the device, through the public entry points with
    host arrays (copies included), beside LAPACK through numpy on the host cores: the grid
    eigenproblem of the workload's H (zheev, src/quichotte.f90:79-83) and the Loewdin
    transform at the size of the 40-atom helicene model (124 orbitals, 248 spin-orbitals;
    seeded synthetic S = I + perturbation, H0, SOC matrix)."""
    def best(f):
        ts = []
        for _ in range(repeats):
            t = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t)
        return 1e3 * min(ts)
    rng = np.random.default_rng(40)
    N = 124
    P = rng.standard_normal((N, N))
    S = np.eye(N) + 0.05 * (P + P.T) / np.linalg.norm(P + P.T, 2)
    H0 = rng.standard_normal((N, N))
    H0 = 0.5 * (H0 + H0.T)
    X = rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
    Lam = 0.005 * (X + X.conj().T)

    def lowdin_numpy():
        ev, U = np.linalg.eigh(S)
        W = U / np.sqrt(np.sqrt(ev))
        Sx2, Sm2 = np.kron(S, np.eye(2)), np.kron(W @ W.T, np.eye(2))
        Hn = Sm2 @ (np.kron(H0, np.eye(2)) + 0.5 * (Sx2 @ Lam + Lam @ Sx2)) @ Sm2
        return 0.5 * (Hn + Hn.conj().T)
    E, _, info = qb.hermitian_eigensystem(m.H)
    Hd, _ = qb.dftb_lowdin(S, H0, Lam, True)
    Hn = lowdin_numpy()
    return {"eigenvalues_ms": best(lambda: qb.hermitian_eigenvalues(m.H)),
            "eigensystem_ms": best(lambda: qb.hermitian_eigensystem(m.H)),
            "eigensystem_numpy_ms": best(lambda: np.linalg.eigh(m.H)),
            "eigensystem_rel_err": float(np.max(np.abs(E - np.linalg.eigvalsh(m.H))) / np.max(np.abs(E))),
            "lowdin_ms": best(lambda: qb.dftb_lowdin(S, H0, Lam, True)), "lowdin_numpy_ms": best(lowdin_numpy),
            "lowdin_rel_err": float(np.max(np.abs(Hd - Hn)) / np.max(np.abs(Hn))),
            "workload": f"eigenvalues (the grid) and eigenpairs of the {m.Norb}x{m.Norb} H; Loewdin at N=124 "
                        "(248 spin-orbitals); "
                        f"host arrays, best of {repeats}; numpy = LAPACK on the host cores"}


def setup_scan(qb):
    """Sizes and batches of the device set-up beside LAPACK (numpy) on the host cores: random
    Hermitian matrices (seeded) for the eigenproblem, seeded S = I + perturbation, H0 and SOC
    matrix for the Loewdin transform. Wall times through the public API with host arrays,
    the best of 3 calls for the small cases, after one call of every kernel."""
    rng = np.random.default_rng(0)

    def herm(N):
        X = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        return (X + X.conj().T) / 2

    def wall(f, repeats=1):
        best = None
        for _ in range(repeats):
            t = time.perf_counter()
            r = f()
            dt = time.perf_counter() - t
            best = dt if best is None else min(best, dt)
        return r, best
    # every kernel once (the first launch of a kernel in a process loads it)
    qb.hermitian_eigensystem(herm(16))
    qb.hermitian_eigenvalues(herm(16))
    qb.dftb_lowdin(np.eye(4), np.eye(4), np.zeros((8, 8), complex))
    out = {}
    for N, batch in [(120, 1), (120, 64), (248, 1), (248, 16), (512, 1), (1024, 1), (2048, 1)]:
        A = np.stack([herm(N) for _ in range(batch)])
        rep = 3 if N * N * batch <= 1 << 20 else 1
        (E, _, info), tg = wall(lambda: qb.hermitian_eigensystem(A), rep)
        (En, _), tc = wall(lambda: np.linalg.eigh(A), rep)
        out[f"eigensystem_N{N}_batch{batch}"] = {"device_s": tg, "numpy_s": tc, "info": int(np.max(info)),
                                                 "rel_err": float(np.max(np.abs(E - En)) / np.max(np.abs(En)))}
        (Ev, info), tg = wall(lambda: qb.hermitian_eigenvalues(A), rep)
        Env, tc = wall(lambda: np.linalg.eigvalsh(A), rep)
        out[f"eigenvalues_N{N}_batch{batch}"] = {"device_s": tg, "numpy_s": tc, "info": int(np.max(info)),
                                                 "rel_err": float(np.max(np.abs(Ev - Env)) / np.max(np.abs(Env)))}
    for N in (124, 1024):
        P = rng.standard_normal((N, N))
        S = np.eye(N) + 0.05 * (P + P.T) / np.linalg.norm(P + P.T, 2)
        H0 = rng.standard_normal((N, N))
        H0 = 0.5 * (H0 + H0.T)
        X = rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
        Lam = 0.005 * (X + X.conj().T)

        def ref():
            ev, U = np.linalg.eigh(S)
            W = U / np.sqrt(np.sqrt(ev))
            Sx2, Sm2 = np.kron(S, np.eye(2)), np.kron(W @ W.T, np.eye(2))
            Hn = Sm2 @ (np.kron(H0, np.eye(2)) + 0.5 * (Sx2 @ Lam + Lam @ Sx2)) @ Sm2
            return 0.5 * (Hn + Hn.conj().T)
        rep = 3 if N <= 256 else 1
        (H, _), tg = wall(lambda: qb.dftb_lowdin(S, H0, Lam, True), rep)
        Hn, tc = wall(ref, rep)
        out[f"lowdin_N{N}"] = {"device_s": tg, "numpy_s": tc,
                               "rel_err": float(np.max(np.abs(H - Hn)) / np.max(np.abs(Hn)))}
    return {"setup_scan": out, "numpy_threads": os.cpu_count()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sample", type=int, default=SAMPLE_N, help="energies of the CPU sample grid")
    ap.add_argument("--cpu-points", type=int, default=3, help="timed voltages in the GPU arm's CPU sample")
    ap.add_argument("--n-omega", type=int, default=N_OMEGA, help="smaller grids for profiling only")
    ap.add_argument("--nhist", type=int, default=BROYDEN["nhist"], help="smaller histories for profiling only")
    ap.add_argument("--helix", default=f"{N_IONS}x{N_TURNS}", help="sites/turn x turns; other sizes for profiling only")
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: time kernel variants per size (default); 2/3: force variant 1/2 (profiling only)")
    ap.add_argument("--serve", type=int, default=16,
                    help="requests of the serving stream (0: none; the full stream is 512)")
    ap.add_argument("--serve-rate", type=float, default=2.0, help="Poisson arrivals per second")
    ap.add_argument("--serve-inflight", type=int, default=4, help="solves on the device at once")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="both: the FP64 form, then the mixed form (headline value), with their ratio")
    ap.add_argument("--setup-scan", action="store_true",
                    help="time the device set-up (eigenproblem, Loewdin) over sizes against LAPACK, print, exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.setup_scan:
        import quichotte_b200 as qb
        print(json.dumps(setup_scan(qb)), flush=True)
        return 0
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import quichotte_b200 as qb

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    qb.autotune(args.autotune)
    ions, turns = (int(v) for v in args.helix.split("x"))
    m = model_cfg1(qb, args.n_omega, ions, turns)
    block = voltage_block(rank, world)
    seq = [block[k % len(block)] for k in range(args.warmup + args.steps)]
    fresh = [k == 0 or (k % len(block) == 0) for k in range(len(seq))]
    obs_bytes = 8 * (2 * m.Norb * m.Norb + m.Norb * m.n_omega + 2 * m.n_omega)
    settings = dict(BROYDEN, nhist=args.nhist)

    def run_arm(precision):
        """warm-up + timed IV points of one solver form; the two forms do not fit in HBM
        together, so each arm creates and releases its own solver"""
        solver = qb.Solver(m, precision=precision, device=local, **settings)
        prev_ok = False
        for k in range(args.warmup):
            # continuation as the reference's sweep: fresh after an unconverged voltage
            r = solver.solve_scf(seq[k], fresh[k] or not prev_ok)
            prev_ok = r["converged"]
            solver.current(seq[k])
            solver.observables()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        solver.profile(True)
        l0 = qb.kernel_launches()
        dev_s, points = 0.0, []
        wall0 = time.perf_counter()
        for k in range(args.warmup, args.warmup + args.steps):
            r = solver.solve_scf(seq[k], fresh[k] or not prev_ok)
            prev_ok = r["converged"]
            dev_s += r["seconds"]
            J = solver.current(seq[k])
            o = solver.observables()  # G_less_obs, dosd, trU, trD back to host buffers
            points.append(dict(V=seq[k], converged=r["converged"], n_iter=r["n_iter"], n_mixed=r["n_mixed"],
                               seconds=r["seconds"], J=J, occ=np.imag(np.diag(o["G_less_obs"])).copy(),
                               G=o["G_less_obs"], dosd=o["dosd"]))
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        n_conv = sum(int(p["converged"]) for p in points)
        out = dict(launches=qb.kernel_launches() - l0, prof=solver.profile(False), clk=clocks.stop(), points=points,
                   nA=solver.nA, Nf=solver.Nf, n_vec=solver.n_vec)
        solver.close()
        if world > 1:
            dev_s, wall, n_conv = reduce_replicas(dev_s, wall, n_conv, device="cuda")
            dist.barrier()
        out.update(dev_s=dev_s, wall=wall, n_conv=n_conv, value=n_conv / dev_s if dev_s > 0 else 0.0,
                   e2e=n_conv / wall if wall > 0 else 0.0)
        return out

    arms = {}
    for prec in (["fp64", "mixed"] if args.precision == "both" else [args.precision]):
        arms[prec] = run_arm(qb.QS_PREC_MIXED if prec == "mixed" else qb.QS_PREC_FP64)
    head = arms.get("mixed") or arms["fp64"]
    f64 = arms.get("fp64")
    dev_s, wall, n_conv = head["dev_s"], head["wall"], head["n_conv"]
    launches, clk = head["launches"], head["clk"]
    prof = (f64 or head)["prof"]
    if rank == 0:
        peaks, src = measured_peaks()
        # roofline of the dominant kernel of the FP64 form (largest device time):
        # algorithmic work per launch
        N, nA, n = m.Norb, head["nA"], m.n_omega
        fam, (ms, cnt) = max(prof.items(), key=lambda kv: kv[1][0])
        nY, Nf, nvec = nA * nA + nA * (nA + 1) // 2, head["Nf"], head["n_vec"]
        nh = args.nhist
        work = {  # algorithmic FLOPs (FP64 compute-bound kernels) or bytes (HBM-bound) per launch
            "dyson_gj": ("fp64", n * 8.0 * N ** 3),                       # G^r: N^3 complex MACs per energy
            "keldysh_scf2": ("fp64", n * 16.0 * nA ** 3),                 # G^< = G SL G^a: 2 nA^3 complex MACs
            "sig2_fwdA": ("hbm", nvec * 8.0 + nY * Nf * 16.0),            # read packed G, write Y
            "sig2_mid": ("hbm", (nY + 2.0 * nA * nA) * Nf * 16.0),         # read Y, write V
            "sig2_invC": ("hbm", 2.0 * nA * nA * Nf * 16.0 + 2.0 * nA * nA * n * 16.0),  # read V, write Sigma
            "broyden": ("hbm", nvec * (64.0 + 12.0 * nh) / 3.0),          # per iteration / 3 launches
        }
        # DRAM bytes per launch measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum)
        # on the 120x120 helix: Dyson and Keldysh per energy at 1024 energies
        # (profiles/dyson_bgj_helix120_n1024.md, profiles/keldysh_tc_helix120_n1024.md); the
        # Broyden kernels per vector element (profiles/broyden_kernels_helix120.md)
        traffic_per_unit = {"dyson_gj": ((236.776192e6 + 183.729152e6) / 1024, n),
                            "keldysh_scf2": ((1064.643e6 + 800.101376e6) / 1024, n)}
        roof = None
        if fam in work and cnt:
            kind, per_launch = work[fam]
            t = ms / cnt * 1e-3
            if kind == "fp64":
                achieved, peak, unit = per_launch / t / 1e12, 37.0, "TFLOP/s"
                src_note = "nominal B200 FP64 37 TFLOP/s (MEASURED_PEAKS.json has no FP64 figure)"
            else:
                achieved, peak, unit = per_launch / t / 1e9, peaks.get("hbm_gbs", 6650.0), "GB/s"
                src_note = f"hbm_gbs of MEASURED_PEAKS.json ({src})"
            tpu = traffic_per_unit.get(fam) if (N, nA) == (120, 120) else None
            roof = {"kernel": fam, "bound": kind, "achieved": achieved, "peak": peak, "unit": unit,
                    "frac": achieved / peak, "traffic": tpu[0] * tpu[1] if tpu else None,
                    "traffic_note": "DRAM bytes per launch from an ncu capture, scaled per unit" if tpu else None,
                    "peak_source": src_note,
                    "per_launch_work": per_launch, "launches": cnt, "avg_launch_ms": ms / cnt}
        prec_name = "mixed" if "mixed" in arms else "fp64"
        pts = head["points"]
        line = {
            "metric": "converged IV points/s", "value": n_conv / dev_s if dev_s > 0 else 0.0,
            "unit": "IV points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if prec_name == "mixed" else "f64", "data": "synthetic",
            "config": bench_config(n, ions, turns, args.nhist, world),
            "form": prec_name,
            "voltages": [p["V"] for p in pts],
            "converged": [bool(p["converged"]) for p in pts],
            "scf_steps_per_point": [p["n_iter"] for p in pts],
            "converged_points": n_conv,
            "e2e": {"value": n_conv / wall if wall > 0 else 0.0, "unit": "IV points/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": obs_bytes},
            "gpu_launches": launches,
            "kernel_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1]},
            "roofline": roof,
            "clocks": clk,
            "currents_A": [list(p["J"]) for p in pts],
        }
        if "mixed" in arms:
            line["mixed_form"] = ("Sigma2 FFTs, 2x2 algebra and spectra in FP32 while max|F| > max(1e-5, 100 tolf) "
                                  "(the FP32 noise floor is ~1e-5); then FP64 steps until an FP64 residual meets "
                                  "tolf; Dyson/Keldysh, Broyden and observables FP64")
            line["fp32_steps_per_point"] = [p["n_mixed"] for p in pts]
        if f64 is not None and "mixed" in arms:
            line["fp64"] = {"value": f64["value"], "e2e": f64["e2e"], "ms_per_step": 1000.0 * f64["dev_s"] / args.steps,
                            "converged": [bool(p["converged"]) for p in f64["points"]],
                            "scf_steps_per_point": [p["n_iter"] for p in f64["points"]],
                            "kernel_ms": {k: round(v[0], 3) for k, v in f64["prof"].items() if v[1]}}
            line["mixed_over_fp64"] = head["value"] / f64["value"] if f64["value"] > 0 else None
            line["err_vs_fp64"] = observable_errors(f64["points"], pts)
            line["kernel_ms_mixed"] = {k: round(v[0], 3) for k, v in head["prof"].items() if v[1]}
        if world == 1 and args.serve > 0:
            line["serving"] = run_serving(qb, args.serve, args.serve_rate, args.serve_inflight, qb.QS_PREC_FP64)
            line["serving"]["workload"] = (f"serving stream, first {args.serve} of the seeded 512-request stream: random "
                                           "helices, sites/turn 3-12, turns 1-8, U 0.2-1.5 eV, V -1..1 V, 4096-32768 "
                                           "energies, Poisson arrivals; one fresh-start IV point per request, FP64, "
                                           "Broyden nhist 8; requests above the HBM budget are refused")
        if world == 1:
            line["setup"] = setup_timing(qb, m)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_line(qb, seq[args.warmup:args.warmup + args.cpu_points], args.ref_sample,
                                                     ions, turns, local)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
