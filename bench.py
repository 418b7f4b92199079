"""Benchmark: converged IV points per second of QUICHOTTE's order-2 SCF on B200.

Workload (one "step" = one IV point: solve_scf at the next voltage of the sweep, with
continuation from the previous one, then Current and the observables):
  helix of 10 sites/turn x 6 turns (60 sites, 120x120 complex H), E_CC = 0, t = 1.0 eV,
  SOC lambda = 0.01 eV, radius 0.7 nm, pitch 0.34 nm/turn, hand = +1, wide-band leads
  Gamma_L = Gamma_R = 0.5 eV on the first and last site, U = 1.0 eV on every site,
  2nd order, T = 300 K, mu = 0, 16384 energies on [-12, 12] eV, V from -1 to 1 V in
  steps of 0.05 V (41 voltages), Broyden: reference defaults (alpha_mix 0.5, 16-column
  single-precision history, tolf 1e-6). Synthetic input (the model is analytic).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--precision both|fp64|mixed]
                  [--serve R] [--serve-rate r] [--serve-inflight k]

Default: the FP64 form, then the mixed form (the headline value), their ratio and the
current error of the mixed form against the FP64 one; then a serving stream (p50/p99
latency of IV-point requests through qs_server).

N > 1 (launched with torch.distributed.run): replicas. Rank r solves its own contiguous
block of the voltage sweep; no data-path collective. value = all IV points / max over
ranks of the device time. The reference arm (--impl reference) times the CPU oracle
(a restatement of the reference's Fortran path) on the host cores.
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
    m.alpha_mix, m.nhist, m.tolf, m.maxscf, m.single_history = 0.5, 16, 1e-6, 300, True
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


# SCF steps per IV point of this workload, measured on B200 (both arms run the same
# Broyden algorithm, so the oracle takes the same number of steps up to rounding)
STEPS_PER_POINT = 25.5


def cpu_baseline_sample(n_sample=4096, steps_per_point=STEPS_PER_POINT, threads=None):
    """The CPU oracle on a bounded sample of the workload: one SCF step (scf_residual2:
    Sigma2 by FFT + the Dyson/Keldysh sweep) of the same helix on the same energy window
    with n_sample energies, scaled linearly to the 16384-energy grid and multiplied by the
    SCF steps of one IV point. The Broyden update is left out (in the CPU's favour)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    import quichotte_b200 as qb
    m = model_cfg1(qb, n_sample)
    s = oracle_lib.solver(m, nhist=0)
    x = s.initial_vector(VOLTS[0])
    t0 = time.perf_counter()
    F, ab = s.residual(VOLTS[0], x)
    dt = time.perf_counter() - t0
    s.close()
    scale = N_OMEGA / n_sample
    per_point = dt * scale * steps_per_point
    return {"value": 1.0 / per_point, "unit": "IV points/s", "cores": threads or os.cpu_count(), "kind": "port",
            "sample": f"CPU oracle (OpenMP, OpenBLAS zgetrf/zgetri, own FFT), one scf_residual2 of the same helix "
                      f"on {n_sample} energies over [-12,12] eV: {dt:.2f} s; x{scale:g} to 16384 energies and "
                      f"x{steps_per_point:g} SCF steps per IV point; Broyden update not counted"}


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
    over energies, LAPACK zgetrf/zgetri from OpenBLAS, its own FFT) on the host cores."""
    if rank != 0:
        return 0
    nthr = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(nthr))
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cb = cpu_baseline_sample(args.ref_sample, threads=nthr)
        if k >= args.warmup:
            times.append(1.0 / cb["value"])
    t = sum(times)
    v = args.steps / t
    line = {"metric": "converged IV points/s", "value": v, "unit": "IV points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "helix 10x6 (120x120), 16384 energies on [-12,12] eV, order 2, U=1.0 eV, "
                                   "V sweep -1..1 V step 0.05"},
            "cpu_baseline": {"value": v, "unit": "IV points/s", "cores": nthr, "kind": "port", "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "IV points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    ap.add_argument("--ref-sample", type=int, default=4096)
    ap.add_argument("--n-omega", type=int, default=N_OMEGA, help="smaller grids for profiling only")
    ap.add_argument("--nhist", type=int, default=16, help="smaller histories for profiling only")
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

    def run_arm(precision):
        """warm-up + timed IV points of one solver form; the two forms do not fit in HBM
        together, so each arm creates and releases its own solver"""
        solver = qb.Solver(m, precision=precision, device=local, alpha_mix=0.5, nhist=args.nhist, tolf=1e-6,
                           maxscf=300, single_history=1)
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
        dev_s, n_conv, iters, mixed_steps, currents = 0.0, 0, [], [], []
        wall0 = time.perf_counter()
        for k in range(args.warmup, args.warmup + args.steps):
            r = solver.solve_scf(seq[k], fresh[k] or not prev_ok)
            prev_ok = r["converged"]
            dev_s += r["seconds"]
            n_conv += int(r["converged"])
            iters.append(r["n_iter"])
            mixed_steps.append(r["n_mixed"])
            currents.append(solver.current(seq[k]))
            solver.observables()  # G_less_obs, dosd, trU, trD back to host buffers
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        out = dict(launches=qb.kernel_launches() - l0, prof=solver.profile(False), clk=clocks.stop(), iters=iters,
                   mixed_steps=mixed_steps, currents=currents, nA=solver.nA, Nf=solver.Nf, n_vec=solver.n_vec)
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
    launches, clk, iters = head["launches"], head["clk"], head["iters"]
    prof = (f64 or head)["prof"]
    if rank == 0:
        points = args.steps * world
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
        # DRAM bytes per energy measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on
        # the 120x120 helix with 1024 energies (profiles/dyson_bgj_helix120_n1024.md,
        # profiles/keldysh_tc_helix120_n1024.md); the traffic of a launch is per energy, so it
        # scales with the number of energies
        traffic_per_energy = {"dyson_gj": (236.776192e6 + 183.729152e6) / 1024,
                              "keldysh_scf2": (1064.643e6 + 800.101376e6) / 1024}
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
            tpe = traffic_per_energy.get(fam) if (N, nA) == (120, 120) else None
            roof = {"kernel": fam, "bound": kind, "achieved": achieved, "peak": peak, "unit": unit,
                    "frac": achieved / peak, "traffic": tpe * n if tpe else None,
                    "traffic_note": "DRAM bytes per launch, ncu capture at 1024 energies scaled to the launch" if tpe else None,
                    "peak_source": src_note,
                    "per_launch_work": per_launch, "launches": cnt, "avg_launch_ms": ms / cnt}
        prec_name = "mixed" if "mixed" in arms else "fp64"
        line = {
            "metric": "converged IV points/s", "value": n_conv / dev_s if dev_s > 0 else 0.0,
            "unit": "IV points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if prec_name == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"helix {ions}x{turns} ({N}x{N} complex), {n} energies on [-12,12] eV, order 2, U=1.0 eV, "
                                   "V sweep -1..1 V step 0.05 with continuation", "precision": prec_name, "nhist": args.nhist,
                       "parallelism": f"replicas x{world}", "l2": "working set ~147 GB >> L2 (no flush needed)",
                       "scf_steps_per_point": iters, "converged_points": n_conv},
            "e2e": {"value": n_conv / wall if wall > 0 else 0.0, "unit": "IV points/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": obs_bytes},
            "gpu_launches": launches,
            "kernel_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1]},
            "roofline": roof,
            "clocks": clk,
            "currents_A": [list(c) for c in head["currents"]],
        }
        if "mixed" in arms:
            line["config"]["mixed"] = ("Sigma2 FFTs, 2x2 algebra and spectra in FP32 while max|F| > max(1e-5, 100 tolf) "
                                       "(the FP32 noise floor is ~1e-5); then FP64 steps until an FP64 residual meets "
                                       "tolf; Dyson/Keldysh, Broyden and observables FP64")
            line["config"]["fp32_steps_per_point"] = head["mixed_steps"]
        if f64 is not None and "mixed" in arms:
            j64, jmx = np.array(f64["currents"]), np.array(head["currents"])
            line["fp64"] = {"value": f64["value"], "e2e": f64["e2e"], "ms_per_step": 1000.0 * f64["dev_s"] / args.steps,
                            "scf_steps_per_point": f64["iters"], "kernel_ms": {k: round(v[0], 3) for k, v in
                                                                               f64["prof"].items() if v[1]}}
            line["mixed_over_fp64"] = head["value"] / f64["value"] if f64["value"] > 0 else None
            line["current_rel_err_vs_fp64"] = float(np.max(np.abs(jmx - j64)) / np.max(np.abs(j64)))
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
            line["cpu_baseline"] = cpu_baseline_sample(args.ref_sample)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
