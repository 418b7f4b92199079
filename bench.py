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

Default: the FP64 form (the headline value), then the mixed form beside it with its ratio
and the error of every observable against the FP64 one over the points both converged;
the CPU oracle on a bounded sample of the same sweep; then a serving stream (p50/p99
latency of IV-point requests through qs_server). --case sancho / cfg2 / cfg4 run the other
workloads (their lines name them).

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


def finite(obj):
    """The line's values with every non-finite float replaced by None (strict JSON)."""
    if isinstance(obj, dict):
        return {k: finite(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [finite(v) for v in obj]
    if isinstance(obj, (float, np.floating)):
        return float(obj) if np.isfinite(obj) else None
    if isinstance(obj, np.integer):
        return int(obj)
    return obj


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# Broyden settings of the workload: the reference's input defaults (src/input_output.f90:
# 109-114). Both arms and every form use them.
BROYDEN = dict(alpha_mix=0.5, nhist=16, tolf=1e-6, maxscf=300, single_history=1)
# energies of the CPU sample: 1/16 of the grid (every part of an SCF iteration, residual
# and Broyden update, does the same work per energy)
SAMPLE_N = 1024
# SCF iterations per voltage of this sweep in the FP64 form on B200 (all 41 voltages, swept
# -1 -> 1 V with continuation, fresh after an unconverged voltage, maxscf 300; one B200, the
# default Broyden settings; -0.75 ... +0.20 V from the bench's own run with 5 warm-up and 20
# timed points); 300 marks a voltage that did not converge. The CPU arm multiplies
# its measured time per iteration by this work (the oracle runs the same algorithm, so the same
# iterations).
SWEEP_ITERS_B200 = dict(zip(VOLTS, [32, 27, 27, 26, 25, 25, 24, 23, 22, 21, 20, 19, 18, 16, 17, 19, 23, 24, 110, 245,
                                    300, 300, 300, 300, 300, 300, 210, 16, 18, 20, 23, 25, 26, 27, 28, 27, 28, 29,
                                    30, 30, 31]))


def bench_config(n_omega, ions, turns, nhist, world):
    """The static description of the workload, identical in every arm's line."""
    N = 2 * ions * turns
    b = dict(BROYDEN, nhist=nhist)
    return {"workload": f"helix {ions}x{turns} ({N}x{N} complex), {n_omega} energies on [-12,12] eV, order 2, "
                        "U=1.0 eV, lambda=0.01 eV, Gamma_L=Gamma_R=0.5 eV, T=300 K; V sweep -1..1 V step 0.05 "
                        "with continuation; the first W voltages warm up, the next K are timed",
            "broyden": {"alpha_mix": b["alpha_mix"], "nhist": b["nhist"], "history": "single" if b["single_history"]
                        else "double", "tolf": b["tolf"], "maxscf": b["maxscf"]},
            "forms": "FP64 GPU form (headline), then the mixed form (under \"mixed\")",
            "parallelism": f"replicas x{world}", "l2": "working set ~147 GB >> L2 126 MB (no flush needed)"}


def _oracle(threads):
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    return oracle_py


def cpu_iteration_times(V, n_keep, n_sample=SAMPLE_N, threads=None, ions=N_IONS, turns=N_TURNS):
    """Wall times of n_keep SCF iterations of the CPU oracle (oracle/oracle_py.py: the model
    built in numpy, only liboracle.so loaded) on the same helix, window and Broyden settings
    with n_sample energies, counting only iterations with a full history (the steady state
    of a solve); tolf = 0, so every iteration does its whole work."""
    op = _oracle(threads)
    m = op.Helix(ions, turns, PITCH * turns * (ions - 1) / ions, RADIUS, 1.0, 0.0, 1.0, 0.01, 1.0, 0.5, 0.5, 0.5, 300.0,
                 0.0, W_LO, (W_HI - W_LO) / n_sample, n_sample)
    nh_full, times = BROYDEN["nhist"], []
    for _ in range(4):  # a solve that runs away ends early: start again
        s = op.Solver(m, **dict(BROYDEN, tolf=0.0, maxscf=nh_full + 3 + n_keep - len(times)))
        r, dt = s.solve_timed(V, True)
        s.close()
        times += [t for t, step in zip(dt, r["log"]) if step[3] == nh_full]
        if len(times) >= n_keep:
            break
    return times[:n_keep]


def iters_per_converged_point(volts, iters, converged):
    """SCF iterations the sweep spent per converged IV point over `volts`."""
    it = sum(iters[V] for V in volts)
    conv = sum(int(converged[V]) for V in volts)
    return it / conv if conv else 0.0


def model_cfg0(qb, n_omega=4096):
    """The CPU-runnable configuration: 4 sites/turn x 2 turns (16 x 16 H), U = 0.5 eV, 4096
    energies on [-10, 10] eV, Broyden mixing 0.1 and tolf 1e-8 (reference history otherwise)."""
    args = dict(N_ions=4, N_turns=2, hel_length=PITCH * 2 * 3 / 4, hel_radius=RADIUS, hand=1.0, E_CC=0.0, t_hop=1.0,
                lamb=0.01, U_int=0.5, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0)
    ev = np.linalg.eigvalsh(qb.Model.helix(dw=1.0, up=1.0, delta=0.1, **args).H)
    delta = 20.0 / n_omega
    m = qb.Model.helix(dw=ev[0] + 10.0, up=10.0 - ev[-1] + 0.5 * delta, delta=delta, **args)
    assert m.n_omega == n_omega, m.n_omega
    return m


HARTREE = 27.211386245988  # eV; the DFTB+ files hold H0 in Hartree (src/hamiltonian.f90:612)


def _dftb_square(path, A):
    """A DFTB+ square matrix file as read by read_dftb_square (src/hamiltonian.f90:556-609)."""
    n = A.shape[0]
    with open(path, "w") as f:
        f.write(f"#      REAL   NALLORB   NKPOINT\n          T {n:9d}         1\n#   IKPOINT\n          1\n# MATRIX\n")
        for row in A:
            f.write(" ".join(f"{v:.17e}" for v in row) + "\n")


def make_cfg2_case(path, n_omega=32768, seed=40):
    """The synthetic helicene-like molecule of the multi-orbital configuration, written as a
    dftb_hs case (hamiltonian = dftb_hs; seeded): 28 C (s, py, pz, px) on a helix of 6 atoms
    a turn (radius 0.14 nm, 0.35 nm a turn) and 12 H (s) on every other C, 0.11 nm further out
    (124 orbitals, 248 spin-orbitals). H0: on-site -6 eV (C s), 0 eV (C p), -2 eV (H s);
    Slater-Koster-like hoppings -2.5 eV exp(-(r - 0.14 nm)/0.1 nm) times the direction cosines
    of the p orbitals involved, within 0.45 nm, plus N(0, 0.05 eV) noise; written in Hartree.
    S = I + P with P symmetric, ||P||_2 = 0.08 (so S is positive definite). p-shell SOC
    xi = 0.00849 eV in the dual form. U = 0.8 eV on the 64 orbitals of C1..C15 and C28 (the two
    contact atoms included, so the active block is 128 spin-orbitals), 0 elsewhere. Leads on
    C1 (left) and C28 (right). The grid spans the spectrum +-1 eV with n_omega points."""
    rng = np.random.default_rng(seed)
    os.makedirs(path, exist_ok=True)
    nC, nH = 28, 12
    th = 2 * np.pi * np.arange(nC) / 6
    posC = np.stack([0.14 * np.cos(th), 0.14 * np.sin(th), 0.35 * np.arange(nC) / 6], axis=1)
    hC = np.arange(0, 2 * nH, 2)  # C atoms carrying an H
    posH = np.stack([0.25 * np.cos(th[hC]), 0.25 * np.sin(th[hC]), posC[hC, 2]], axis=1)
    pos = np.vstack([posC, posH])
    elem = ["C"] * nC + ["H"] * nH
    orb = []  # (atom, kind) with kind 0 = s, 1..3 = py, pz, px
    for a, e in enumerate(elem):
        orb += [(a, 0)] + ([(a, 1), (a, 2), (a, 3)] if e == "C" else [])
    No = len(orb)
    H0 = np.zeros((No, No))
    for i, (a, ka) in enumerate(orb):
        H0[i, i] = (-6.0 if ka == 0 else 0.0) if elem[a] == "C" else -2.0
    dirc = {1: 1, 2: 2, 3: 0}  # py, pz, px -> y, z, x
    for i, (a, ka) in enumerate(orb):
        for j, (b, kb) in enumerate(orb):
            if j <= i or a == b:
                continue
            d = pos[b] - pos[a]
            r = np.linalg.norm(d)
            if r > 0.45:
                continue
            l = d / r
            f = (1.0 if ka == 0 else l[dirc[ka]]) * (1.0 if kb == 0 else -l[dirc[kb]])
            t = -2.5 * np.exp(-(r - 0.14) / 0.1) * f + rng.normal(0.0, 0.05)
            H0[i, j] = H0[j, i] = t
    P = rng.standard_normal((No, No))
    P = P + P.T
    S = np.eye(No) + 0.08 * P / np.linalg.norm(P, 2)
    _dftb_square(os.path.join(path, "hamsqr1.dat"), H0 / HARTREE)
    _dftb_square(os.path.join(path, "oversqr.dat"), S)
    with open(os.path.join(path, "molecule.xyz"), "w") as f:
        f.write(f"{len(elem)}\nsynthetic helicene-like molecule [Angstrom]\n")
        for e, p in zip(elem, pos):
            f.write(f"{e} {10 * p[0]:.8f} {10 * p[1]:.8f} {10 * p[2]:.8f}\n")
    inter = set(range(15)) | {27}
    with open(os.path.join(path, "U_per_orbital.dat"), "w") as f:
        for a, _ in orb:
            f.write(f"{0.8 if a in inter else 0.0}\n")

    def write_input(dw, up, delta, mu=0.0):
        with open(os.path.join(path, "input.dat"), "w") as f:
            f.write("hamiltonian = dftb_hs\nham_file = hamsqr1.dat\noverlap_file = oversqr.dat\n"
                    "xyz_file = molecule.xyz\nmax_angular_momentum = C:p H:s\nsoc_xi = C:0.00849\n"
                    "soc_form = dual\nlead_left_atoms = 1\nlead_right_atoms = 28\nhubbard_file = U_per_orbital.dat\n"
                    f"T = 300.d0\nV = 0.1d0\nVf = 0.3d0\ndelv = 0.1d0\nmu = {float(mu)!r}\norder = 2\nU_int = 0.8d0\n"
                    f"GammaL_up = 0.5d0\nGammaL_down = 0.5d0\nGammaR = 0.5d0\ndw = {float(dw)!r}\n"
                    f"up = {float(up)!r}\ndelta = {float(delta)!r}\n")
    write_input(1.0, 1.0, 0.05)
    return write_input


def model_cfg2(qb, path, n_omega):
    """The cfg2 case loaded through the host layer, its grid fitted to n_omega points, with mu
    in the middle of the widest gap between the spin-orbital levels within 20 of half filling
    (the synthetic molecule's spectrum is dense there: 30-180 meV spacings)."""
    write_input = make_cfg2_case(path, n_omega)
    ev = np.sort(qb.Model.load(path).Ev)
    delta = (ev[-1] - ev[0] + 2.0) / n_omega
    half = len(ev) // 2
    k = half - 20 + int(np.argmax(np.diff(ev[half - 20:half + 21])))
    write_input(1.0, 1.0 + 0.5 * delta, delta, mu=0.5 * (ev[k] + ev[k + 1]))
    m = qb.Model.load(path)
    assert m.n_omega == n_omega, m.n_omega
    return m


CFG0_BROYDEN = dict(alpha_mix=0.1, nhist=16, tolf=1e-8, maxscf=300, single_history=1)
CFG0_VOLTS = [round(0.1 * k, 10) for k in range(11)]


def cfg0_sweep(solver):
    """The cfg0 sweep V = 0..1 V step 0.1 with continuation: per-point converged flag,
    iterations, currents, wall time of the sweep."""
    out, ok = [], False
    t0 = time.perf_counter()
    for k, V in enumerate(CFG0_VOLTS):
        r = solver.solve_scf(V, k == 0 or not ok)
        ok = r["converged"]
        out.append((ok, r["n_iter"], solver.current(V)))
    return out, time.perf_counter() - t0


def cpu_baseline_line(qb, V, n_keep, ions, turns, device, iters_per_point, ipp_note):
    """cpu_baseline of the GPU arm's line: (1) the CPU oracle's time per SCF iteration on a
    1/16 sample of this workload (as in the reference arm), times the SCF iterations per
    converged IV point of this run's FP64 sweep; (2) real, unscaled converged IV points of the
    CPU-runnable configuration (the 4 x 2 helix, 4096 energies, V = 0..1 V) on the CPU oracle
    and on the GPU's FP64 form in the same run."""
    nthr = os.cpu_count()
    times = cpu_iteration_times(V, n_keep, SAMPLE_N, threads=nthr, ions=ions, turns=turns)
    t_it = float(np.mean(times)) * N_OMEGA / SAMPLE_N
    v = 1.0 / (t_it * iters_per_point) if times and iters_per_point > 0 else 0.0
    op = _oracle(nthr)
    mq = model_cfg0(qb)
    mo = op.Helix(4, 2, PITCH * 2 * 3 / 4, RADIUS, 1.0, 0.0, 1.0, 0.01, 0.5, 0.5, 0.5, 0.5, 300.0, 0.0, mq.w_init,
                  mq.delta, mq.n_omega)
    so = op.Solver(mo, **CFG0_BROYDEN)
    cpu_pts, cpu_s = cfg0_sweep(so)
    so.close()
    sg = qb.Solver(mq, device=device, **CFG0_BROYDEN)
    gpu_pts, gpu_s = cfg0_sweep(sg)
    sg.close()
    jc = np.array([p[2] for p in cpu_pts])
    jg = np.array([p[2] for p in gpu_pts])
    both = [k for k in range(len(CFG0_VOLTS)) if cpu_pts[k][0] and gpu_pts[k][0]]
    cc, gc = sum(int(p[0]) for p in cpu_pts), sum(int(p[0]) for p in gpu_pts)
    return {"value": v, "unit": "IV points/s", "cores": nthr, "kind": "port",
            "sample": f"CPU oracle (OpenMP over energies, OpenBLAS zgetrf/zgetri/dposv, radix-4 FFT; oracle/) on "
                      f"{nthr} threads: {len(times)} SCF iterations (residual + Broyden update, full 16-column history) "
                      f"of the same helix on {SAMPLE_N} of the 16384 energies, {np.mean(times):.3f} s each, x16 = "
                      f"{t_it:.2f} s per full iteration; x {iters_per_point:.1f} SCF iterations per converged IV point "
                      f"({ipp_note}); the initial and final sweeps of a point are not counted (in the CPU's favour)",
            "seconds_per_iteration": t_it, "iterations_per_converged_point": iters_per_point,
            "cfg0_real_sweep": {
                "workload": "4x2 helix (16x16), U=0.5 eV, 4096 energies on [-10,10] eV, V 0..1 V step 0.1 with "
                            "continuation, alpha_mix 0.1, tolf 1e-8, 16-column single-precision history",
                "cpu": {"converged": cc, "wall_s": cpu_s, "value": cc / cpu_s if cpu_s > 0 else 0.0,
                        "scf_steps_per_point": [p[1] for p in cpu_pts], "cores": nthr},
                "gpu_fp64": {"converged": gc, "wall_s": gpu_s, "value": gc / gpu_s if gpu_s > 0 else 0.0,
                             "scf_steps_per_point": [p[1] for p in gpu_pts]},
                "gpu_over_cpu": (gc / gpu_s) / (cc / cpu_s) if cc and gpu_s > 0 else None,
                "current_max_diff_rel": float(np.max(np.abs(jg[both] - jc[both])) / np.max(np.abs(jc[both])))
                if both else None}}


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
            "mean_queue_s": float(np.mean([r["t_start"] - r["t_arrival"] for r in ok])) if ok else None,
            "p50_service_s": float(np.percentile([r["t_done"] - r["t_start"] for r in ok], 50)) if ok else None,
            "p99_service_s": float(np.percentile([r["t_done"] - r["t_start"] for r in ok], 99)) if ok else None,
            "fp32_steps": int(sum(r["n_mixed"] for r in ok)), "scf_steps": int(sum(r["n_iter"] for r in ok)),
            "throughput_per_s": conv / span if span > 0 else 0.0, "span_s": span,
            "orbitals": [int(x[3]) for x in reqs]}


def run_reference(args, rank, world):
    """--impl reference: the oracle (a restatement of the reference's CPU path: OpenMP over
    energies, LAPACK zgetrf/zgetri/dposv from OpenBLAS, its own FFT; oracle/, which loads
    nothing of the product) on all host cores. Each step is a bounded sample of the workload:
    one SCF iteration (residual + Broyden update with the full history) of the same helix,
    window and settings on 1/16 of the energies, timed on its own. ms_per_step is that
    measured time; the value converts it into converged IV points per second of the workload
    with the x16 energy scale and the SCF iterations per converged point that the same sweep
    window takes (SWEEP_ITERS_B200, the same algorithm in FP64 on B200)."""
    if rank != 0:
        return 0
    nthr = os.cpu_count()
    ions, turns = (int(v) for v in args.helix.split("x"))
    seq = voltage_block(0, 1)[:args.warmup + args.steps]
    window = seq[args.warmup:]
    t0 = time.perf_counter()
    times = cpu_iteration_times(window[0], args.warmup + args.steps, args.ref_sample, threads=nthr, ions=ions,
                                turns=turns)
    timed = times[args.warmup:]
    t_step = float(np.mean(timed)) if timed else 0.0
    known = all(V in SWEEP_ITERS_B200 for V in window)
    ipp = iters_per_converged_point(window, SWEEP_ITERS_B200, {V: SWEEP_ITERS_B200[V] < BROYDEN["maxscf"]
                                                                for V in window}) if known else 0.0
    scale = N_OMEGA / args.ref_sample
    v = 1.0 / (t_step * scale * ipp) if known and timed and 0 < ipp < float("inf") else 0.0
    desc = (f"CPU oracle (OpenMP over energies, OpenBLAS zgetrf/zgetri/dposv, radix-4 FFT; oracle/) on {nthr} threads: "
            f"each step one SCF iteration (residual + Broyden update, full 16-column history) of the same helix on "
            f"{args.ref_sample} of the 16384 energies ({t_step:.3f} s); value = 1 / (step x {scale:g} energies x "
            f"{ipp:.1f} SCF iterations per converged IV point of voltages {window[0]:g}..{window[-1]:g}, measured on "
            f"B200 with the same algorithm)")
    line = {"metric": "converged IV points/s", "value": v, "unit": "IV points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": bench_config(args.n_omega, ions, turns, args.nhist, world),
            "cpu_baseline": {"value": v, "unit": "IV points/s", "cores": nthr, "kind": "port", "sample": desc,
                             "seconds_per_full_iteration": t_step * scale, "iterations_per_converged_point": ipp},
            "e2e": {"value": v, "unit": "IV points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "run_s": time.perf_counter() - t0}
    print(json.dumps(finite(line), allow_nan=False), flush=True)
    return 0


def run_case(args, device):
    """--case cfg2 / cfg4: the FP64 and mixed forms on a short sweep with continuation of the
    multi-orbital molecule (make_cfg2_case: N = 248, nA = 128, 16384 energies instead of 32768,
    8-column history) or of the 16 x 8 helix (N = nA = 256, lambda = 0.02 eV, U = 1.0 eV, 4096
    energies on [-15, 15] eV instead of 65536, 4-column history): the full sizes need more
    than one B200's HBM in FP64 (the SCF vectors and Broyden history alone exceed 180 GB)."""
    import tempfile

    import quichotte_b200 as qb
    if args.case == "cfg2":
        m = model_cfg2(qb, tempfile.mkdtemp(prefix="qs_cfg2_"), 16384)
        nh, volts = 8, [0.1, 0.2, 0.3]
        workload = ("synthetic 40-atom helicene-like molecule (28 C s,p + 12 H s; 248 spin-orbitals), dftb_hs form "
                    "(S = I + P, ||P|| = 0.08; SOC xi = 0.00849 eV dual), U = 0.8 eV on 64 C orbitals (nA = 128), "
                    "16384 energies over the spectrum +-1 eV; deviation: 16384 energies instead of 32768 and an "
                    "8-column history (the full grid needs > 180 GB in FP64)")
    else:
        args4 = dict(N_ions=16, N_turns=8, hel_length=PITCH * 8 * 15 / 16, hel_radius=RADIUS, hand=1.0, E_CC=0.0,
                     t_hop=1.0, lamb=0.02, U_int=1.0, GammaL_up=0.5, GammaL_down=0.5, GammaR=0.5, T=300.0, mu=0.0)
        ev = np.linalg.eigvalsh(qb.Model.helix(dw=1.0, up=1.0, delta=0.1, **args4).H)
        n = 4096
        delta = 30.0 / n
        m = qb.Model.helix(dw=ev[0] + 15.0, up=15.0 - ev[-1] + 0.5 * delta, delta=delta, **args4)
        nh, volts = 4, [-1.0, -0.95, -0.9]
        workload = ("helix 16x8 (256x256 complex), lambda = 0.02 eV, U = 1.0 eV, 4096 energies on [-15,15] eV; "
                    "deviation: 4096 energies instead of 65536 and a 4-column history (the full grid's SCF vectors "
                    "alone are 4 x 103 GB), voltages solved one after another with continuation")
    settings = dict(BROYDEN, nhist=nh)
    out = {}
    for prec, name in ((qb.QS_PREC_FP64, "fp64"), (qb.QS_PREC_MIXED, "mixed")):
        s = qb.Solver(m, precision=prec, device=device, **settings)
        s.profile(True)
        pts, ok, dev = [], False, 0.0
        t0 = time.perf_counter()
        for k, V in enumerate(volts):
            r = s.solve_scf(V, k == 0 or not ok)
            ok = r["converged"]
            dev += r["seconds"]
            o = s.observables()
            pts.append(dict(V=V, converged=ok, n_iter=r["n_iter"], n_mixed=r["n_mixed"], J=s.current(V),
                            occ=np.imag(np.diag(o["G_less_obs"])).copy(), G=o["G_less_obs"], dosd=o["dosd"]))
        wall = time.perf_counter() - t0
        prof = s.profile(False)
        out[name] = dict(points=pts, dev_s=dev, wall_s=wall, gib=s.device_gib(), nA=s.nA,
                         kernel_ms={k: round(v[0], 3) for k, v in prof.items() if v[1]})
        s.close()
    f64, mix = out["fp64"], out["mixed"]
    conv = lambda a: sum(int(p["converged"]) for p in a["points"])
    line = {"metric": "converged IV points/s", "value": conv(mix) / mix["dev_s"] if mix["dev_s"] > 0 else 0.0,
            "unit": "IV points/s", "n_gpus": 1, "steps": len(volts), "warmup": 0, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic", "case": args.case,
            "config": {"workload": workload, "N": m.Norb, "nA": f64["nA"], "n_omega": m.n_omega, "nhist": nh,
                       "voltages": volts},
            "fp64": {"value": conv(f64) / f64["dev_s"] if f64["dev_s"] > 0 else 0.0, "device_s": f64["dev_s"],
                     "converged": [p["converged"] for p in f64["points"]],
                     "scf_steps_per_point": [p["n_iter"] for p in f64["points"]], "device_gib": f64["gib"],
                     "kernel_ms": f64["kernel_ms"]},
            "mixed": {"value": conv(mix) / mix["dev_s"] if mix["dev_s"] > 0 else 0.0, "device_s": mix["dev_s"],
                      "converged": [p["converged"] for p in mix["points"]],
                      "scf_steps_per_point": [p["n_iter"] for p in mix["points"]],
                      "fp32_steps_per_point": [p["n_mixed"] for p in mix["points"]], "kernel_ms": mix["kernel_ms"]},
            "mixed_over_fp64": (conv(mix) / mix["dev_s"]) / (conv(f64) / f64["dev_s"]) if conv(f64) and conv(mix)
            else None,
            "err_vs_fp64": observable_errors(f64["points"], mix["points"]),
            "currents_A": [list(p["J"]) for p in f64["points"]]}
    print(json.dumps(finite(line), allow_nan=False), flush=True)
    return 0


SANCHO_CHAIN = dict(N_sites=10, E_CC=2.0, t_hop=-0.4, U_int=0.5, GammaL=1.0, GammaR=1.0, T=300.0, mu=2.0, dw=1.0,
                    up=1.0, delta=0.004, order=3)
SANCHO_VOLTS = [-0.5, -0.25, 0.0, 0.25, 0.5]


def sancho_input(path, chain, volts):
    """SANCHO's input.dat for the chain (the keys of SANCHO/src/input_output.f90:28-104) and
    the voltage sweep volts[0] .. volts[-1]"""
    os.makedirs(path, exist_ok=True)
    keys = dict(chain, V=volts[0], Vf=volts[-1], delv=volts[1] - volts[0], alpha_mix=0.3, nhist=8, maxscf=200,
                tolf=1e-6)
    with open(os.path.join(path, "input.dat"), "w") as f:
        for k, v in keys.items():
            f.write(f"{k} = {v}\n")
    return path


def run_sancho(args, device):
    """--case sancho: SANCHO's order-3 chain (10 sites, 883 energies, U 0.5 eV; SANCHO's
    regression case scaled up: the same chain, a finer grid and more sites) swept over five
    voltages with continuation on the B200 solver (include/qsa200.h), its kernel families
    against the FP64 roofline, and the CPU oracle's time per SCF iteration of the same sweep."""
    import tempfile

    import quichotte_b200 as qb
    import sancho_b200 as sb
    d = sancho_input(tempfile.mkdtemp(prefix="qs_sancho_"), SANCHO_CHAIN, SANCHO_VOLTS)
    m = sb.SanchoModel.load(d)
    s = sb.SanchoSolver(m, device=device)
    # warm-up: one fresh solve (module load, first launches)
    s.solve_scf(SANCHO_VOLTS[0], True)
    s.profile(True)
    l0 = qb.kernel_launches()
    pts, ok, wall = [], False, 0.0
    for k, V in enumerate(SANCHO_VOLTS):
        t = time.perf_counter()
        r = s.solve_scf(V, k == 0 or not ok)
        J = s.current(V)
        s.observables()
        wall += time.perf_counter() - t
        ok = r["converged"]
        pts.append(dict(V=V, converged=ok, n_iter=r["n_iter"], J=J))
    prof = s.profile(False)
    launches = qb.kernel_launches() - l0
    n_it = sum(p["n_iter"] for p in pts)
    conv = sum(int(p["converged"]) for p in pts)
    Na, n = m.N_sites, m.n_omega
    # algorithmic FP64 work per SCF iteration of the direct sums (complex MAC = 8 flops):
    # chi and phi 6 MACs per (element, output, summand) over n^2 (output, summand) pairs each,
    # the particle-hole and particle-particle convolutions 3 MACs each
    fl_bub = 2 * 6 * 8 * Na * Na * n * n
    fl_sig = 2 * 3 * 8 * Na * Na * n * n
    ms_bub, ms_sig = prof["bubbles"][0], prof["sigma"][0]
    peak = 37.0  # TFLOP/s, B200 FP64 (nominal; the measured peaks hold no FP64 figure)
    achieved = fl_bub * n_it / (ms_bub * 1e-3) / 1e12 if ms_bub > 0 else 0.0
    # CPU: the oracle's time per SCF iteration (one residual of the same chain at the first voltage)
    cpu = {}
    if not args.no_cpu_baseline:
        op = _oracle(os.cpu_count())
        om = op.SanchoChain(**SANCHO_CHAIN)
        o = op.SanchoSolver(om)
        x = o.initial_vector(SANCHO_VOLTS[0])
        t = time.perf_counter()
        o.residual(SANCHO_VOLTS[0], x)
        t_it = time.perf_counter() - t
        cpu = {"value": conv / (t_it * n_it) if t_it > 0 else 0.0, "unit": "IV points/s", "cores": os.cpu_count(),
               "kind": "port", "seconds_per_scf_iteration": t_it,
               "sample": f"one scf_residual of the same chain (OpenMP over elements) x {n_it} SCF iterations "
                         "the B200 sweep took"}
    line = {"metric": "converged IV points/s", "value": conv / wall if wall > 0 else 0.0, "unit": "IV points/s",
            "n_gpus": 1, "steps": len(SANCHO_VOLTS), "warmup": 1, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "case": "sancho",
            "config": {"workload": f"SANCHO chain, {Na} sites, order 3, {n} energies (delta 0.004 eV), U 0.5 eV, "
                                   "E_CC 2 eV, t -0.4 eV, Gamma 1 eV, T 300 K, mu 2 eV; V -0.5..0.5 step 0.25 with "
                                   "continuation; alpha_mix 0.3, nhist 8, tolf 1e-6 (SANCHO's defaults)"},
            "scf_iterations": [p["n_iter"] for p in pts], "converged": [p["converged"] for p in pts],
            "currents": [p["J"] for p in pts], "seconds_per_scf_iteration": wall / max(n_it, 1),
            "kernel_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1]}, "gpu_launches": launches,
            "roofline": {"kernel": "sa_bubbles (chi + phi)", "bound": "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "peak_kind": "nominal",
                         "flop_per_iteration": fl_bub,
                         "sigma_tflops": fl_sig * n_it / (ms_sig * 1e-3) / 1e12 if ms_sig > 0 else 0.0},
            "cpu_baseline": cpu}
    print(json.dumps(finite(line), allow_nan=False), flush=True)
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
    Ev, _ = qb.hermitian_eigenvalues(m.H)
    return {"eigenvalues_ms": best(lambda: qb.hermitian_eigenvalues(m.H)),
            "eigenvalues_numpy_ms": best(lambda: np.linalg.eigvalsh(m.H)),
            "eigenvalues_rel_err": float(np.max(np.abs(Ev - np.linalg.eigvalsh(m.H))) / np.max(np.abs(Ev))),
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
        rep = 3
        calls = []
        for _ in range(rep):  # each call timed: the spread between calls of one size
            (H, _), t1 = wall(lambda: qb.dftb_lowdin(S, H0, Lam, True), 1)
            calls.append(t1)
        Hn, tc = wall(ref, rep)
        out[f"lowdin_N{N}"] = {"device_s": min(calls), "device_calls_s": calls, "numpy_s": tc,
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
    ap.add_argument("--cpu-iters", type=int, default=3, help="SCF iterations timed in the GPU arm's CPU sample")
    ap.add_argument("--n-omega", type=int, default=N_OMEGA, help="smaller grids for profiling only")
    ap.add_argument("--nhist", type=int, default=BROYDEN["nhist"], help="smaller histories for profiling only")
    ap.add_argument("--helix", default=f"{N_IONS}x{N_TURNS}", help="sites/turn x turns; other sizes for profiling only")
    ap.add_argument("--autotune", type=int, default=1,
                    help="1: time kernel variants per size (default); 2/3: force variant 1/2 (profiling only)")
    ap.add_argument("--serve", type=int, default=16,
                    help="requests of the serving stream (0: none; the full stream is 512)")
    ap.add_argument("--serve-rate", type=float, default=0.15,
                    help="Poisson arrivals per second (0.15: below the ~0.2/s the device serves with 4 solves in "
                         "flight, so the latencies are service times, not a growing queue)")
    ap.add_argument("--serve-inflight", type=int, default=4, help="solves on the device at once")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="both: the FP64 form (headline value), then the mixed form, with their ratio")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving stream (--serve requests at --serve-rate), FP64 then mixed, and print "
                         "its line")
    ap.add_argument("--case", default="cfg1", choices=["cfg1", "cfg2", "cfg4", "sancho"],
                    help="cfg1: the workload above (default); cfg2 / cfg4: the multi-orbital molecule and the "
                         "256-state helix at the reduced sizes one B200 holds (their line names the deviation); "
                         "sancho: SANCHO's order-3 chain on the B200 SANCHO solver")
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
    if args.case == "sancho":
        return run_sancho(args, local)
    if args.case != "cfg1":
        return run_case(args, local)
    if args.serve_only:
        import quichotte_b200 as qb
        line = {"metric": "served IV-point requests: p50/p99 latency and throughput", "case": "cfg3",
                "workload": (f"first {args.serve} of the seeded 512-request stream: random helices, sites/turn 3-12, "
                             "turns 1-8, U 0.2-1.5 eV, V -1..1 V, 4096-32768 energies on [-10,10] eV, Poisson "
                             f"arrivals at {args.serve_rate}/s, {args.serve_inflight} solves in flight; one fresh-start "
                             "IV point per request, Broyden nhist 8; requests above the HBM budget are refused")}
        for name, prec in (("fp64", qb.QS_PREC_FP64), ("mixed", qb.QS_PREC_MIXED)):
            line[name] = run_serving(qb, args.serve, args.serve_rate, args.serve_inflight, prec)
        print(json.dumps(finite(line), allow_nan=False), flush=True)
        return 0

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
    # the headline is the FP64 form (the reference's arithmetic); the mixed form stands beside it
    head = arms.get("fp64") or arms["mixed"]
    f64 = arms.get("fp64")
    mix = arms.get("mixed")
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
        # Broyden kernels per vector element (profiles/broyden_kernels_helix120_n1024.md)
        traffic_per_unit = {"dyson_gj": ((236.776192e6 + 183.729152e6) / 1024, n),
                            "keldysh_scf2": ((1064.643e6 + 800.101376e6) / 1024, n),
                            # hist_update_split + x_update + vec_norms of one step (history
                            # full) per SCF-vector element, averaged over the 3 launches
                            "broyden": ((4.072997376e9 + 0.356998144e9 + 3.539108352e9 + 0.344236544e9
                                         + 0.707824128e9) / (3 * 14400 * 1024) / 3, nvec)}
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
        prec_name = "fp64" if f64 is not None else "mixed"
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
            "fp32_steps_per_point": [p["n_mixed"] for p in pts] if prec_name == "mixed" else None,
            "e2e": {"value": n_conv / wall if wall > 0 else 0.0, "unit": "IV points/s", "h2d_bytes_per_step": 8,
                    "d2h_bytes_per_step": obs_bytes},
            "gpu_launches": launches,
            "kernel_ms": {k: round(v[0], 3) for k, v in prof.items() if v[1]},
            "roofline": roof,
            "clocks": clk,
            "currents_A": [list(p["J"]) for p in pts],
        }
        if mix is not None and f64 is not None:
            line["mixed"] = {
                "form": ("on fresh starts: Sigma2 FFTs, 2x2 algebra and spectra in FP32, and the Keldysh products on "
                         "the fastest of the 3xTF32 tensor-core kernel and the FP64 ones (autotuned), while max|F| is "
                         "above max(1e-5, 100 tolf) and still falling; then FP64 steps until an FP64 residual meets "
                         "tolf; continued starts FP64 throughout; Dyson, Broyden and observables FP64"),
                "value": mix["value"], "e2e": mix["e2e"], "ms_per_step": 1000.0 * mix["dev_s"] / args.steps,
                "converged": [bool(p["converged"]) for p in mix["points"]],
                "scf_steps_per_point": [p["n_iter"] for p in mix["points"]],
                "fp32_steps_per_point": [p["n_mixed"] for p in mix["points"]],
                "kernel_ms": {k: round(v[0], 3) for k, v in mix["prof"].items() if v[1]},
                "clocks": mix["clk"], "gpu_launches": mix["launches"],
                "over_fp64": mix["value"] / f64["value"] if f64["value"] > 0 else None,
                "err_vs_fp64": observable_errors(f64["points"], mix["points"])}
        if world == 1 and args.serve > 0:
            line["serving"] = run_serving(qb, args.serve, args.serve_rate, args.serve_inflight, qb.QS_PREC_FP64)
            line["serving"]["workload"] = (f"serving stream, first {args.serve} of the seeded 512-request stream: random "
                                           "helices, sites/turn 3-12, turns 1-8, U 0.2-1.5 eV, V -1..1 V, 4096-32768 "
                                           "energies, Poisson arrivals; one fresh-start IV point per request, FP64, "
                                           "Broyden nhist 8; requests above the HBM budget are refused")
        if world == 1:
            line["setup"] = setup_timing(qb, m)
        if world == 1 and not args.no_cpu_baseline:
            ref_pts = (f64 or head)["points"]
            its = sum(p["n_iter"] for p in ref_pts)
            conv = sum(int(p["converged"]) for p in ref_pts)
            ipp = its / conv if conv else 0.0
            line["cpu_baseline"] = cpu_baseline_line(
                qb, seq[args.warmup], args.cpu_iters, ions, turns, local, ipp,
                f"this run's {'FP64' if f64 else prec_name} sweep: {its} iterations, {conv} converged points")
        print(json.dumps(finite(line), allow_nan=False), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
