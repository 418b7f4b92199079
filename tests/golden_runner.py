"""Golden-file runner: the reference's tests/run_tests.f90 restated for pytest.

For a case listed in tests/golden/cases.txt, the case files are copied into a work
directory, the program runs there, its exit code is checked, and every reference file
is compared number by number: |new - ref| <= tol_abs + tol_rel*|ref| with
tol_abs = 1e-6, tol_rel = 1e-5 (tests/run_tests.f90:14,48-49,224). Non-numeric fields
are skipped, as the reference's runner does.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
GOLDEN_SANCHO = os.path.join(GOLDEN, "sancho")  # SANCHO's suite (SANCHO/tests), same runner and tolerances
TOL_ABS, TOL_REL = 1e-6, 1e-5


def cases(root=GOLDEN):
    out = []
    for line in open(os.path.join(root, "cases.txt")):
        line = line.strip()
        if not line or line.startswith("#"):
            continue
        parts = line.split()
        out.append((parts[0], int(parts[1]), parts[2:]))
    return out


def _fields(path):
    rows = []
    for line in open(path):
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        rows.append(s.split())
    return rows


def _num(tok):
    try:
        return float(tok.replace("D", "E").replace("d", "e"))
    except ValueError:
        return None


def compare_files(new, ref, ta=TOL_ABS, tr=TOL_REL):
    """Returns (ok, worst |diff|, message)."""
    if not os.path.exists(new):
        return False, float("inf"), f"missing output {new}"
    a, b = _fields(new), _fields(ref)
    if len(a) != len(b):
        return False, float("inf"), f"{new}: {len(a)} data lines, expected {len(b)}"
    worst, bad = 0.0, []
    for ln, (ra, rb) in enumerate(zip(a, b), 1):
        if len(ra) != len(rb):
            return False, float("inf"), f"{new} line {ln}: {len(ra)} columns, expected {len(rb)}"
        for col, (x, y) in enumerate(zip(ra, rb), 1):
            xv, yv = _num(x), _num(y)
            if xv is None or yv is None:
                continue
            d = abs(xv - yv)
            worst = max(worst, d)
            if d > ta + tr * abs(yv):
                bad.append(f"line {ln} col {col}: {xv!r} vs ref {yv!r}")
    return (not bad), worst, "; ".join(bad[:3])


def run_case(exe, case, workroot, env=None, timeout=600, root=GOLDEN):
    """Copy the case, run `exe` in it. Returns (exit code, work dir)."""
    src = os.path.join(root, "cases", case)
    work = os.path.join(workroot, case)
    if os.path.isdir(work):
        shutil.rmtree(work)
    os.makedirs(work)
    for f in os.listdir(src):
        p = os.path.join(src, f)
        if os.path.isfile(p):
            shutil.copy(p, work)
    e = dict(os.environ)
    if env:
        e.update(env)
    with open(os.path.join(work, "stdout.txt"), "w") as out:
        r = subprocess.run([exe, work], stdout=out, stderr=subprocess.STDOUT, env=e, timeout=timeout)
    return r.returncode, work


def check_case(exe, case, rc_expected, refs, workroot, env=None, root=GOLDEN):
    rc, work = run_case(exe, case, workroot, env, root=root)
    msgs = []
    ok = rc == rc_expected
    if not ok:
        msgs.append(f"exit code {rc}, expected {rc_expected} (see {work}/stdout.txt)")
    worst = {}
    for r in refs:
        good, w, m = compare_files(os.path.join(work, r), os.path.join(root, "cases", case, "reference", r))
        worst[r] = w
        if not good:
            ok = False
            msgs.append(m)
    return ok, worst, "; ".join(msgs), work
