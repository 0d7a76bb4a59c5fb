"""Generate the test fixtures: key files and golden P(t) vectors.

    python tests/golden/make_fixtures.py            # key files only (no reference needed)
    python tests/golden/make_fixtures.py --golden   # + golden vectors from oracle/_ref

Key files (tests/golden/keys/) use the reference's key-file format
(etoheom-cpu/lib/param.cpp:102-332).  The ETO bath lines were fitted once with
eto-heom_b200/etofit.py (a restatement of etom/ohmic_ETOM.py) and are frozen below,
because curve_fit results move with the scipy version.

Interpretation recorded here: "2 ETO modes per site" = one fitted oscillator = two
BATH lines (+w, -w) per site, which reproduces the ADO counts 70 / 680 / 2925 / 210.
The "perturbative amplitude 1e-4 in dipole units" is E0 = 0.5308 cm^-1, so that
E0 * |mu| / hbar = 1e-4 fs^-1 for a unit dipole.

Golden vectors (tests/golden/ref/*.npz) are the reference's own code -- its
etoheom-cpu/lib sources compiled unmodified against the GSL-API shim
(oracle/Makefile `ref` target) and driven by oracle/ref_driver.cpp -- printed at
full precision.  Synthetic systems stand in for a public dataset (the reference
has none); every random choice comes from a fixed numpy seed.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KEYS = os.path.join(HERE, "keys")
REF = os.path.join(HERE, "ref")
ROOT = os.path.dirname(os.path.dirname(HERE))

# Frozen ETO fits (etofit.ohmic / etofit.superohmic, one oscillator -> two lines).
OHMIC_35_106_77K = ("0.006593820648078373", [
    "0.00010950 -0.00005111 0.02549399 0.00000001",
    "0.00010950 -0.00005111 0.02549399 -0.00000001"])
SUPEROHMIC_50_150_300K = ("0.009419743782969104", [
    "0.00019549 -0.00007598 0.04532376 0.08233007",
    "0.00019549 -0.00007598 0.04532376 -0.08233007"])
# The reference's own example bath (example/CPU_dimer_ohmic/key.key-tmpl:25-33).
REF_EXAMPLE_BATH = ("0.008995192714312095", [
    "0.00311213 -0.00252971 0.12340683 0.00000006",
    "0.00311213 -0.00252971 0.12340683 -0.00000006",
    "-0.00296194 0.00259667 0.12950563 0.02683512",
    "-0.00296194 0.00259667 0.12950563 -0.02683512",
    "0.00001177 -0.00003282 0.00754453 0.00000000",
    "0.00001177 -0.00003282 0.00754453 -0.00000000"])

E0 = "0.5308"


def key_text(size, K, L, H, bath, dipoles, pulses, time, n_sample=1, seed=7, sigma=None,
             single_manifold=False, extra=""):
    """Render a key file.  H is the single_size x single_size block in cm^-1."""
    sys_size = size if single_manifold else size + (size - 1) * (size - 2) // 2
    out = ["# synthetic fixture (tests/golden/make_fixtures.py)", "SIZE", str(size), ""]
    if single_manifold:
        out += ["MANIFOLD", "single", ""]
    out += ["HEOM", f"{K} {L}", "", "HAMILTONIAN"]
    out += [" ".join(f"{v:.10g}" for v in row) for row in H]
    out += ["", "DISORDER", f"{n_sample} {seed}"]
    sig = np.zeros((size, size)) if sigma is None else np.asarray(sigma)
    out += [" ".join(f"{v:.10g}" for v in row) for row in sig]
    out += [""] * (sys_size - size)  # the CPU parser reads sys_size rows (param.cpp:145)
    out += ["", "TEMPERATURE", "77", "", "BATH", bath[0], str(len(bath[1]))] + list(bath[1])
    out += ["", "DIPOLE", str(len(dipoles))]
    out += [f"{i} {j} {x:.10g} {y:.10g} {z:.10g}" for i, j, x, y, z in dipoles]
    out += ["", "POLARIZATION", "0 0 0 0", "", "PULSE", "3"]
    out += [f"{E0} {tau:g} {taup:g} {w:g}" for tau, taup, w in pulses]
    out += ["", "TIME", " ".join(f"{v:g}" for v in time)]
    if extra:
        out += ["", extra]
    return "\n".join(out) + "\n"


def dynamics_key_text(H, K, L, bath, time):
    """A population-dynamics key file (the format of param::param_dynamics,
    etoheom-cpu/lib/param.cpp:250-348: no ground state, no disorder, dipoles or pulses)."""
    out = ["# synthetic population-dynamics fixture (tests/golden/make_fixtures.py)", "SIZE", str(len(H)), "",
           "HEOM", f"{K} {L}", "", "HAMILTONIAN"]
    out += [" ".join(f"{v:.10g}" for v in row) for row in H]
    out += ["", "BATHTYPE", "ohmic", "", "TEMPERATURE", "77", "", "BATH", bath[0], str(len(bath[1]))] + list(bath[1])
    out += ["", "TIME ", " ".join(f"{v:g}" for v in time)]
    return "\n".join(out) + "\n"


def dimer_H():
    return [[0, 0, 0], [0, 12400, 100], [0, 100, 12600]]


def dimer_key(tau=(50, 150, 250), t_end=1000, dt=0.5, pstep=0.5, **kw):
    return key_text(3, 2, 4, dimer_H(), OHMIC_35_106_77K,
                    [(0, 1, 0.0, 0.0, 1.0), (0, 2, 0.0, 0.0, 1.0)],
                    [(t, 20, 12500) for t in tau], (0, t_end, dt, pstep), **kw)


def aggregate(n_sites, seed, e_mean, e_sd, j_max, e_fixed=None):
    rng = np.random.default_rng(seed)
    e = np.array(e_fixed, float) if e_fixed is not None else rng.normal(e_mean, e_sd, n_sites)
    H = np.zeros((n_sites + 1, n_sites + 1))
    for a in range(n_sites):
        H[a + 1, a + 1] = round(float(e[a]), 4)
    for a in range(n_sites):
        for b in range(a + 1, n_sites):
            j = round(float(rng.uniform(-j_max, j_max)), 4)
            H[a + 1, b + 1] = H[b + 1, a + 1] = j
    mu = rng.normal(0, 1, (n_sites, 3))
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    dip = [(0, a + 1, *map(float, np.round(mu[a], 6))) for a in range(n_sites)]
    return H.tolist(), dip


def chain(n_sites, seed, e_sd, j_nn):
    rng = np.random.default_rng(seed)
    e = rng.normal(12400, e_sd, n_sites)
    H = np.zeros((n_sites + 1, n_sites + 1))
    for a in range(n_sites):
        H[a + 1, a + 1] = round(float(e[a]), 4)
        if a + 1 < n_sites:
            H[a + 1, a + 2] = H[a + 2, a + 1] = j_nn
    mu = rng.normal(0, 1, (n_sites, 3))
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    return H.tolist(), [(0, a + 1, *map(float, np.round(mu[a], 6))) for a in range(n_sites)]


def scan_points(t0=50.0, t1_step=5.0, n_t1=64, t2_step=100.0, n_t2=8, t3=400.0):
    """The 2DES delay scan: (tau1, tau2, tau3, t_end, kind) for every point.
    Rephasing: pulse 1 first; non-rephasing: pulse 2 first (gen_2d_data.sh:37-61)."""
    pts = []
    for kind in ("R", "NR"):
        for i2 in range(n_t2):
            for i1 in range(n_t1):
                t1, t2 = i1 * t1_step, i2 * t2_step
                if kind == "R":
                    tau = (t0, t0 + t1, t0 + t1 + t2)
                else:
                    tau = (t0 + t1, t0, t0 + t1 + t2)
                pts.append((tau[0], tau[1], tau[2], tau[2] + t3, kind))
    return pts


def write_keys():
    os.makedirs(KEYS, exist_ok=True)
    files = {}
    # c0: dimer, L=4, 2001 steps.
    files["c0_dimer.key"] = dimer_key()
    files["c0_dimer_short.key"] = dimer_key(t_end=300)
    # c2 scan template (TAU1..3 / T_END substituted per point, as the reference's
    # script/IO-scripts/key.key-tmpl).
    files["c2_dimer_scan.key-tmpl"] = (dimer_key().replace("50 20 12500", "TAU1 20 12500", 1)
                                       .replace("150 20 12500", "TAU2 20 12500", 1)
                                       .replace("250 20 12500", "TAU3 20 12500", 1)
                                       .replace("0 1000 0.5 0.5", "0 T_END 0.5 0.5"))
    # c1: 7-site FMO-like aggregate with the two-exciton manifold, N=29, L=3.
    H, dip = aggregate(7, 2024, 12400, 200, 100)
    files["c1_fmo.key"] = key_text(8, 7, 3, H, OHMIC_35_106_77K, dip,
                                   [(50, 20, 12500), (150, 20, 12500), (250, 20, 12500)], (0, 2000, 0.5, 0.5))
    # c1 through all three pulse windows (601 steps, records from pulse 3 at 250 fs).
    files["c1_fmo_300fs.key"] = key_text(8, 7, 3, H, OHMIC_35_106_77K, dip,
                                         [(50, 20, 12500), (150, 20, 12500), (250, 20, 12500)], (0, 300, 0.5, 0.5))
    files["c1_fmo_short.key"] = key_text(8, 7, 3, H, OHMIC_35_106_77K, dip,
                                         [(0, 20, 12500), (1, 20, 12500), (0, 20, 12500)], (0, 3, 0.5, 0.5))
    # c3: 12-site chain, single-excitation manifold (extension keyword), L=3.
    H, dip = chain(12, 77, 150, 80)
    files["c3_chain.key"] = key_text(13, 12, 3, H, SUPEROHMIC_50_150_300K, dip,
                                     [(50, 20, 12500)] * 3, (0, 3000, 0.5, 0.5), single_manifold=True)
    files["c3_chain_short.key"] = key_text(13, 12, 3, H, SUPEROHMIC_50_150_300K, dip,
                                           [(0, 20, 12500)] * 3, (0, 10, 0.5, 0.5), single_manifold=True)
    # c4: trimer with two-exciton manifold (N=7), L=4.
    H, dip = aggregate(3, 4, 0, 0, 120, e_fixed=[12300, 12450, 12600])
    files["c4_trimer.key"] = key_text(4, 3, 4, H, OHMIC_35_106_77K, dip,
                                      [(50, 20, 12500), (150, 20, 12500), (350, 20, 12500)], (0, 1000, 0.5, 0.5))
    # c4 fit workload: P(t1, t3) recorded every 2 fs (128 t3 samples per point over 254 fs)
    files["c4_trimer_fit.key"] = key_text(4, 3, 4, H, OHMIC_35_106_77K, dip,
                                          [(50, 20, 12500), (150, 20, 12500), (350, 20, 12500)], (0, 1000, 0.5, 2))
    files["c4_trimer_short.key"] = key_text(4, 3, 4, H, OHMIC_35_106_77K, dip,
                                            [(20, 20, 12500), (50, 20, 12500), (80, 20, 12500)], (0, 160, 0.5, 0.5))
    # Disorder + several samples: exercises the RNG stream, the diagonal sort and averaging.
    files["t_disorder.key"] = dimer_key(tau=(30, 60, 90), t_end=140, n_sample=3, seed=114,
                                        sigma=[[0, 0, 0], [0, 42.4, 0], [0, 0, 42.4]])
    # The reference's own example system (example/CPU_dimer_ohmic/key.key-tmpl), K=2, L=2,
    # 6 bath lines (91 ADOs), dt = 2 fs, print every 10 fs, two samples.
    files["t_ref_example.key"] = key_text(3, 2, 2, [[0, 0, 0], [0, 400, 100], [0, 100, 500]], REF_EXAMPLE_BATH,
                                          [(0, 1, 1.0, 0.0, 0.0), (0, 2, 0.0, 1.0, 0.0)],
                                          [(210, 20, 500), (260, 20, 500), (260, 20, 500)], (0, 900, 2, 10),
                                          n_sample=2, seed=114,
                                          sigma=[[0, 0, 0], [0, 42.4, 0], [0, 0, 42.4]])
    # Delay-scan template with disorder averaging (2 samples) for the heom_scan driver
    # (TAU1..3 / T_END substituted as script/IO-scripts/gen_2d_data.sh does).
    files["t_scan.key-tmpl"] = (dimer_key(tau=(30, 60, 90), t_end=140, n_sample=2, seed=114,
                                          sigma=[[0, 0, 0], [0, 42.4, 0], [0, 0, 42.4]])
                                .replace("30 20 12500", "TAU1 20 12500", 1)
                                .replace("60 20 12500", "TAU2 20 12500", 1)
                                .replace("90 20 12500", "TAU3 20 12500", 1)
                                .replace("0 140 0.5 0.5", "0 T_END 0.5 0.5"))
    # Population dynamics (CPU_dynamics): a dimer and a trimer, site 1 initially excited.
    files["d_dimer.key"] = dynamics_key_text([[0, 80], [80, 150]], 2, 3, OHMIC_35_106_77K, (0, 400, 1, 5))
    files["d_trimer.key"] = dynamics_key_text([[150, 95, -30], [95, 0, 60], [-30, 60, 300]], 3, 3,
                                              REF_EXAMPLE_BATH, (0, 200, 0.5, 2))
    # Large first-order field (no perturbative smallness) and a negative site energy,
    # which the reference's diagonal sort treats specially (dynamics.cpp:24-27).
    files["t_strong.key"] = key_text(3, 2, 3, [[0, 0, 0], [0, -50, 300], [0, 300, 400]], OHMIC_35_106_77K,
                                     [(0, 1, 0.3, -0.2, 0.9), (0, 2, 0.5, 0.1, -0.8)],
                                     [(10, 8, 200), (30, 8, 200), (45, 8, 200)], (0, 80, 0.25, 0.5))
    for name, text in files.items():
        with open(os.path.join(KEYS, name), "w") as f:
            f.write(text)
    return sorted(files)


def parse_driver_output(text):
    """Parse ref_driver / heom_oracle output into (traj[n_sample, 3, n], combined[n])."""
    trajs, comb, cur, mode = [], [], None, None
    for line in text.splitlines():
        if line.startswith("#traj"):
            cur = []
            trajs.append(cur)
            mode = "t"
        elif line.startswith("#combined"):
            mode = "c"
        elif line.startswith("#"):
            mode = None
        elif mode == "t":
            v = [float(x) for x in line.split()]
            cur.append([complex(v[0], v[1]), complex(v[2], v[3]), complex(v[4], v[5])])
        elif mode == "c":
            v = [float(x) for x in line.split()]
            comb.append(complex(v[0], v[1]))
    traj = np.array([np.array(t).T for t in trajs], dtype=np.complex128) if trajs else np.zeros((0, 3, 0))
    return traj, np.array(comb, dtype=np.complex128)


DYNAMICS = ["d_dimer.key", "d_trimer.key"]
GOLDEN = ["c0_dimer_short.key", "c0_dimer.key", "c4_trimer_short.key", "t_disorder.key",
          "t_ref_example.key", "t_strong.key", "c1_fmo_short.key",
          "c4_trimer.key",      # config-4 system at 0-1000 fs, 2001 steps
          "c1_fmo_300fs.key",   # ~12 min of CPU (dense N = 29 zgemm)
          "c1_fmo.key"]         # ~2 h 20 min of CPU (4001 steps)


# The delay scan of the heom_scan driver test (gen_2d_data.sh parameters).
SCAN_ARGS = dict(t0=30, propagate=40, tau_step=10, tau_bound=20, T=("0", "50"))


def gen_2d_keys(template_text, t0, propagate, tau_step, tau_bound, T):
    """Restatement of script/IO-scripts/gen_2d_data.sh:37-61: {file name: key text}."""
    def emit(tau1, tau2, tau3, t_end):
        return (template_text.replace("TAU1", str(tau1)).replace("TAU2", str(tau2))
                .replace("TAU3", str(tau3)).replace("T_END", str(t_end)))
    out = {}
    for t in T:
        tv = int(t)
        for i in range(0, tau_bound + 1, tau_step):
            out[f"key_{i}_{t}.key"] = emit(t0, t0 + i, t0 + i + tv, t0 + i + tv + propagate)
        for i in range(-tau_bound, 0, tau_step):
            a = -i
            out[f"key_{i}_{t}.key"] = emit(t0 + a, t0, t0 + a + tv, t0 + a + tv + propagate)
    return out


def write_golden():
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    if not os.path.exists(drv):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref"])
    os.makedirs(REF, exist_ok=True)
    for name in GOLDEN:
        out = subprocess.run([drv, os.path.join(KEYS, name)], check=True, capture_output=True, text=True).stdout
        traj, comb = parse_driver_output(out)
        np.savez_compressed(os.path.join(REF, name.replace(".key", ".npz")), traj=traj, combined=comb)
        print(f"{name}: traj {traj.shape} combined {comb.shape}")
    # The unmodified CPU_2DES executable's stdout, for byte-compatibility of the CLI.
    exe = os.path.join(ROOT, "oracle", "_ref", "CPU_2DES")
    for name in ["c0_dimer_short.key", "t_disorder.key"]:
        out = subprocess.run([exe, os.path.join(KEYS, name)], check=True, capture_output=True, text=True).stdout
        with open(os.path.join(REF, name.replace(".key", ".out")), "w") as f:
            f.write(out)
    # Population dynamics: full-precision populations (ref_dynamics) and CPU_dynamics stdout.
    dyn = os.path.join(ROOT, "oracle", "_ref", "ref_dynamics")
    cdyn = os.path.join(ROOT, "oracle", "_ref", "CPU_dynamics")
    for name in DYNAMICS:
        kp = os.path.join(KEYS, name)
        out = subprocess.run([dyn, kp, "1", "2"], check=True, capture_output=True, text=True).stdout
        pops = [[float(x) for x in blk.split("\n")[1:] if x.strip()] for blk in out.split("#site")[1:]]
        np.savez_compressed(os.path.join(REF, name.replace(".key", ".npz")), population=np.array(pops))
        # CPU_dynamics prints "Running <path>": run it from the key's directory with the bare name
        txt = subprocess.run([cdyn, name], cwd=KEYS, check=True, capture_output=True, text=True).stdout
        with open(os.path.join(REF, name.replace(".key", ".out")), "w") as f:
            f.write(txt)
        print(f"{name}: populations {np.array(pops).shape}")
    # CPU_2DES outputs of the driver's delay scan: 2d-output/out_{tau}_{T}.out
    import tempfile
    scan_out = os.path.join(REF, "scan")
    os.makedirs(scan_out, exist_ok=True)
    keys = gen_2d_keys(open(os.path.join(KEYS, "t_scan.key-tmpl")).read(), **SCAN_ARGS)
    with tempfile.TemporaryDirectory() as d:
        for name, text in sorted(keys.items()):
            kp = os.path.join(d, name)
            with open(kp, "w") as f:
                f.write(text)
            out = subprocess.run([exe, kp], check=True, capture_output=True, text=True).stdout
            with open(os.path.join(scan_out, "out" + name[3:-4] + ".out"), "w") as f:
                f.write(out)
    print(f"scan: {len(keys)} CPU_2DES outputs")


def scan_key_text(row):
    """The c2 scan template with one point's pulse times and end time."""
    text = open(os.path.join(KEYS, "c2_dimer_scan.key-tmpl")).read()
    r = [repr(float(v)) for v in row[:4]]
    return text.replace("TAU1", r[0]).replace("TAU2", r[1]).replace("TAU3", r[2]).replace("T_END", r[3])


def truth_points():
    """Stratified subset of the 1024-point c2 scan: for each of rephasing / non-rephasing
    and each of the 8 waiting times, 3 coherence times drawn from a fixed seed (the
    shortest, t1 = 0, at T = 0 and the longest, t1 = 315 fs, at T = 700 fs forced in).
    Returns [(grid index, (tau1, tau2, tau3, t_end))]."""
    grid = scan_points()
    rng = np.random.default_rng(2026)
    out = []
    for ik, kind in enumerate(("R", "NR")):
        for i2 in range(8):
            idx = sorted(int(v) for v in rng.choice(64, 3, replace=False))
            if i2 == 0:
                idx[0] = 0
            if i2 == 7:
                idx[-1] = 63
            for i1 in sorted(set(idx)):
                g = (ik * 8 + i2) * 64 + i1
                assert grid[g][4] == kind
                out.append((g, grid[g][:4]))
    return out


def c4_fit_rows(t0=50.0, n_t1=32, t1_step=5.0, t2=200.0, t3_span=255.0):
    """The config-4 grid: rephasing points t1 = 0..155 fs at t2 = 200 fs; with records
    every 2 fs from pulse 3 on, t_end = tau3 + 255 fs gives 128 t3 samples per point."""
    rows = []
    for i in range(n_t1):
        t1 = i * t1_step
        tau3 = t0 + t1 + t2
        rows.append((t0, t0 + t1, tau3, tau3 + t3_span))
    return rows


def short_scan_rows(t0=50.0, t1s=(0.0, 35.0, 80.0, 155.0), t2s=(0.0, 100.0, 300.0), t3=150.0):
    """The shortened scan geometry of the GPU scan tests (t3 = 150 fs)."""
    rows = []
    for t2 in t2s:
        for t1 in t1s:
            rows.append((t0, t0 + t1, t0 + t1 + t2, t0 + t1 + t2 + t3))   # rephasing
            rows.append((t0 + t1, t0, t0 + t1 + t2, t0 + t1 + t2 + t3))   # non-rephasing
    return rows


def _run_point(args):
    exe, text, extra = args
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        kp = os.path.join(d, "p.key")
        with open(kp, "w") as f:
            f.write(text)
        out = subprocess.run([exe, kp, *extra], check=True, capture_output=True, text=True).stdout
    return parse_driver_output(out)


def write_truth(workers=None):
    """Binary128 truth (heom_oracle --quad: the reference's scheme on its own double
    data, propagated and combined in binary128) for
      * truth_c2.npz: the stratified 48-point subset of the c2 scan at full length
        (t3 = 400 fs), with the reference build's own double result beside it;
      * truth_scan_short.npz: the 24-point shortened scan of the GPU scan tests;
      * truth_c0_dimer_short.npz: the c0 short point of the smoke check.
    About 30 s of CPU per full-length point; points run in parallel processes."""
    from concurrent.futures import ThreadPoolExecutor
    oracle_exe = os.path.join(ROOT, "oracle", "heom_oracle")
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    for exe, tgt in ((oracle_exe, "all"), (ref_exe, "ref")):
        if not os.path.exists(exe):
            subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), tgt])
    workers = workers or max(1, (os.cpu_count() or 2) - 1)

    def pack(rows, results):
        counts = [len(c) for _, c in results]
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        return np.array(rows, dtype=np.float64), off, np.concatenate([c for _, c in results])

    sets = {"c2": [r for _, r in truth_points()], "scan_short": short_scan_rows()}
    with ThreadPoolExecutor(workers) as ex:
        for name, rows in sets.items():
            jobs = [(oracle_exe, scan_key_text(r), ["--quad"]) for r in rows]
            truth = list(ex.map(_run_point, jobs))
            R, off, P = pack(rows, truth)
            extra = {}
            if name == "c2":
                extra["grid_index"] = np.array([g for g, _ in truth_points()], dtype=np.int64)
                ref = list(ex.map(_run_point, [(ref_exe, scan_key_text(r), []) for r in rows]))
                R2, off2, Pref = pack(rows, ref)
                assert np.array_equal(off, off2)
                extra["reference"] = Pref
            np.savez_compressed(os.path.join(REF, f"truth_{name}.npz"), rows=R, offsets=off, truth=P, **extra)
            print(f"truth_{name}: {len(rows)} points, {len(P)} records")
    write_truth_keys(workers)


TRUTH_KEYS = ["c0_dimer_short.key", "c4_trimer_short.key", "t_disorder.key", "c4_trimer.key"]


def write_truth_keys(workers=None):
    """Binary128 truth of single key files (truth_<key>.npz: traj, combined) and of the
    heom_scan driver's delay scan (truth_scan_driver.npz: one combined output per
    out_{tau}_{T}.out file, disorder-averaged over the key's two samples)."""
    from concurrent.futures import ThreadPoolExecutor
    oracle_exe = os.path.join(ROOT, "oracle", "heom_oracle")
    workers = workers or max(1, (os.cpu_count() or 2) - 1)
    with ThreadPoolExecutor(workers) as ex:
        res = list(ex.map(_run_point, [(oracle_exe, open(os.path.join(KEYS, k)).read(), ["--quad"])
                                       for k in TRUTH_KEYS]))
        for k, (traj, comb) in zip(TRUTH_KEYS, res):
            np.savez_compressed(os.path.join(REF, "truth_" + k.replace(".key", ".npz")), traj=traj, combined=comb)
            print(f"truth_{k}: {len(comb)} records")
        keys = gen_2d_keys(open(os.path.join(KEYS, "t_scan.key-tmpl")).read(), **SCAN_ARGS)
        names = sorted(keys)
        res = list(ex.map(_run_point, [(oracle_exe, keys[n], ["--quad"]) for n in names]))
        counts = [len(c) for _, c in res]
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        outs = np.array(["out" + n[3:-4] + ".out" for n in names])
        np.savez_compressed(os.path.join(REF, "truth_scan_driver.npz"), names=outs, offsets=off,
                            truth=np.concatenate([c for _, c in res]))
        print(f"truth_scan_driver: {len(names)} files")


TRUTH_SPLIT_KEYS = ["c1_fmo_300fs.key"]   # ~1 h of CPU per trajectory (N = 29, binary128)


def _split_values(text):
    """Rows of `heom_oracle --quad-mask` output as exact (re, im) fractions (hi + lo)."""
    from fractions import Fraction
    out = []
    for line in text.splitlines():
        if line.startswith("#") or not line.strip():
            continue
        a, b, c, d = (float(x) for x in line.split())
        out.append((Fraction(a) + Fraction(b), Fraction(c) + Fraction(d)))
    return out


def write_truth_split():
    """Binary128 truth of large keys: the three trajectories run as separate processes
    (heom_oracle --quad-mask, values as hi/lo double pairs) and are combined exactly,
    p111 - p110 - p101, before rounding to double (truth_<key>.npz: combined)."""
    from concurrent.futures import ThreadPoolExecutor
    exe = os.path.join(ROOT, "oracle", "heom_oracle")

    def run(args):
        name, mask = args
        return subprocess.run([exe, os.path.join(KEYS, name), "--quad-mask", mask], check=True,
                              capture_output=True, text=True).stdout

    for name in TRUTH_SPLIT_KEYS:
        with ThreadPoolExecutor(3) as ex:
            outs = list(ex.map(run, [(name, m) for m in ("111", "110", "101")]))
        t111, t110, t101 = (_split_values(o) for o in outs)
        comb = np.array([complex(float(a[0] - b[0] - c[0]), float(a[1] - b[1] - c[1]))
                         for a, b, c in zip(t111, t110, t101)], dtype=np.complex128)
        np.savez_compressed(os.path.join(REF, "truth_" + name.replace(".key", ".npz")), combined=comb)
        print(f"truth_{name}: {len(comb)} records")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--golden", action="store_true", help="golden vectors from the reference build (oracle/_ref)")
    ap.add_argument("--truth", action="store_true", help="binary128 truth vectors (heom_oracle --quad)")
    ap.add_argument("--truth-split", action="store_true",
                    help="binary128 truth of the large keys, one process per trajectory (hours)")
    a = ap.parse_args()
    print("\n".join(write_keys()))
    if a.golden:
        write_golden()
    if a.truth:
        write_truth()
    if a.truth_split:
        write_truth_split()
