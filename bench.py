"""Benchmark of the H.psi hot path on the 16-atom bcc workload (96^3 grid, 128 bands, FP64).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one Kohn-Sham H.psi (FD8 kinetic + local potential + GTH
Kleinman-Bylander nonlocal) over all 128 real Gamma-point bands of the
2x2x2 bcc supercell (a = 12 bohr, h = 0.125 bohr, 16 atoms), seeded synthetic
psi ~ U[-0.5, 0.5] (seed 2) and a seeded synthetic local potential.

value  = algorithmic H.psi bytes / device time (GB/s), all ranks, inputs resident in HBM;
         algorithmic bytes per apply = nb*N*(8 read + 8 write) + 8*N (V) + projector tables.
e2e    = the same bytes / time of the public-API call on pinned HOST psi in and H.psi out
         (qsb_ham_apply_host: host->device and device->host copies inside the timed region,
         band chunks pipelined so that both copy directions and the apply overlap).
N > 1  : each rank applies H to its own 128-band slice of a 128*N-band set (band
         decomposition, no data-path collective): weak scaling.
--impl reference: the reference's own CPU operators (oracle/_ref, compiled from the
         reference source) on the host cores, bands split over processes as the
         reference's state decomposition does; bounded sample per step.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "qumasun-workshop-template_b200")
ORACLE = os.path.join(ROOT, "oracle")

METRIC = "LOBPCG SCF wall-time to 1e-6 Ha/atom: mixed vs FP64 on B200; HBM GB/s of H·ψ"
UNIT = "GB/s"
NX = NY = NZ = 96
H_GRID = 0.125
NB = 128
A_CELL = 6.0
REPS = 2
SEED = 2
GTH = dict(nl=2, r=(0.40, 0.55), h=(5.0, 1.5))
RCUT = 6.0


def positions():
    pos = []
    for i in range(REPS):
        for j in range(REPS):
            for k in range(REPS):
                base = np.array([i, j, k], float) * A_CELL
                pos.append(base)
                pos.append(base + 0.5 * A_CELL)
    return np.array(pos)


def potential(N):
    rng = np.random.default_rng(SEED + 1000)
    return rng.uniform(-1.0, 1.0, size=N)


def algorithmic_bytes(nb, N, n_proj_points, wmax, elem=8):
    return nb * N * 2 * elem + N * elem + n_proj_points * wmax * elem


def max_over_ranks(values, dist, device):
    """Per-rank timings -> their maxima over all ranks (the job's time)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_gbs(bytes_per_rank, world, ms):
    """Whole-job throughput: every rank moves bytes_per_rank in the (max-over-ranks) time ms."""
    return world * bytes_per_rank / (ms * 1e-3) / 1e9


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), hw=parts[5], hwt=parts[6], swt=parts[7],
                                 pcap=parts[8], util=float(parts[9])))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return None
        load = [r for r in rows if r["util"] > 0] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median([r["sm"] for r in load])), "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(load)}


# ---------------------------------------------------------------------------
# CPU reference arm (the reference's own operators, oracle/_ref)
# ---------------------------------------------------------------------------
def _ref_worker(args):
    """Runs in a spawned process: H.psi on `count` bands with the reference's code."""
    seed, count, reps = args
    sys.path.insert(0, ORACLE)
    import oracle as O
    if O.ref_available():
        O.ref_set_threads(1)
    N = NX * NY * NZ
    grid = (NX, NY, NZ, H_GRID, H_GRID, H_GRID)
    V = potential(N)
    rng = np.random.default_rng(seed)
    psi = rng.uniform(-0.5, 0.5, size=(count, N))
    sp = [dict(nl=GTH["nl"], r=GTH["r"], h=GTH["h"])] * (2 * REPS ** 3)
    times = []
    if O.ref_available():
        cube = O.gth_cube_tables(positions(), sp, NX, NY, NZ, H_GRID, H_GRID, H_GRID, RCUT)
        run = lambda: O.ref_hamiltonian(grid, V, cube, psi, count)
    else:
        tab = O.gth_tables(positions(), sp, H_GRID, H_GRID, H_GRID, RCUT)
        run = lambda: O.hamiltonian(grid, V, tab, psi, count)
    run()  # warm
    for _ in range(reps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    return times


def _ref_solver_c0(cores):
    """Runs in a spawned process: the reference's own EigenLOBPCG_d_multi per
    iteration, and a whole config-0 SCF to 1e-6 Ha / atom with it as the
    eigensolver (oracle/scf_oracle.py: the loop and its density, Hartree, LDA,
    occupations and Kerker-DIIS pieces restated in numpy, every LOBPCG call the
    reference's), on `cores` BLAS threads."""
    sys.path.insert(0, ORACLE)
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import oracle as O
    import scf_oracle as S
    from cases import SCF_C0, scf_inputs
    if not O.ref_available():
        return None
    O.ref_set_threads(cores)
    inp = scf_inputs()
    nx, ny, nz, dx, dy, dz = inp["grid"]
    N = nx * ny * nz
    cube = O.gth_cube_tables(inp["pos"], inp["sp"], nx, ny, nz, dx, dy, dz)
    V = S.gth_local_potential(inp["grid"], inp["pos"], inp["sp"])
    X = inp["X"].copy()
    keep = np.zeros_like(X)
    ev = np.zeros(SCF_C0["nb"])
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        O.ref_lobpcg_d(inp["grid"], V, cube, X, keep, SCF_C0["nb"], 2, ev, True)       # warm
        t0 = time.perf_counter()
        O.ref_lobpcg_d(inp["grid"], V, cube, X, keep, SCF_C0["nb"], 8, ev, False)
        t_iter = (time.perf_counter() - t0) / 8
    t0 = time.perf_counter()
    r = S.scf(inp["grid"], inp["pos"], inp["sp"], SCF_C0["nb"], SCF_C0["n_el"], inp["X"], **SCF_C0["params"])
    t_scf = time.perf_counter() - t0
    return {"lobpcg_ms_per_iteration": t_iter * 1e3, "scf_seconds": t_scf, "scf_steps": int(r["steps"]),
            "scf_final_energy_ha": float(r["energies"][-1]), "cores": cores}


def cpu_kind():
    sys.path.insert(0, ORACLE)
    import oracle as O
    return "reference" if O.ref_available() else "port"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    N = NX * NY * NZ
    bands_per_proc = 1
    steps, warm = args.steps, args.warmup
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        t0 = time.perf_counter()
        res = pool.map(_ref_worker, [(SEED + 17 * i, bands_per_proc, warm + steps) for i in range(cores)])
        wall = time.perf_counter() - t0
    # per step: every process applies H to its bands once; step time = slowest process
    per_step = [max(r[warm + s] for r in res) for s in range(steps)]
    t = float(np.mean(per_step))
    nb = cores * bands_per_proc
    sphere_pts = _sphere_points()
    value = algorithmic_bytes(nb, N, sphere_pts, 4) / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": warm, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded psi U[-0.5,0.5], seeded potential, GTH projectors)",
        "config": {"workload": "H.psi, bcc 2x2x2 supercell (16 atoms), 96^3 grid, FP64 real Gamma",
                   "bands_per_step": nb, "grid": [NX, NY, NZ]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": cpu_kind(),
                         "sample": f"{nb} of 128 bands per step, one band per process, {cores} spawned processes "
                                   f"(state decomposition), 1 BLAS thread each; wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # the SCF-wall-time half of the metric on the host: config 0 (2-atom bcc,
    # 32^3, 16 bands, LDA, Kerker-DIIS, |dE| < 1e-6 Ha / atom)
    with ctx.Pool(1) as pool:
        sc = pool.map(_ref_solver_c0, [cores])[0]
    if sc is not None:
        line["scf_c0_cpu"] = dict(sc, kind="reference",
                                  sample="config 0 whole SCF; every eigensolver call the reference's "
                                         "EigenLOBPCG_d_multi (OpenBLAS on the host cores), the loop's "
                                         "other pieces the numpy restatement (oracle/scf_oracle.py)")
    print(json.dumps(line))
    return 0


def _sphere_points():
    sys.path.insert(0, ORACLE)
    import oracle as O
    sp = [dict(nl=GTH["nl"], r=GTH["r"], h=GTH["h"])] * (2 * REPS ** 3)
    tab = O.gth_tables(positions(), sp, H_GRID, H_GRID, H_GRID, RCUT)
    return int(tab[0].sum())


def cpu_baseline_sample():
    """The reference (oracle/_ref) H.psi timed on the host on a bounded band sample."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        t1 = pool.map(_ref_worker, [(SEED, 1, 1)])[0][0]
    count = int(max(1, min(NB, math.floor(10.0 / max(t1, 1e-3)))))
    with ctx.Pool(1) as pool:
        t = pool.map(_ref_worker, [(SEED, count, 1)])[0][0]
    N = NX * NY * NZ
    value = algorithmic_bytes(count, N, _sphere_points(), 4) / t / 1e9
    return {"value": value, "unit": UNIT, "cores": 1, "kind": cpu_kind(),
            "sample": f"{count} of 128 bands of the same workload, one process, 1 thread, {t:.1f} s"}


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def gram_section(N, p, stream, reps=5):
    """The mixed-precision Rayleigh-Ritz Gram at the LOBPCG shape of this
    workload (U^T U over N grid points, p = 3 x bands fp32 columns, upper
    tiles): split-BF16x3 and INT8 Ozaki on the tensor cores (split included),
    against the fp64 DGEMM of the drop-in.  TFLOP/s are algorithmic for the
    full p x p product (2 N p^2), whatever part of it a kernel computes."""
    import ctypes
    import torch
    import qsb
    U = torch.rand(p, N, dtype=torch.float32, device="cuda") - 0.5
    T = torch.empty(p, p, dtype=torch.float64, device="cuda")
    out = {"grid_points": N, "columns": p, "upper_tiles": True}
    for name, wsq, fn in (("bf16x3", qsb.lib.qsb_gram_bf16x3_workspace, qsb.lib.qsb_gram_bf16x3),
                          ("int8_ozaki", qsb.lib.qsb_gram_ozaki_int8_workspace, qsb.lib.qsb_gram_ozaki_int8)):
        nbytes = ctypes.c_size_t()
        assert wsq(ctypes.c_int64(N), p, p, 1, ctypes.byref(nbytes)) == 0
        ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
        call = lambda: fn(1, ctypes.c_int64(N), p, p, ctypes.c_void_p(U.data_ptr()), ctypes.c_void_p(U.data_ptr()),
                          ctypes.c_void_p(T.data_ptr()), p, 1, ctypes.c_void_p(ws.data_ptr()),
                          ctypes.c_size_t(nbytes.value), ctypes.c_void_p(stream.cuda_stream))
        assert call() == 0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "tflops_algorithmic": 2.0 * N * p * p / (ms * 1e-3) / 1e12}
        del ws
    U64 = U.double()
    U64 @ U64.t()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        U64 @ U64.t()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    out["fp64_dgemm"] = {"ms": ms, "tflops_algorithmic": 2.0 * N * p * p / (ms * 1e-3) / 1e12}
    del U, U64, T
    torch.cuda.empty_cache()
    return out


NB_OCC = 48          # 16 atoms x 6 valence electrons / 2 (spin-paired)
EIG_TOL = 1e-6       # Ha, every occupied eigenvalue against the FP64 converged values


def lobpcg_section(H, psi, N, NB, dV, n_occ, stream, max_calls=60):
    """EigenLOBPCG_d_multi-style solves (4 iterations per call, the way an SCF
    step calls it) from one dV-orthonormal start, FP64 drop-in and mixed
    precision: ms per steady iteration, and device time until every occupied
    eigenvalue is within EIG_TOL of the FP64 solver's converged values."""
    import torch
    import qsb
    X0 = torch.linalg.qr(psi.t())[0].t().contiguous() / math.sqrt(dV)
    out = {"bands": NB, "occupied": n_occ, "iterations_per_call": 4, "tolerance_ha": EIG_TOL}
    traces = {}
    for prec in ("fp64", "mixed"):
        es = qsb.EigenSolver(N, NB, False, prec)
        es.set_hamiltonian(H)
        X = X0.clone()
        keep = torch.zeros_like(X)
        ev = np.zeros(NB)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # steady-state iteration time: a first-time call and a steady call (they
        # size the dense-solver workspaces), then 3 iterations timed
        es.lobpcg_d(dV, NB, 1, ev, X, keep, True)
        es.lobpcg_d(dV, NB, 1, ev, X, keep, False)
        torch.cuda.synchronize()
        e0.record(stream)
        es.lobpcg_d(dV, NB, 3, ev, X, keep, False)
        e1.record(stream)
        torch.cuda.synchronize()
        it, _ = es.last_stats()
        ms_it = e0.elapsed_time(e1) / max(it, 1)
        # convergence run from the same start, every call timed on the device
        X.copy_(X0)
        keep.zero_()
        times, evs = [], []
        limit = max_calls if prec == "fp64" else 2 * max_calls
        for c in range(limit):
            e0.record(stream)
            es.lobpcg_d(dV, NB, 4, ev, X, keep, c == 0)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            evs.append(ev.copy())
            if prec == "fp64" and c > 2 and np.abs(evs[-1][:n_occ] - evs[-2][:n_occ]).max() < 1e-10:
                break
            if prec == "mixed" and "fp64" in traces:
                if np.abs(evs[-1][:n_occ] - traces["fp64"][1][-1][:n_occ]).max() < EIG_TOL:
                    break
        traces[prec] = (np.array(times), np.array(evs))
        out[prec] = {"ms_per_iteration": ms_it}
        if prec == "mixed":
            out[prec]["overlap_dropped_max"], out[prec]["overlap_min_kept"], out[prec]["drop_tolerance"] = \
                es.overlap_stats()
            out[prec]["last_call_cholesky_solves"], out[prec]["last_call_overlap_basis_solves"] = es.solve_stats()
        es.close()
        del X, keep
        torch.cuda.empty_cache()
    ref = traces["fp64"][1][-1][:n_occ]
    for prec in ("fp64", "mixed"):
        times, evs = traces[prec]
        err = np.abs(evs[:, :n_occ] - ref[None, :]).max(axis=1)
        hit = np.nonzero(err < EIG_TOL)[0]
        o = out[prec]
        o["calls_to_tolerance"] = int(hit[0]) + 1 if len(hit) else None
        o["seconds_to_tolerance"] = float(times[:hit[0] + 1].sum() * 1e-3) if len(hit) else None
        o["final_max_error_ha"] = float(err[-1])
    if out["fp64"]["seconds_to_tolerance"] and out["mixed"]["seconds_to_tolerance"]:
        out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds_to_tolerance"] / out["mixed"]["seconds_to_tolerance"]
    out["note"] = ("eigensolver part of the SCF metric on a fixed H (the whole SCF loop is the scf section); "
                   "reference eigenvalues = FP64 solver converged to 1e-10 Ha change")
    return out


# SCF workloads: bcc cells of the a = 6 bohr cell (GTH Z 6, r_loc 0.45, C1 -4,
# C2 0.6; s + p projectors), h = 0.125 bohr, LDA, Fermi 0.01 Ha, 4 LOBPCG
# iterations per step, Kerker (q0 0.8) + DIIS depth 6, |dE| < 1e-6 Ha / atom.
SCF_CONFIGS = {
    "c2": dict(reps=2, n=96, bands=128, jitter=0.0, seed=2),     # 16 atoms, 96 electrons
    "c3": dict(reps=3, n=144, bands=384, jitter=0.1, seed=3),    # 54 atoms, 324 electrons, displaced
}
GTH_LOCAL = dict(zion=6.0, rloc=0.45, c1=-4.0, c2=0.6)


def scf_positions(reps, jitter, seed):
    pos = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                base = np.array([i, j, k], float) * A_CELL
                pos.append(base)
                pos.append(base + 0.5 * A_CELL)
    pos = np.array(pos)
    if jitter > 0.0:
        pos = pos + np.random.default_rng(seed).normal(0.0, jitter, pos.shape)
    return pos


def scf_section(name, tol_ref=1e-8, max_steps=None, rho_tol=1e-8, polish_steps=12):
    """SCF wall time to 1e-6 Ha / atom, FP64 drop-in vs mixed precision, from one
    dV-orthonormal seeded start with the same mixer.  Both runs continue to
    |dE| < tol_ref per atom (or the step cap); the FP64 run's final energy is
    the reference E*.  Time to tolerance = summed wall seconds of the steps up
    to the first step after which |E - E*| / atom stays below 1e-6 (steps timed
    by the driver's host clock; each step ends with its energy on the host).
    Also reported: the stopping-rule point |dE| / atom < 1e-6 of each run, and
    at both end points the forces on every atom (local + nonlocal + Ewald)
    and the occupied Rayleigh quotients.  rho_tol > 0 also requires
    int |rho_out - rho_in| / N_e < rho_tol of both end points, so that they
    differ by the precision, not by where the stopping rule left each run.
    The mixed run stops its own loop at |dE| / atom < tol_ref and then, with
    polish_steps > 0, goes on in FP64 (qsb_scf_set_polish) until the same
    energy and density tolerances: FP32 rounding in its states holds its
    density residual at a few 1e-8 and its forces ~1e-5 off.
    seconds_to_end_point is the whole run to its end point, polish included."""
    import torch
    import qsb
    cfg = SCF_CONFIGS[name]
    n, nb = cfg["n"], cfg["bands"]
    cap = max_steps or (120 if name == "c2" else 160)
    h = A_CELL * cfg["reps"] / n
    N, dV = n ** 3, h ** 3
    pos = scf_positions(cfg["reps"], cfg["jitter"], cfg["seed"])
    na = len(pos)
    n_el = GTH_LOCAL["zion"] * na
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, [0] * na, [GTH["nl"]], [GTH["r"]], [GTH["h"]], RCUT)
    H.set_potential(np.zeros(N))
    gen = torch.Generator(device="cuda").manual_seed(cfg["seed"])
    psi = torch.rand(nb, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    X0 = torch.linalg.qr(psi.t())[0].t().contiguous() / math.sqrt(dV)
    del psi
    out = {"config": name, "atoms": na, "grid": [n, n, n], "bands": nb, "electrons": n_el,
           "lobpcg_iterations_per_step": 4, "tolerance_ha_per_atom": 1e-6, "reference_tolerance_ha_per_atom": tol_ref,
           "step_cap": cap, "density_residual_tolerance": rho_tol,
           "mixed_fp64_polish_steps_max": polish_steps,
           "mixing": "Kerker q0 0.8 A 0.5 + DIIS depth 6", "smearing_ha": 0.01}
    runs, forces, rq, polish, res_end = {}, {}, {}, None, {}
    for prec in ("fp64", "mixed"):
        es = qsb.EigenSolver(N, nb, False, prec)
        scf = qsb.SCF(H, es, nb, n_el)
        scf.set_gth_local(pos, [0] * na, [GTH_LOCAL["zion"]], [GTH_LOCAL["rloc"]], [GTH_LOCAL["c1"]],
                          [GTH_LOCAL["c2"]])
        es64 = None
        if prec == "mixed" and polish_steps > 0:
            es64 = qsb.EigenSolver(N, nb, False, "fp64")
            scf.set_polish(es64, polish_steps, tol_ref, rho_tol)
        else:
            scf.set_density_tolerance(rho_tol)
        X = X0.clone()
        keep = torch.zeros_like(X)
        scf.run(X, keep, 4, 1, 1e-6)           # one step: sizes the solver's workspaces
        X.copy_(X0)
        keep.zero_()
        torch.cuda.synchronize()
        e, ev, occ = scf.run(X, keep, 4, cap, tol_ref)
        if es64 is not None:
            first, count = scf.polish_stats()
            polish = {"first_step": first + 1 if first >= 0 else None, "steps": count}
        # adjoint forces on every atom at the end point, local + nonlocal
        # device-timed, + Ewald (host)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record()
        f = scf.local_forces() + np.asarray(H.nonlocal_energy_force(X, occ, na)[1]).reshape(na, 3)
        t1.record()
        torch.cuda.synchronize()
        f = f + qsb.ewald(pos, [GTH_LOCAL["zion"]] * na, [A_CELL * cfg["reps"]] * 3)[1]
        forces[prec] = (f, t0.elapsed_time(t1))
        rq[prec] = (ev, occ)
        runs[prec] = (e, scf.step_seconds())
        res_end[prec] = float(scf.step_residuals()[-1])
        scf.close()
        es.close()
        if es64 is not None:
            es64.close()
        del X, keep
        torch.cuda.empty_cache()
    e_ref = runs["fp64"][0][-1]
    for prec, (e, t) in runs.items():
        err = np.abs(e - e_ref) / na
        ok = np.nonzero(err >= 1e-6)[0]
        k = 0 if len(ok) == 0 else int(ok[-1]) + 1          # first step after which all stay within
        hit = k < len(e)
        de = np.abs(np.diff(e)) / na
        stop = np.nonzero(de < 1e-6)[0]
        ks = int(stop[0]) + 1 if len(stop) else None          # stopping rule |dE| / atom < 1e-6
        out[prec] = {"steps_run": len(e), "stopped_before_cap": len(e) < cap, "seconds_run": float(np.sum(t)),
                     "steps_to_tolerance": k + 1 if hit else None,
                     "seconds_to_tolerance": float(np.sum(t[:k + 1])) if hit else None,
                     "final_error_ha_per_atom": float(err[-1]),
                     "stopping_rule_step": ks + 1 if ks is not None else None,
                     "stopping_rule_seconds": float(np.sum(t[:ks + 1])) if ks is not None else None,
                     "stopping_rule_error_ha_per_atom": float(err[ks]) if ks is not None else None,
                     "seconds_to_end_point": float(np.sum(t)),
                     "end_point_density_residual": res_end[prec],
                     "final_energy_ha": float(e[-1])}
    if polish is not None:
        out["mixed"]["fp64_polish"] = polish
    if out["fp64"]["seconds_to_tolerance"] and out["mixed"]["seconds_to_tolerance"]:
        out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds_to_tolerance"] / out["mixed"]["seconds_to_tolerance"]
    out["speedup_to_end_point_mixed_vs_fp64"] = (out["fp64"]["seconds_to_end_point"] /
                                                 out["mixed"]["seconds_to_end_point"])
    occupied = rq["fp64"][1] > 1e-6
    out["mixed_vs_fp64_end_point"] = {
        "max_force_error_ha_per_bohr": float(np.abs(forces["mixed"][0] - forces["fp64"][0]).max()),
        "max_force_ha_per_bohr": float(np.abs(forces["fp64"][0]).max()),
        "max_occupied_eigenvalue_error_ha": float(np.abs(rq["mixed"][0] - rq["fp64"][0])[occupied].max()),
        "force_ms": {k: v[1] for k, v in forces.items()}}
    out["note"] = ("E excludes the constant ion-ion term; E* = FP64 run's final energy; the mixed run's "
                   "final_error_ha_per_atom is its error against it (bar 1e-6); end-point errors compare "
                   "the two runs' end points (both density-converged; the mixed one after its FP64 polish): "
                   "forces local + nonlocal + Ewald on every atom (bar 1e-5 Ha/bohr), Rayleigh quotients "
                   "of the bands with occupation > 1e-6 (bar 1e-6 Ha)")
    H.close()
    return out


# config 1: O + 2 H in a 20 bohr box, 112^3, GTH-form species (O: one s
# projector; H: local only), 4 occupied + 4 empty bands
WATER_O = dict(zion=6.0, rloc=0.247, c1=-16.58, c2=2.40, r=0.222, h=18.27)
WATER_H = dict(zion=1.0, rloc=0.2, c1=-4.18, c2=0.725)


def scf_c0_section():
    """Config 0 (2-atom bcc, 32^3, 16 bands) SCF to |dE| < 1e-6 Ha / atom on the
    device, FP64 and mixed, from the same seeded orthonormal start as the
    reference arm's host run (psi U[-0.5, 0.5] from PCG64(0), orthonormalised): wall seconds."""
    import torch
    import qsb
    n, nb, n_el = 32, 16, 12.0
    h = A_CELL / n
    N = n ** 3
    pos = np.array([[0.0, 0.0, 0.0], [0.5 * A_CELL] * 3])
    # psi ~ U[-0.5, 0.5] from numpy PCG64(0) (the host run's start), then
    # dV-orthonormalised on the device (qsb_orthonormalize)
    psi0 = np.random.default_rng(0).uniform(-0.5, 0.5, size=(nb, N))
    out = {"config": "c0", "atoms": 2, "grid": [n, n, n], "bands": nb, "tolerance_ha_per_atom": 1e-6}
    for prec in ("fp64", "mixed"):
        H = qsb.Hamiltonian(n, n, n, h, h, h)
        H.set_gth_projectors(pos, [0, 0], [GTH["nl"]], [GTH["r"]], [GTH["h"]], RCUT)
        H.set_potential(np.zeros(N))
        es = qsb.EigenSolver(N, nb, False, prec)
        scf = qsb.SCF(H, es, nb, n_el)
        scf.set_gth_local(pos, [0, 0], [GTH_LOCAL["zion"]], [GTH_LOCAL["rloc"]], [GTH_LOCAL["c1"]],
                          [GTH_LOCAL["c2"]])
        scf.set_mixing(0.5, 0.8, 6)
        scf.set_smearing(0.01)
        for rep in range(2):                     # the first run sizes the workspaces
            X = qsb.orthonormalize(torch.from_numpy(psi0).cuda(), N, h ** 3)
            keep = torch.zeros_like(X)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e, ev, occ = scf.run(X, keep, 4, 60, 1e-6)
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
        out[prec] = {"seconds": t, "steps": len(e), "final_energy_ha": float(e[-1])}
        scf.close()
        es.close()
        H.close()
    return out


def config4_section(scf_steps=3):
    """Config 4's two parts on one GPU.
    Independent systems: 32 cubic cells with edges from {32, 40, 48, 56, 64}
    (h = 0.25 bohr), 8-64 real bands and 1-4 GTH atoms at seeded positions
    (seed 4); one H.psi of all of them through qsb_ham_apply_batch (the FD8 + V
    part in one persistent launch) against the systems' own qsb_ham_apply one
    after another, and with the autotuner on.
    k-points: config 0's cell on a 48^3 grid (h = 0.125) with the 4 x 4 x 4
    Gamma-centred mesh (64 k-points, weight 1/64, no symmetry reduction), 24
    complex bands per k (12 electrons), k-point SCF steps (qsb_scf_run_kpoints),
    FP64 and mixed (complex64 bundles): wall seconds per step over `scf_steps`
    steps from seeded orthonormal starts."""
    import torch
    import qsb
    rng = np.random.default_rng(4)
    hams, psis, outs, nbs = [], [], [], []
    alg = 0
    for i in range(32):
        n = int(rng.choice([32, 40, 48, 56, 64]))
        nb = int(rng.integers(8, 65))
        na = int(rng.integers(1, 5))
        hh = 0.25
        pos = rng.uniform(0, n * hh, (na, 3))
        H = qsb.Hamiltonian(n, n, n, hh, hh, hh)
        H.set_potential(rng.uniform(-1, 1, n ** 3))
        H.set_gth_projectors(pos, [0] * na, [GTH["nl"]], [GTH["r"]], [GTH["h"]], RCUT)
        hams.append(H)
        psis.append(torch.rand(nb, n ** 3, dtype=torch.float64, device="cuda") - 0.5)
        outs.append(torch.empty_like(psis[-1]))
        nbs.append(nb)
        alg += nb * n ** 3 * 16 + n ** 3 * 8
    out = {"systems": {"count": 32, "bands_total": int(sum(nbs)),
                       "grid_points_total": int(sum(h.N for h in hams)), "algorithmic_bytes": alg}}

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def per_system():
        for H, p, o in zip(hams, psis, outs):
            H.apply(p, o)
    t_b = timed(lambda: qsb.apply_batch(hams, psis, outs))
    t_p = timed(per_system)
    qsb.set_autotune(True)
    t_t = timed(lambda: qsb.apply_batch(hams, psis, outs))
    qsb.set_autotune(False)
    out["systems"].update({"batched_ms": t_b, "per_system_ms": t_p, "autotuned_ms": t_t,
                           "batched_gbs": alg / t_b / 1e6, "per_system_gbs": alg / t_p / 1e6,
                           "autotune_log": qsb.autotune_report().strip().splitlines()[-1:]})
    for H in hams:
        H.close()
    del psis, outs
    torch.cuda.empty_cache()
    # k-point part
    n, nb, n_el = 48, 24, 12.0
    hh = A_CELL / n
    N = n ** 3
    b = 2 * math.pi / A_CELL
    kvec = np.array([[i * b / 4, j * b / 4, k * b / 4] for i in range(4) for j in range(4) for k in range(4)])
    w = np.full(64, 1.0 / 64)
    pos = np.array([[0.0, 0.0, 0.0], [0.5 * A_CELL] * 3])
    kp = {"kpoints": 64, "grid": [n, n, n], "bands_per_k": nb, "electrons": n_el, "steps_timed": scf_steps}
    for prec in ("fp64", "mixed"):
        H = qsb.Hamiltonian(n, n, n, hh, hh, hh)
        H.set_gth_projectors(pos, [0, 0], [GTH["nl"]], [GTH["r"]], [GTH["h"]], RCUT)
        H.set_potential(np.zeros(N))
        es = qsb.EigenSolver(N, nb, True, prec)
        scf = qsb.SCF(H, es, nb, n_el)
        scf.set_gth_local(pos, [0, 0], [GTH_LOCAL["zion"]], [GTH_LOCAL["rloc"]], [GTH_LOCAL["c1"]], [GTH_LOCAL["c2"]])
        scf.set_kpoints(kvec, w)
        gen = torch.Generator(device="cuda").manual_seed(4)
        Xs = []
        for k in range(64):
            x = torch.rand(nb, 2, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
            Xs.append(qsb.orthonormalize(x, N, hh ** 3, True))
        keeps = [torch.zeros_like(x) for x in Xs]
        scf.run_kpoints(Xs, keeps, 4, 1, 1e-6)            # sizes the workspaces
        torch.cuda.synchronize()
        e, ev, occ = scf.run_kpoints(Xs, keeps, 4, scf_steps, 1e-12)
        t = scf.step_seconds()
        kp[prec] = {"seconds_per_step": float(np.mean(t)), "steps": len(e), "last_energy_ha": float(e[-1])}
        scf.close()
        es.close()
        H.close()
        del Xs, keeps
        torch.cuda.empty_cache()
    kp["speedup_per_step_mixed_vs_fp64"] = kp["fp64"]["seconds_per_step"] / kp["mixed"]["seconds_per_step"]
    out["kpoints"] = kp
    return out


def relax_section(fmax=1e-4):
    """Wall time of the LBFGS relaxation of config 1 (qsb_relax_lbfgs: SCF warm
    from the previous geometry's states, local + nonlocal + Ewald forces) from
    its jittered start to max |F| < fmax, FP64."""
    import torch
    import qsb
    n, L = 112, 20.0
    h = L / n
    N = n ** 3
    pos = np.array([[0.0, 0.0, 0.0], [1.43, 1.11, 0.0], [-1.43, 1.11, 0.0]])
    pos = pos + np.random.default_rng(1).normal(0.0, 0.05, pos.shape) + L / 2
    species = [0, 1, 1]
    proj = ([1, 0], [[WATER_O["r"], 0.0], [0.0, 0.0]], [[WATER_O["h"], 0.0], [0.0, 0.0]], 9.0)
    sps = (WATER_O, WATER_H)
    local = tuple([sp[k] for sp in sps] for k in ("zion", "rloc", "c1", "c2"))
    H = qsb.Hamiltonian(n, n, n, h, h, h)
    H.set_gth_projectors(pos, species, *proj)
    H.set_potential(np.zeros(N))
    es = qsb.EigenSolver(N, 8, False, "fp64")
    scf = qsb.SCF(H, es, 8, 8.0)
    scf.set_gth_local(pos, species, *local)
    scf.set_density_tolerance(1e-7)
    gen = torch.Generator(device="cuda").manual_seed(1)
    psi = torch.rand(8, N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    X = torch.linalg.qr(psi.t())[0].t().contiguous() / math.sqrt(h ** 3)
    keep = torch.zeros_like(X)
    torch.cuda.synchronize()
    t0 = time.time()
    p, e, f = scf.relax(X, keep, pos, species, proj, local, scf_tol=1e-9, max_iter=40, fmax=fmax)
    torch.cuda.synchronize()
    seconds = time.time() - t0
    out = {"config": "water, 20 bohr box, 112^3, 8 bands", "lbfgs_steps": int(len(e) - 1), "seconds": seconds,
           "max_force_ha_per_bohr": float(np.linalg.norm(f, axis=1).max()), "fmax": fmax,
           "energy_drop_ha": float(e[0] - e[-1]),
           "oh_bonds_bohr": [float(np.linalg.norm(p[1] - p[0])), float(np.linalg.norm(p[2] - p[0]))]}
    scf.close()
    es.close()
    H.close()
    return out


def fft_kinetic_section(H, psi, hpsi, stream, alg_bytes, steps=20):
    """Device time of one H.psi with the FFT kinetic (qsb_ham_set_kinetic(1):
    batched cuFFT D2Z / Z2D in 32-band chunks, |G|^2 / 2, 1/N + V psi fused,
    the same nonlocal kernels) on the bench workload; the same algorithmic bytes
    as the FD8 apply for comparison (an FFT re-reads each band several times)."""
    import torch
    H.set_kinetic(1)
    try:
        for _ in range(3):
            H.apply(psi, hpsi)
        torch.cuda.synchronize()
        H.get_timing()
        H.set_timing(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            H.apply(psi, hpsi)
        e1.record(stream)
        torch.cuda.synchronize()
        H.set_timing(False)
        ms = e0.elapsed_time(e1) / steps
        pm, km, em, applies, _ = H.get_timing()
    finally:
        H.set_kinetic(0)
    return {"ms_per_apply": ms, "algorithmic_gbs": alg_bytes / ms / 1e6,
            "breakdown_ms": {"nonlocal_projection": pm / applies, "fft_kinetic_plus_v": km / applies,
                             "nonlocal_expansion": em / applies}}


def main():
    global NB
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-lobpcg", action="store_true")
    ap.add_argument("--no-scf", action="store_true")
    ap.add_argument("--scf-config", default="c2", choices=sorted(SCF_CONFIGS),
                    help="SCF workload: c2 (16 atoms, 96^3, 128 bands; default) or c3 (54 atoms, 144^3, 384 bands)")
    ap.add_argument("--relax", action="store_true",
                    help="also time the LBFGS relaxation of config 1 (water, 112^3) to max |F| < 1e-4 Ha/bohr")
    ap.add_argument("--scf-tol-ref", type=float, default=1e-8,
                    help="|dE| / atom both SCF runs continue to (the FP64 end point is E*)")
    ap.add_argument("--scf-rho-tol", type=float, default=1e-8,
                    help="also require int |rho_out - rho_in| / N_e below this at both SCF end points (0: off)")
    ap.add_argument("--scf-polish-steps", type=int, default=12,
                    help="FP64 polish steps allowed after the mixed run's own stop (0: no polish)")
    ap.add_argument("--scf-max-steps", type=int, default=None, help="SCF step cap (default 120 for c2, 160 for c3)")
    ap.add_argument("--config4", action="store_true",
                    help="also run config 4: 32 uneven independent systems through the batched H.psi, and "
                         "k-point SCF steps at 64 k x 48^3 x 24 complex bands (FP64 and mixed)")
    ap.add_argument("--only-hpsi", action="store_true",
                    help="time the device-resident H.psi only (no e2e, FFT, Gram, LOBPCG, SCF or CPU sections); "
                         "the profiler captures use it")
    ap.add_argument("--only-lobpcg-mixed", action="store_true",
                    help="time two steady mixed-precision LOBPCG iterations only, after one first-time and one "
                         "steady call (the profiler captures use it)")
    ap.add_argument("--only-fft", action="store_true",
                    help="time the device-resident FFT-kinetic H.psi only (the profiler captures use it)")
    ap.add_argument("--bands", type=int, default=NB,
                    help="bands per GPU (default 128, the benchmark workload; smaller only for profiler captures)")
    args = ap.parse_args()
    NB = args.bands
    if args.impl == "reference":
        return run_reference(args)
    assert args.warmup >= 3, "at least 3 warm-up steps"

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    sys.path.insert(0, PKG)
    import qsb

    N = NX * NY * NZ
    H = qsb.Hamiltonian(NX, NY, NZ, H_GRID, H_GRID, H_GRID)
    H.set_potential(potential(N))
    pos = positions()
    H.set_gth_projectors(pos, [0] * len(pos), [GTH["nl"]], [GTH["r"]], [GTH["h"]], RCUT)
    n_pts, n_proj = H.projector_info()

    gen = torch.Generator().manual_seed(SEED + 7919 * rank)
    psi_host = (torch.rand(NB, N, dtype=torch.float64, generator=gen) - 0.5).pin_memory()
    hpsi_host = torch.empty_like(psi_host).pin_memory()
    psi = psi_host.cuda()
    hpsi = torch.empty_like(psi)
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        H.apply(psi, hpsi)
    torch.cuda.synchronize()
    H.get_timing()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)

    # ---- device-resident timing -------------------------------------------------
    H.set_timing(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        H.apply(psi, hpsi)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    H.set_timing(False)
    ms = e0.elapsed_time(e1) / args.steps
    proj_ms, sten_ms, exp_ms, applies, launches = H.get_timing()
    # keep the GPU busy long enough for the clock sampler to see the load
    t_end = time.time() + 1.0
    while time.time() < t_end:
        for _ in range(20):
            H.apply(psi, hpsi)
        torch.cuda.synchronize()

    if args.only_lobpcg_mixed:
        clocks.stop()
        dV = H_GRID ** 3
        X = torch.linalg.qr(psi.t())[0].t().contiguous() / math.sqrt(dV)
        es = qsb.EigenSolver(N, NB, False, "mixed")
        es.set_hamiltonian(H)
        keep = torch.zeros_like(X)
        ev = np.zeros(NB)
        es.lobpcg_d(dV, NB, 1, ev, X, keep, True)
        es.lobpcg_d(dV, NB, 1, ev, X, keep, False)
        torch.cuda.synchronize()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        es.lobpcg_d(dV, NB, 2, ev, X, keep, False)
        l1.record(stream)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"metric": "mixed LOBPCG iteration", "bands_per_gpu": NB,
                              "ms_per_iteration": l0.elapsed_time(l1) / 2,
                              "note": "--only-lobpcg-mixed: two steady iterations"}))
        es.close()
        H.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    if args.only_fft:
        clocks.stop()
        fft = fft_kinetic_section(H, psi, hpsi, stream, algorithmic_bytes(NB, N, n_pts, 4), steps=args.steps)
        if rank == 0:
            print(json.dumps({"metric": "FFT-kinetic H.psi", "bands_per_gpu": NB, "fft_kinetic": fft,
                              "note": "--only-fft: device-resident FFT-kinetic H.psi timing only"}))
        H.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    if args.only_hpsi:
        clocks.stop()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": whole_job_gbs(algorithmic_bytes(NB, N, n_pts, 4), world, ms),
                              "unit": UNIT, "ms_per_step": ms, "bands_per_gpu": NB,
                              "breakdown_ms": {"nonlocal_projection": proj_ms / max(applies, 1),
                                               "stencil": sten_ms / max(applies, 1),
                                               "nonlocal_expansion": exp_ms / max(applies, 1)},
                              "note": "--only-hpsi: device-resident H.psi timing only"}))
        H.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # ---- end to end through the public API with host buffers -------------------
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        H.apply_host(psi_host, hpsi_host)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        H.apply_host(psi_host, hpsi_host)      # qsb_ham_apply_host: chunked, copies both ways overlapped
    f1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = f0.elapsed_time(f1) / e2e_steps

    # ---- the same H.psi with the FFT kinetic (the reference's default operator) --
    fft = fft_kinetic_section(H, psi, hpsi, stream, algorithmic_bytes(NB, N, n_pts, 4))

    # ---- block LOBPCG on the same H: FP64 drop-in vs mixed precision ----------
    lob = None
    gram = gram_section(N, 3 * NB, stream)
    if not args.no_lobpcg:
        lob = lobpcg_section(H, psi, N, NB, H_GRID ** 3, n_occ=min(NB_OCC, NB), stream=stream)
    # ---- whole SCF to 1e-6 Ha/atom: FP64 drop-in vs mixed precision (one system, N = 1 only)
    scf = None
    if not args.no_scf and world == 1:
        scf = scf_section(args.scf_config, args.scf_tol_ref, args.scf_max_steps, args.scf_rho_tol,
                          args.scf_polish_steps)
    relax = relax_section() if args.relax and world == 1 else None
    scf_c0 = scf_c0_section() if not args.no_scf and world == 1 else None
    config4 = config4_section() if args.config4 and world == 1 else None
    clk = clocks.stop()

    ms, e2e_ms = max_over_ranks([ms, e2e_ms], dist, "cuda")
    alg = algorithmic_bytes(NB, N, n_pts, 4)
    value = whole_job_gbs(alg, world, ms)
    e2e_value = whole_job_gbs(alg, world, e2e_ms)
    peak, peak_kind = load_peaks()
    # dominant kernel: the FD8 + V stencil; its algorithmic bytes are psi read +
    # Hpsi write + V
    sten_avg_s = sten_ms / max(applies, 1) * 1e-3
    sten_bytes = NB * N * 16 + N * 8
    achieved = sten_bytes / sten_avg_s / 1e9
    traffic = None
    tr_file = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_file):
        traffic = json.load(open(tr_file)).get("fd8_ws_kernel_bytes_per_launch")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded psi U[-0.5,0.5], seeded potential, analytic GTH projectors)",
        "config": {"workload": "H.psi, bcc 2x2x2 supercell (16 atoms, a=12 bohr), 96^3 grid (h=0.125), "
                               f"{NB} bands per GPU, FP64 real Gamma, FD8 + V + GTH s+p KB nonlocal",
                   "grid": [NX, NY, NZ], "bands_per_gpu": NB, "atoms": len(pos), "projector_points": n_pts,
                   "parallelism": f"band decomposition x{world}",
                   "l2": "inputs larger than L2 (psi 906 MB per GPU)"},
        "band_grid_points_per_s": world * NB * N / (ms * 1e-3),
        "breakdown_ms": {"nonlocal_projection": proj_ms / max(applies, 1), "stencil": sten_ms / max(applies, 1),
                         "nonlocal_expansion": exp_ms / max(applies, 1)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "fd8_ws_kernel (FD8 + V, MODE 1)",
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": NB * N * 8, "d2h_bytes_per_step": NB * N * 8,
                "ms_per_step": e2e_ms},
        "gpu_launches": launches,
        "fft_kinetic": fft,
        "relax": relax,
        "lobpcg": lob,
        "scf": scf,
        "scf_c0": scf_c0,
        "config4": config4,
        "gram": gram,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    if rank == 0:
        print(json.dumps(line))
    H.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
