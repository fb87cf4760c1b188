"""Benchmark: PMCHWT MLFMA matvecs/s on one B200 (plain FP64 path).

Workload (default): dielectric sphere of radius 5 lambda at 300 MHz,
icosphere subdivided 6 times (81,920 triangles, 122,880 RWGs, 245,760
unknowns), eps_r = 2.5 - 0.1j, leaf box 0.25 lambda, 7-point rule; x seeded
uniform on the unit disk (mt19937_64 seed 0). Synthetic mesh (the
reference's meshes are not distributed). A step is one operator application
w = A x. The operator tables (8.7 GB of leaf patterns alone) are far larger
than L2, so no explicit flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints ONE JSON line on rank 0. Under torchrun every rank runs an
independent replica on its own GPU (the path does not shard: "replicas
only"); the device time is the max over ranks and value = total matvecs of
all ranks / that time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "PMCHWT solve s/RHS to 1e-3 residual & matvec/s vs plain FP64 GPU MLFMA path"
UNIT = "matvec/s"
FREQ = 3.0e8


def launches_per_apply(max_level: int, tune: dict) -> int:
    """Kernels one operator apply launches: the aggregation (one launch for
    both media with agg variant 1, else one per medium); per medium one
    interpolation per level pair, the translations (the leaf level and the
    other levels as two launches with m2l variants 2-7, else one per level)
    and one anterpolation per level pair; then the leaf testing + near-field
    kernel (two kernels with leaf variant 1)."""
    lv = max_level - 2
    # segmented translation variants: the leaf level and the other levels as two launches
    m2l = 2 if tune["m2l.variant"] in (2, 3, 4, 5, 6, 7, 8) else lv + 1
    agg = 1 if tune.get("agg.variant", 0) == 1 else 2
    leaf = 2 if tune.get("leaf.variant", 0) == 1 else 1
    return agg + 2 * (lv + m2l + lv) + leaf


def workload(args):
    from mlfma_pmchwt_b200 import mesh as M
    lam = M.wavelength(FREQ)
    if args.size == "full":
        return dict(name="sphere r=5 lambda, icosphere sub 6, 245,760 unknowns, eps_r 2.5-0.1j, leaf 0.25 lambda, "
                         "7-pt rule, FP64", sub=6, radius=5 * lam, eps=complex(2.5, -0.1), leaf=0.25)
    if args.size == "mid":
        return dict(name="sphere r=2.5 lambda, icosphere sub 5, 61,440 unknowns, eps_r 4, leaf 0.25 lambda, "
                         "7-pt rule, FP64", sub=5, radius=2.5 * lam, eps=complex(4.0, 0.0), leaf=0.25)
    return dict(name="sphere r=1 m, icosphere sub 3, 3,840 unknowns, eps_r 4, leaf 0.25 lambda, 7-pt rule, FP64",
                sub=3, radius=1.0, eps=complex(4.0, 0.0), leaf=0.25)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 25 ms; each sample is
    stamped with the host clock when it arrives, and stop() keeps the samples
    inside the window mark_begin() .. mark_end() (the timed region)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[tuple[float, str]] = []
        self.window = (None, None)

    def start(self, wait_s: float = 3.0):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "25"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        t = time.perf_counter()  # until the sampler is running
        while not self.lines and time.perf_counter() - t < wait_s:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark_begin(self):
        self.window = (time.perf_counter(), None)

    def mark_end(self):
        self.window = (self.window[0], time.perf_counter())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.05)  # the sample that closes the window
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self._t.join(timeout=2)
        t0, t1 = self.window
        inside = [ln for t, ln in self.lines if t0 is not None and t1 is not None and t0 <= t <= t1 + 0.05]
        rows = inside if inside else [ln for _, ln in self.lines]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in rows:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "in_timed_region": bool(inside)}


def dist_setup(backend: str = "nccl"):
    """One process per GPU (torchrun environment); replicas only: the
    process group carries the timing barrier and the max over ranks."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def replica_rate(ms_local: float, steps: int, world: int, device) -> tuple[float, float]:
    """Whole-job applies per second of N replicas: every rank applies `steps`
    times; the job's time is the slowest rank's (max over ranks)."""
    ms_total = allreduce_max(ms_local, world, device)
    return world * steps / (ms_total / 1000.0), ms_total


def allreduce_max(v: float, world: int, device) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def stage_bytes(op) -> dict:
    """Algorithmic bytes per apply for each stage, every operand touched once."""
    inf = op.info
    L = op.max_level
    c16 = 16.0
    b = {"aggregation": 0.0, "interpolation_up": 0.0, "translation": 0.0, "anterpolation_down": 0.0,
         "leaf_testing_near": 0.0}
    for Ks in (inf.K_k1, inf.K_k2):
        Kl = Ks[L - 2]
        Bl = inf.boxes[L - 2]
        b["aggregation"] += op.N * 3 * Kl * c16 + Bl * 6 * Kl * c16
        for l in range(2, L):
            i = l - 2
            b["interpolation_up"] += inf.boxes[i + 1] * 6 * Ks[i + 1] * c16 + inf.boxes[i] * 6 * Ks[i] * c16
        for l in range(2, L + 1):
            i = l - 2
            # Sm read once, Bm written once
            b["translation"] += 2 * inf.boxes[i] * 6 * Ks[i] * c16
            if l > 2:
                # parent Bm read once, child Bm read and written
                b["anterpolation_down"] += inf.boxes[i - 1] * 6 * Ks[i - 1] * c16 + 2 * inf.boxes[i] * 6 * Ks[i] * c16
        b["leaf_testing_near"] += op.N * 3 * Kl * c16 + Bl * 6 * Kl * c16
    b["leaf_testing_near"] += inf.near_pairs * 3 * c16 + 4 * op.n * c16
    return b


def translation_flops(op) -> float:
    """FP64 flops of the translation per apply: every interaction-list pair,
    both media, 6 pattern components, one complex multiply-add (8 flops)
    per direction."""
    inf = op.info
    return float(sum(inf.far_pairs[i] * (inf.K_k1[i] + inf.K_k2[i]) * 6 * 8 for i in range(op.max_level - 1)))


def fp64_peak_tflops(dev) -> float:
    """Measured FP64 throughput of this GPU: cuBLAS DGEMM (torch.matmul on
    float64, 4096^3), best of 5 with CUDA events."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def cpu_baseline_reference(args, wl, rank: int) -> dict | None:
    """The reference's own OpenMP matvec (oracle/_ref) on this host's cores."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    from mlfma_pmchwt_b200 import mesh as M
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    m = M.icosphere(wl["sub"], wl["radius"])
    nas = M.write_nas(m, Path("/tmp") / f"bench_ref_{os.getpid()}.nas")
    t0 = time.perf_counter()
    ref = O.RefOperator(nas, freq=FREQ, eps_r=wl["eps"], leaf_coeff=wl["leaf"])
    setup = time.perf_counter() - t0
    x = M.unit_disk_vector(ref.n, 0)
    ref.apply(x)  # warm-up
    times = []
    budget = args.cpu_budget
    t_start = time.perf_counter()
    while True:
        t = time.perf_counter()
        ref.apply(x)
        times.append(time.perf_counter() - t)
        if time.perf_counter() - t_start > budget or len(times) >= 50:
            break
    ref.close()
    return {"value": 1.0 / float(np.median(times)), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(times)} full reference matvecs (median) of the same operator after its "
                      f"{setup:.1f} s OpenMP setup; oracle/_ref built from the reference sources",
            "setup_s": setup}


def cpu_solve_baseline(args, local: int) -> dict | None:
    """The reference's own GMRES solve (MLFMM::matrix_solver -> MGMRES::mgmres,
    Code/GMRES.h:65-217, OpenMP matvecs) on the 3,840-unknown sphere (radius
    1 m, icosphere sub 3, eps_r 4, leaf 0.25 lambda; plane wave along -z,
    x-polarised): GMRES(30) to 1e-3, bounded at --cpu-solve-its iterations
    (it does not converge without a preconditioner). Beside it, the same
    GMRES(30) on the GPU with the same cap, and the GPU's FGMRES with the
    near-field preconditioner to convergence."""
    from oracle import oracle as O
    if not O.ref_available() or args.cpu_solve_its <= 0:
        return None
    from mlfma_pmchwt_b200 import MLFMM, plane_wave
    from mlfma_pmchwt_b200 import mesh as M
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    m = M.icosphere(3, 1.0)
    nas = M.write_nas(m, Path("/tmp") / f"bench_solve_{os.getpid()}.nas")
    ref = O.RefOperator(nas, freq=FREQ, eps_r=4.0, leaf_coeff=0.25)
    V = ref.rhs(0.0, 0.0, 0.0)[0]
    its = args.cpu_solve_its
    t = time.perf_counter()
    _, info = ref.solve(V, itr_max=its, mr=30, tol_abs=0.0, tol_rel=1e-3)
    ref_s = time.perf_counter() - t
    ref.close()
    true_r = info.get("true_residuals") or [float("nan")]
    op = MLFMM(m, freq=FREQ, eps_r=4.0, leaf_coeff=0.25, device=local)
    op.matrix_solver(V, itr_max=30, mr=30, tol_abs=0.0, tol_rel=1e-3)  # warm-up (graph capture)
    _, sg = op.matrix_solver(V, itr_max=its, mr=30, tol_abs=0.0, tol_rel=1e-3)
    _, sf = op.matrix_solver(V, itr_max=its, mr=30, tol_abs=0.0, tol_rel=1e-3, inner_its=8)
    op.close()
    return {"workload": "sphere r=1 m, icosphere sub 3, 3,840 unknowns, eps_r 4, leaf 0.25 lambda; plane wave "
                        "along -z, x-polarised", "cores": cores, "kind": "reference",
            "reference_gmres30": {"seconds": round(ref_s, 3), "iterations": len(info.get("history", [])),
                                  "s_per_iteration": round(ref_s / max(len(info.get("history", [])), 1), 5),
                                  "rel_residual": float(true_r[-1]), "tol": 1e-3, "itr_max": its},
            "gpu_gmres30": {"seconds": round(sg["seconds"], 4), "iterations": sg["iterations"],
                            "s_per_iteration": round(sg["seconds"] / max(sg["iterations"], 1), 6),
                            "rel_residual": sg["rel_residual"], "converged": sg["converged"]},
            "gpu_fgmres30_near8": {"seconds": round(sf["seconds"], 4), "iterations": sf["iterations"],
                                   "rel_residual": sf["rel_residual"], "converged": sf["converged"]}}


def run_reference_arm(args):
    # the reference's CPU matvec runs on rank 0 alone; no collective is needed
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    wl = workload(args)
    base = cpu_baseline_reference(args, wl, 0)
    if base is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmlfma_ref.so not built"}))
        return 0
    # steps: each step one reference matvec (bounded by --cpu-budget)
    line = {"metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / base["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": wl["name"], "parallelism": "openmp", "l2": "inputs larger than L2"},
            "impl": "reference", "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def measured_traffic(workload: str, stage: str, tune: dict):
    """DRAM bytes (read + write) per apply of a stage's kernels, from the
    one-pass ncu capture recorded in profiles/dram_traffic.json (command
    there), when it was taken on this workload with the same kernel choice;
    else None."""
    f = ROOT / "profiles" / "dram_traffic.json"
    if not f.exists():
        return None
    rec = json.loads(f.read_text())
    if rec.get("workload") != workload:
        return None
    ent = rec.get("stages", {}).get(stage)
    if not ent or any(tune.get(k) != v for k, v in ent.get("tuning", {}).items()):
        return None
    return ent["dram_bytes_per_apply"]


def parse_tuning(spec: str) -> dict | None:
    """'auto' -> None (autotune); else 'key=value,...' fixed kernel variants."""
    if spec == "auto":
        return None
    out = {}
    for item in spec.split(","):
        k, v = item.split("=")
        out[k.strip()] = int(v)
    return out


def solve_record(st: dict, inner_its: int) -> dict:
    rec = {"s_per_rhs": round(st["seconds"], 4), "iterations": st["iterations"], "converged": st["converged"],
           "rel_residual": st["rel_residual"], "restart": 50, "tol": 1e-3, "matvecs": st["matvecs"],
           "timing": "faster of two identical solves"}
    if inner_its:
        rec["solver"] = f"FGMRES(50), right preconditioner = {inner_its} GMRES steps on the near field"
        rec["near_products"] = st["near_products"]
    else:
        rec["solver"] = "GMRES(50)"
    return rec


def multi_rhs_study(args, local: int, mixed_only: bool = False) -> dict:
    """Many incidences on one body: sphere r = 2.5 lambda (icosphere sub 5,
    61,440 unknowns), eps_r 4, leaf 0.25 lambda; 128 plane waves, theta_i =
    i * 180/127, phi = 0, polarisation alternating theta / phi. Lockstep
    solves to 1e-3 with the complex64 operator inside FP64 refinement and in
    FP64; an FP64 lockstep solve to 1e-6 is the oracle for the monostatic
    RCS (backscatter at (theta_i, 0)) of each incidence."""
    from mlfma_pmchwt_b200 import MLFMM, plane_wave
    from mlfma_pmchwt_b200 import mesh as M
    lam = M.wavelength(FREQ)
    R = args.rhs
    op = MLFMM(M.icosphere(5, 2.5 * lam), freq=FREQ, eps_r=4.0, leaf_coeff=0.25, device=local, precision="mixed")
    th = np.array([180.0 * i / (R - 1) for i in range(R)])
    B = np.stack([op.compute_v_pmchwt(*plane_wave(90.0 * (i % 2), th[i], 0.0)) for i in range(R)])
    out = {"workload": f"sphere r=2.5 lambda, icosphere sub 5, {op.n} unknowns, eps_r 4, leaf 0.25 lambda; "
                       f"{R} plane waves theta 0-180 deg, phi 0, alternating polarisation",
           "rhs": R, "tol": 1e-3}

    def record(st, secs):
        its = [s_["iterations"] for s_ in st]
        return {"s_total": round(secs, 3), "s_per_rhs": round(secs / R, 4), "converged": sum(s_["converged"] for s_ in st),
                "iterations_mean": round(float(np.mean(its)), 2), "iterations_max": int(max(its)),
                "rel_residual_max": max(s_["rel_residual"] for s_ in st), "inner_its": args.study_inner_its}

    t = time.perf_counter()
    Xm, sm = op.solve_mixed_batch(B, itr_max=500, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
    out["mixed_lockstep"] = record(sm, time.perf_counter() - t)
    out["mixed_lockstep"]["solver"] = ("lockstep FGMRES(50) with the complex64 operator and near-field "
                                       "preconditioner, FP64 refinement")
    if mixed_only:
        op.close()
        return out
    t = time.perf_counter()
    Xd, sd = op.matrix_solver_batch(B, itr_max=500, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
    out["fp64_lockstep"] = record(sd, time.perf_counter() - t)
    t = time.perf_counter()
    x1, s1 = op.matrix_solver(B[0], itr_max=500, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
    out["fp64_one_at_a_time_s_per_rhs"] = round(time.perf_counter() - t, 4)
    Xo, so = op.matrix_solver_batch(B, itr_max=1000, mr=50, tol_abs=0.0, tol_rel=1e-6, inner_its=args.study_inner_its)
    mono = lambda X: np.array([op.calculate_rcs_pmchwt(X[i], th[i], 0.0)[1][0, 0] for i in range(R)])
    ro = mono(Xo)
    dm, dd = np.abs(mono(Xm) - ro), np.abs(mono(Xd) - ro)
    out["monostatic_rcs_error_db_vs_fp64_1e-6"] = {
        "mixed_max": round(float(dm.max()), 5), "mixed_median": round(float(np.median(dm)), 5),
        "fp64_1e-3_max": round(float(dd.max()), 5), "fp64_1e-3_median": round(float(np.median(dd)), 5)}
    op.close()
    return out


def full_rhs_study(args, local: int) -> dict:
    """128 incidences on the 245,760-unknown sphere (r = 5 lambda, icosphere
    sub 6, eps_r 2.5 - 0.1j, leaf 0.25 lambda; transfer factors with the
    complex argument, with which the solves converge on this lossy body):
    the lockstep mixed-precision solve (batched complex64 applies with the
    tensor-core leaf stages, near-field preconditioner, FP64 refinement) to
    1e-3, against the plain FP64 GPU path -- GMRES(50) on the FP64 operator
    without a preconditioner, to 1e-3 or 300 iterations -- on 8 of the
    incidences (every 17th), and single FP64 FGMRES on the same 8. Monostatic RCS of 8
    incidences and their bistatic RCS (phi = 0, 361 angles) against FP64
    solves to 1e-6. The excitations come from one batched launch, the far
    fields from the batched bistatic and monostatic kernels."""
    from mlfma_pmchwt_b200 import MLFMM, plane_wave
    from mlfma_pmchwt_b200 import mesh as M
    lam = M.wavelength(FREQ)
    R = 128
    t0 = time.perf_counter()
    op = MLFMM(M.icosphere(6, 5.0 * lam), freq=FREQ, eps_r=2.5 - 0.1j, leaf_coeff=0.25, device=local,
               precision="mixed", tf_complex_argument=True)
    setup = time.perf_counter() - t0
    th = np.array([180.0 * i / (R - 1) for i in range(R)])
    import torch
    Bd = torch.empty((R, op.n), dtype=torch.complex128, device=f"cuda:{local}")
    op.compute_v_pmchwt_batch_device([plane_wave(90.0 * (i % 2), th[i], 0.0) for i in range(R)], Bd.data_ptr())
    torch.cuda.synchronize(local)
    B = Bd.cpu().numpy()
    del Bd
    out = {"workload": f"sphere r=5 lambda, icosphere sub 6, {op.n} unknowns, eps_r 2.5-0.1j, leaf 0.25 lambda, "
                       f"complex-argument transfer factors; {R} plane waves theta 0-180 deg, phi 0, alternating "
                       f"polarisation", "rhs": R, "tol": 1e-3, "setup_s": round(setup, 2)}
    t = time.perf_counter()
    Xm, sm = op.solve_mixed_batch(B, itr_max=500, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
    secs = time.perf_counter() - t
    its = [s_["iterations"] for s_ in sm]
    out["mixed_lockstep"] = {"s_total": round(secs, 3), "s_per_rhs": round(secs / R, 4),
                             "converged": sum(s_["converged"] for s_ in sm),
                             "iterations_mean": round(float(np.mean(its)), 2), "iterations_max": int(max(its)),
                             "rel_residual_max": max(s_["rel_residual"] for s_ in sm),
                             "inner_its": args.study_inner_its}
    plain, fg = [], []
    sample = [17 * k for k in range(8)]  # theta 0-169 deg, the two polarisations in turn
    for i in sample:
        t = time.perf_counter()
        _, st = op.matrix_solver(B[i], itr_max=300, mr=50, tol_abs=0.0, tol_rel=1e-3)
        plain.append((time.perf_counter() - t, st["iterations"], st["converged"], st["rel_residual"]))
        t = time.perf_counter()
        _, st = op.matrix_solver(B[i], itr_max=300, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
        fg.append((time.perf_counter() - t, st["iterations"], st["converged"], st["rel_residual"]))
    for key, rows in (("plain_fp64_gmres", plain), ("fp64_fgmres_one_at_a_time", fg)):
        out[key] = {"s_per_rhs": round(float(np.mean([r[0] for r in rows])), 4),
                    "iterations": [int(r[1]) for r in rows], "converged": int(sum(r[2] for r in rows)),
                    "rel_residual_max": float(max(r[3] for r in rows)), "incidences": len(rows)}
    out["speedup_per_rhs_vs_plain_fp64_gmres"] = round(out["plain_fp64_gmres"]["s_per_rhs"] /
                                                       out["mixed_lockstep"]["s_per_rhs"], 2)
    sel = list(range(0, R, 16))
    Xo = np.stack([op.matrix_solver(B[i], itr_max=500, mr=50, tol_abs=0.0, tol_rel=1e-6,
                                    inner_its=args.study_inner_its)[0] for i in sel])
    out.update(rcs_errors(op, local, Xm[sel], Xo, th[sel]))
    op.close()
    return out


def rcs_errors(op, local: int, X, Xo, th_inc) -> dict:
    """RCS errors (dB) of solutions X against oracle solutions Xo: monostatic
    (backscatter at (theta_i, 0)) and bistatic (phi = 0, theta 0:0.5:180,
    361 angles, total RCS), through the batched far-field kernels."""
    import torch
    from mlfma_pmchwt_b200 import rcs_db
    R = len(X)
    dev = f"cuda:{local}"
    th = np.arange(0.0, 180.01, 0.5)
    ph = np.zeros_like(th)
    res = {}
    for key, V in (("x", X), ("o", Xo)):
        Vd = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
        Fb = torch.empty((R, len(th), 3), dtype=torch.complex128, device=dev)
        Fm = torch.empty((R, 3), dtype=torch.complex128, device=dev)
        s = torch.cuda.current_stream(local).cuda_stream
        op.calculate_rcs_batch_device(R, Vd.data_ptr(), th, ph, Fb.data_ptr(), s)
        op.calculate_rcs_mono_device(R, Vd.data_ptr(), th_inc, np.zeros(R), Fm.data_ptr(), s)
        torch.cuda.synchronize(local)
        fb, fm = Fb.cpu().numpy(), Fm.cpu().numpy()
        res[key] = (np.stack([rcs_db(th, ph, fb[r])[:, 0] for r in range(R)]),
                    np.array([rcs_db(th_inc[r], 0.0, fm[r:r + 1])[0, 0] for r in range(R)]))
    bi = np.abs(res["x"][0] - res["o"][0])
    mono = np.abs(res["x"][1] - res["o"][1])
    # angles within 20 dB of the cut's peak (away from the deep nulls)
    lit = res["o"][0] >= res["o"][0].max(axis=1, keepdims=True) - 20.0
    return {"monostatic_rcs_error_db_vs_fp64_1e-6": {"mixed_max": round(float(mono.max()), 5),
                                                      "mixed_median": round(float(np.median(mono)), 5),
                                                      "incidences": R},
            "bistatic_rcs_error_db_vs_fp64_1e-6": {"max": round(float(bi.max()), 5),
                                                    "median": round(float(np.median(bi)), 5),
                                                    "max_within_20db_of_peak": round(float(bi[lit].max()), 5),
                                                    "angles": len(th), "incidences": R,
                                                    "cut": "phi = 0, theta 0:0.5:180, total RCS"}}


def bodies_study(args, local: int) -> dict:
    """24 uneven dielectric bodies (mesh.uneven_bodies(1): icospheres,
    ellipsoids, superellipsoids; 3,840-61,440 unknowns; lossy eps_r), 16
    plane waves each (theta_i = i * 180/15, phi = 0, polarisation alternating),
    solved to 1e-3 per body by lockstep FGMRES with the complex64 operator
    inside FP64 refinement; transfer factors with the complex argument (the
    bodies are lossy). Each body has its own plan (and so its own streams);
    --bodies-workers host threads run that many bodies at once, largest
    first, so that the small bodies' launches and host round trips overlap
    on the GPU."""
    from concurrent.futures import ThreadPoolExecutor

    from mlfma_pmchwt_b200 import MLFMM, plane_wave
    from mlfma_pmchwt_b200 import mesh as M
    import torch

    def one(b):
        torch.cuda.set_device(local)
        t0 = time.perf_counter()
        op = MLFMM(b["mesh"], freq=FREQ, eps_r=b["eps_r"], leaf_coeff=0.25, device=local, precision="mixed",
                   tf_complex_argument=True)
        setup = time.perf_counter() - t0
        B = np.stack([op.compute_v_pmchwt(*plane_wave(90.0 * (i % 2), 12.0 * i, 0.0)) for i in range(16)])
        t1 = time.perf_counter()
        X, st = op.solve_mixed_batch(B, itr_max=600, mr=50, tol_abs=0.0, tol_rel=1e-3, inner_its=args.study_inner_its)
        solve = time.perf_counter() - t1
        row = {"kind": b["kind"], "unknowns": op.n, "eps_r": [round(b["eps_r"].real, 3), round(b["eps_r"].imag, 4)],
               "setup_s": round(setup, 3), "solve_s": round(solve, 3), "converged": sum(s_["converged"] for s_ in st),
               "iterations_mean": round(float(np.mean([s_["iterations"] for s_ in st])), 1)}
        op.close()
        return row

    bodies = M.uneven_bodies(1, FREQ)
    # largest bodies first (longest-processing-time order), so that the
    # longest solves do not start last; rows are reported in the set's order
    order = sorted(range(len(bodies)), key=lambda i: -len(bodies[i]["mesh"].face_ids))
    t_all = time.perf_counter()
    workers = max(1, args.bodies_workers)
    with ThreadPoolExecutor(max_workers=workers) as pool:
        done = list(pool.map(one, [bodies[i] for i in order]))
    total = time.perf_counter() - t_all
    rows = [None] * len(bodies)
    for i, r in zip(order, done):
        rows[i] = r
    return {"bodies": len(rows), "rhs": 16 * len(rows), "workers": workers, "total_s": round(total, 2),
            "s_per_rhs": round(total / (16 * len(rows)), 4),
            "converged": sum(r["converged"] for r in rows), "per_body": rows}


def learned_study(args, local: int) -> dict:
    """Learned preconditioner. Training: (v, P_near v) pairs with white-noise
    v on --learned-bodies seeded triaxial ellipsoids (mesh.training_ellipsoids:
    semi-axes 0.5-2 lambda, eps_r 2-6, 15,360 unknowns each), objective
    |A M v - v|^2 / |v|^2, Adam, all in the library's kernels. Evaluation: the
    held-out 6 x 2 x 2 lambda ellipsoid (eps_r 3.0 - 0.05j, 245,760 unknowns,
    transfer factors with the complex argument), 32 plane waves, FGMRES(50) to
    1e-3 with inner_its near-field steps, with and without the network;
    bistatic RCS (phi = 0, 361 angles) of 4 incidences against FP64 solves to
    1e-6."""
    from mlfma_pmchwt_b200 import MLFMM, learned
    from mlfma_pmchwt_b200 import mesh as M
    t0 = time.perf_counter()
    train = []
    for k, b in enumerate(M.training_ellipsoids(args.learned_bodies)):
        op = MLFMM(b["mesh"], freq=FREQ, eps_r=b["eps_r"], leaf_coeff=0.25, device=local)
        train.append((op, learned.random_directions(op, 32, inner_its=8, seed=k)))
    harvest_s = time.perf_counter() - t0
    params, hist, train_s = learned.train(train, epochs=args.learned_epochs, lr=1e-3, batch=8)
    for op, _ in train:
        op.close()
    train = None
    hb = M.held_out_ellipsoid()
    t1 = time.perf_counter()
    op = MLFMM(hb["mesh"], freq=FREQ, eps_r=hb["eps_r"], leaf_coeff=0.25, device=local, tf_complex_argument=True)
    setup_s = time.perf_counter() - t1
    inc = learned.incidences(32)
    rhs = [op.compute_v_pmchwt(*pw) for pw in inc]
    held = learned.random_directions(op, 8, inner_its=8, seed=999)
    before = learned.Trainer(learned.init_params(0)).evaluate([(op, held)])
    after = learned.Trainer(params).evaluate([(op, held)])
    gain = learned.solve_gain(op, params, rhs, inner_its=args.inner_its, itr_max=args.solve_its)
    # RCS of 4 incidences: near-field-preconditioned and learned solutions at
    # 1e-3 against FP64 solves to 1e-6
    th = np.linspace(0.0, 180.0, 361)
    ph = np.zeros_like(th)
    err = {"near_field": [], "learned": []}
    for b in rhs[::8]:
        xr, _ = op.matrix_solver(b, tol_rel=1e-6, tol_abs=0.0, mr=50, itr_max=args.solve_its, inner_its=16)
        _, ref_db = op.calculate_rcs_pmchwt(xr, th, ph)
        for tag, p in (("near_field", None), ("learned", params)):
            op.attach_learned(p)
            x, _ = op.matrix_solver(b, tol_rel=1e-3, tol_abs=0.0, mr=50, itr_max=args.solve_its,
                                    inner_its=args.inner_its)
            _, db = op.calculate_rcs_pmchwt(x, th, ph)
            err[tag].append(float(np.abs(db[:, 0] - ref_db[:, 0]).max()))
        op.attach_learned(None)
    out = {"workload": "held-out ellipsoid 6 x 2 x 2 lambda, eps_r 3.0-0.05j, 245,760 unknowns, 32 plane waves",
           "training": {"bodies": args.learned_bodies, "unknowns_each": 15360, "pairs": 32 * args.learned_bodies,
                        "epochs": args.learned_epochs, "objective": "|A M v - v|^2 / |v|^2, white-noise v",
                        "loss_first_epoch": round(hist[0], 5), "loss_last_epoch": round(hist[-1], 5),
                        "harvest_s": round(harvest_s, 2), "train_s": round(train_s, 2)},
           "held_out_objective": {"near_field_only": round(before["network"], 5),
                                  "with_network": round(after["network"], 5)},
           "setup_s": round(setup_s, 2), "inner_its": args.inner_its, "tol": 1e-3,
           "rcs_max_db_error_vs_fp64_1e-6": {k: round(max(v), 4) for k, v in err.items()}}
    for tag in ("near_field", "learned"):
        g = gain[tag]
        out[tag] = {"iterations_mean": round(g["iterations_mean"], 2), "iterations_max": max(g["iterations"]),
                    "s_per_rhs": round(g["s_per_rhs"], 4), "converged": g["converged"]}
    op.close()
    return out


def batched_apply_study(args, local: int, wl: dict) -> dict:
    """The batched complex64 apply of 16 right-hand sides on the workload's
    sphere (mixed-precision plan): per-batch CUDA-event time with the leaf
    aggregation and far-field testing on the tensor cores (batch_tc.variant
    1) and on the CUDA cores (0), with the tree passes once per level for all
    slots (batch_tree.variant 1) and one slot after another (0), against 16
    single complex64 applies, and the rows' relative difference from the FP64
    operator."""
    import torch
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    op = MLFMM(M.icosphere(wl["sub"], wl["radius"]), freq=FREQ, eps_r=wl["eps"], leaf_coeff=wl["leaf"],
               device=local, precision="mixed")
    R = 16
    X = torch.from_numpy(np.stack([M.unit_disk_vector(op.n, 60 + j) for j in range(R)])).cuda(local)
    W = torch.empty_like(X)
    stream = torch.cuda.Stream(local)
    sp = stream.cuda_stream

    def timed(fn, reps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize(local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(local)
        return e0.elapsed_time(e1) / reps

    out = {"workload": wl["name"], "rhs": R, "ms_per_batch": {}}
    for v in (1, 0):
        op.set_tuning("batch_tc.variant", v)
        out["ms_per_batch"]["tensor_cores" if v else "cuda_cores"] = round(
            timed(lambda: op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr(), sp), 3), 3)
    op.set_tuning("batch_tc.variant", 1)
    tree_keep = op.get_tuning("batch_tree.variant")
    for v, key in ((0, "tensor_cores_tree_slot_by_slot"), (1, "tensor_cores_tree_slot_grid")):
        op.set_tuning("batch_tree.variant", v)
        out["ms_per_batch"][key] = round(
            timed(lambda: op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr(), sp), 3), 3)
    op.set_tuning("batch_tree.variant", tree_keep)
    out["ms_per_batch"]["16_single_applies"] = round(16 * timed(
        lambda: op.apply_mixed_device(X[0].data_ptr(), W[0].data_ptr(), sp), 10), 3)
    op.apply_batch_mixed_device(R, X.data_ptr(), W.data_ptr(), sp)
    torch.cuda.synchronize(local)
    Wt = W.cpu().numpy()
    ref = op.apply_batch(X.cpu().numpy())
    out["rel_diff_vs_fp64_max"] = float(max(np.linalg.norm(Wt[j] - ref[j]) / np.linalg.norm(ref[j]) for j in range(R)))
    out["device_status"] = op.device_status()
    op.close()
    return out


def run_product(args):
    import torch
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = workload(args)
    if args.batched_only:  # the batched-apply study alone (small enough for profiler captures)
        if rank == 0:
            print(json.dumps({"batched_apply": batched_apply_study(args, local, wl)}))
        return 0
    if args.lockstep_only:  # the multi-RHS study's lockstep mixed solve alone (for profiler captures)
        if rank == 0:
            print(json.dumps({"multi_rhs": multi_rhs_study(args, local, mixed_only=True)}))
        return 0
    if args.full_rhs_only:  # the 128-incidence study on the 245,760-unknown sphere alone
        if rank == 0:
            print(json.dumps({"multi_rhs_full": full_rhs_study(args, local)}))
        return 0
    if args.learned_only:  # the learned-preconditioner study alone
        if rank == 0:
            print(json.dumps({"learned_preconditioner": learned_study(args, local)}))
        return 0
    m = M.icosphere(wl["sub"], wl["radius"])
    t0 = time.perf_counter()
    op = MLFMM(m, freq=FREQ, eps_r=wl["eps"], leaf_coeff=wl["leaf"], device=local,
               precision="mixed" if args.mixed else "fp64")
    setup_s = time.perf_counter() - t0
    n = op.n
    x_host = M.unit_disk_vector(n, 0)
    x = torch.from_numpy(x_host).to(dev)
    w = torch.empty(n, dtype=torch.complex128, device=dev)
    # a dedicated stream: the legacy default stream has handle 0, which the C
    # ABI reads as "the plan's own stream"
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream

    def step():
        op.apply_device(x.data_ptr(), w.data_ptr(), sp)

    fixed = parse_tuning(args.tuning)
    if fixed is None:
        tune = op.autotune(3)
    else:
        for k, v in fixed.items():
            op.set_tuning(k, v)
        tune = {k: op.get_tuning(k) for k, _ in op.TUNING_KEYS}
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)

    # timed region: device time, max over ranks
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark_begin()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks.mark_end()
    barrier(world)
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    # stage attribution: a second pass with the library's stage events (the
    # two media then run one after the other, so each stage is timed alone)
    op.profile(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(dev)
    stage_ms, napp = op.stage_times()
    op.profile(False)
    value, ms_total = replica_rate(ms_local, args.steps, world, dev)
    ms_per_step = ms_total / args.steps

    # end to end through the C ABI with pinned host buffers
    xh = torch.from_numpy(x_host).pin_memory()
    wh = torch.empty(n, dtype=torch.complex128).pin_memory()
    xh_np, wh_np = xh.numpy(), wh.numpy()
    for _ in range(2):
        op._lib.mlfma_apply(op._h, n, xh_np.ctypes.data_as(_dp_t()), wh_np.ctypes.data_as(_dp_t()))
    barrier(world)
    t = time.perf_counter()
    for _ in range(args.steps):
        rc = op._lib.mlfma_apply(op._h, n, xh_np.ctypes.data_as(_dp_t()), wh_np.ctypes.data_as(_dp_t()))
        if rc != 0:
            raise RuntimeError(op._lib.mlfma_last_error().decode())
    e2e_s = allreduce_max(time.perf_counter() - t, world, dev)
    barrier(world)
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n * 16,
           "d2h_bytes_per_step": n * 16}

    # roofline of the dominant stage (HBM-bound FP64 path)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    sb = stage_bytes(op)
    per_apply_ms = {k: v / max(napp, 1) for k, v in stage_ms.items()}
    dom = max(per_apply_ms, key=per_apply_ms.get)
    achieved = sb[dom] / (per_apply_ms[dom] / 1000.0) / 1e9
    traffic = measured_traffic(wl["name"], dom, tune)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_src, "traffic": traffic,
                "algorithmic_bytes": sb[dom],
                "stage_ms_per_apply": {k: round(v, 4) for k, v in per_apply_ms.items()},
                "stage_note": "stage times from a pass with the two media one after the other; "
                              "the timed apply runs the media's tree passes on two streams",
                "matvec_bytes": sum(sb.values()),
                "matvec_frac": round(sum(sb.values()) / (ms_per_step / 1000.0) / 1e9 / peak, 4),
                "stage_hbm_frac": {k: round(sb[k] / (v / 1000.0) / 1e9 / peak, 4)
                                   for k, v in per_apply_ms.items() if v > 0}}
    # the translation is FP64-arithmetic- and L2-bound rather than HBM-bound:
    # its second bound, against the measured DGEMM rate of this GPU
    fp64_peak = fp64_peak_tflops(dev)
    tflops = translation_flops(op) / (per_apply_ms["translation"] / 1000.0) / 1e12
    roofline["fp64"] = {"kernel": "translation", "flops": translation_flops(op), "achieved": round(tflops, 2),
                        "peak": round(fp64_peak, 2), "unit": "TFLOP/s", "frac": round(tflops / fp64_peak, 4),
                        "peak_source": "measured in this run: cuBLAS DGEMM (torch float64 matmul 4096^3)"}

    # the complex64 operator of the same plan (mixed precision), same timing
    mixed = None
    if args.mixed:
        wm = torch.empty_like(w)
        for _ in range(3):
            op.apply_mixed_device(x.data_ptr(), wm.data_ptr(), sp)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            op.apply_mixed_device(x.data_ptr(), wm.data_ptr(), sp)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        mms = allreduce_max(e0.elapsed_time(e1), world, dev) / args.steps
        step()
        torch.cuda.synchronize(dev)
        err = float(torch.linalg.vector_norm(wm - w) / torch.linalg.vector_norm(w))
        mixed = {"value": round(world * 1000.0 / mms, 3), "unit": UNIT, "ms_per_step": round(mms, 4),
                 "dtype": "c64 tables and arithmetic, c128 vectors", "rel_diff_vs_fp64_apply": err}

    # Solves of the plane-wave excitation (x-polarised, incident along -z) to
    # 1e-3 relative residual. (1) The reference's operator (real-argument
    # transfer factors, as Code/AlgoMLFMM.h:259-281 evaluates them for the
    # lossy medium too) with FGMRES(50) + near-field preconditioner;
    # (2) the same with complex-argument transfer factors h2_l(k2 R), which
    # the lossy medium needs for the far field to match its near field.
    solve = None
    def warm(fn):
        """Runs an identical solve twice and keeps the faster (the first also
        pays first-use costs such as the apply graph's capture)."""
        a, b = fn(), fn()
        return a if a[1]["seconds"] <= b[1]["seconds"] else b

    if args.solve_its > 0:
        from mlfma_pmchwt_b200 import plane_wave
        V = op.compute_v_pmchwt(*plane_wave(0.0, 0.0, 0.0))
        _, st = warm(lambda: op.matrix_solver(V, itr_max=args.solve_its, mr=50, tol_abs=1e-8, tol_rel=1e-3,
                                              inner_its=args.inner_its))
        solve = {"reference_transfer": solve_record(st, args.inner_its)}
        if args.plain_its > 0:
            _, sp_ = op.matrix_solver(V, itr_max=args.plain_its, mr=50, tol_abs=1e-8, tol_rel=1e-3)
            solve["reference_transfer_plain_gmres"] = solve_record(sp_, 0)
            solve["reference_transfer_plain_gmres"]["timing"] = "one solve"
        if wl["eps"].imag != 0.0:
            op.close()
            opc = MLFMM(m, freq=FREQ, eps_r=wl["eps"], leaf_coeff=wl["leaf"], device=local,
                        tf_complex_argument=True, precision="mixed" if args.mixed else "fp64")
            for k, v in tune.items():
                if not k.endswith("_ms"):
                    opc.set_tuning(k, v)
            _, sc = warm(lambda: opc.matrix_solver(V, itr_max=args.solve_its, mr=50, tol_abs=1e-8, tol_rel=1e-3,
                                                   inner_its=args.inner_its))
            solve["complex_transfer"] = solve_record(sc, args.inner_its)
            if args.mixed:
                _, sm = warm(lambda: opc.solve_mixed(V, itr_max=args.solve_its, mr=50, tol_abs=1e-8, tol_rel=1e-3,
                                                     inner_its=args.inner_its, refine_max=10))
                rec = solve_record(sm, args.inner_its)
                rec["solver"] = ("FP64 iterative refinement around complex64 " + rec["solver"] +
                                 "; residual checked with the FP64 operator")
                rec["refinements"] = sm["refinements"]
                solve["complex_transfer_mixed"] = rec
            op = opc

    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": wl["name"], "unknowns": n, "max_level": op.max_level,
                       "parallelism": "replicas" if world > 1 else "single", "l2": "inputs larger than L2",
                       "setup_s": round(setup_s, 2), "device_bytes": op.info.bytes_device,
                       "tuning": tune},
            "e2e": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in e2e.items()},
            "gpu_launches": args.steps * launches_per_apply(op.max_level, tune),
            "roofline": roofline, "clocks": clk}
    if mixed:
        line["mixed_precision"] = mixed
    if args.mixed and world == 1:
        line["batched_apply"] = batched_apply_study(args, local, wl)
    if args.rhs > 0 and world == 1:
        line["multi_rhs"] = multi_rhs_study(args, local)
    if args.bodies and args.size == "full" and world == 1:
        line["uneven_bodies"] = bodies_study(args, local)
    if args.full_rhs and args.size == "full" and world == 1:
        line["multi_rhs_full"] = full_rhs_study(args, local)
    if args.learned and world == 1:
        line["learned_preconditioner"] = learned_study(args, local)
    if solve:
        line["solve"] = solve
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline_reference(args, wl, rank)
        if base:
            line["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
            solve_base = cpu_solve_baseline(args, local)
            if solve_base:
                line["cpu_baseline"]["solve"] = solve_base
    if rank == 0:
        print(json.dumps(line))
    op.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def _dp_t():
    import ctypes
    return ctypes.POINTER(ctypes.c_double)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["product", "reference"], default="product")
    ap.add_argument("--size", choices=["full", "mid", "small"], default="full")
    ap.add_argument("--solve-its", type=int, default=300, help="outer iteration cap of the solves")
    ap.add_argument("--inner-its", type=int, default=None,
                    help="near-field GMRES steps per preconditioning (default: 16 for the 245,760-unknown solve "
                         "and the lockstep studies, 8 for single solves of the smaller spheres)")
    ap.add_argument("--plain-its", type=int, default=300, help="iteration cap of the plain GMRES comparison")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of reference matvecs to time")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-solve-its", type=int, default=300,
                    help="iteration cap of the reference's GMRES(30) solve in the CPU baseline (0: skip)")
    ap.add_argument("--rhs", type=int, default=128, help="incidences of the multi-RHS study (0: skip)")
    ap.add_argument("--no-bodies", dest="bodies", action="store_false",
                    help="skip the 24-body uneven batch study (run by default on the full-size workload)")
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="skip the complex64 (mixed-precision) operator and solve")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the 16-right-hand-side batched complex64 apply study and print its record")
    ap.add_argument("--no-full-rhs", dest="full_rhs", action="store_false",
                    help="skip the 128-incidence study on the 245,760-unknown sphere (run with --size full)")
    ap.add_argument("--full-rhs-only", action="store_true", help="run only that study")
    ap.add_argument("--lockstep-only", action="store_true",
                    help="run only the multi-RHS study's lockstep mixed solve (61,440 unknowns, --rhs incidences)")
    ap.add_argument("--learned", action="store_true", help="also run the learned-preconditioner study")
    ap.add_argument("--learned-only", action="store_true", help="run only the learned-preconditioner study")
    ap.add_argument("--learned-bodies", type=int, default=24,
                    help="training ellipsoids of the learned-preconditioner study")
    ap.add_argument("--learned-epochs", type=int, default=10)
    ap.add_argument("--bodies-workers", type=int, default=6,
                    help="bodies solved at once by the uneven-body study (host threads, one plan each)")
    ap.add_argument("--tuning", default="auto",
                    help="'auto' (autotune) or fixed kernel variants, e.g. m2l.variant=2,up.variant=1")
    args = ap.parse_args(argv)
    # the lockstep studies (61,440-unknown sphere, 24 bodies) use 16 unless given
    args.study_inner_its = 16 if args.inner_its is None else args.inner_its
    if args.inner_its is None:
        args.inner_its = 16 if args.size == "full" else 8
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_product(args)


if __name__ == "__main__":
    sys.exit(main())
