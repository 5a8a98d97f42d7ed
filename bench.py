#!/usr/bin/env python
"""Newton-system throughput on B200: assembly + MAS build + PCG of one implicit-step
Newton iteration (StiffGIPC's per-iteration linear system), mixed FP32-MAS / FP64
refinement vs plain FP64, plus adjoints/s.

Workload (N=1): two stacked soft cubes, each a 21^3 vertex lattice (2 x 40000 tets,
18522 vertices), E = 1e5 / 1e6 Pa, nu = 0.45, friction mu = 0.2, d-hat = 1e-3 m, top
cube with a seeded 1 m/s initial velocity; seeded synthetic positions (uniform 1e-4 m
perturbation).  A step = one Newton system: assembly, MAS hierarchy + inverses, PCG to
the reference criterion r.z <= 1e-4 r0.z0.  Multi-GPU runs are independent replicas.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "stiff-gipc_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Newton-system solves/s, mixed vs FP64 MAS-PCG at 1e-4 residual; adjoints/s"
STEP = "; one Newton system = assembly + MAS build + PCG to r.z <= 1e-4 r0.z0"
WORKLOADS = {
    "two_cubes": "two stacked soft cubes, 2 x 21^3 lattice (80000 tets, 18522 vertices), E 1e5/1e6 Pa, nu 0.45, "
                 "mu 0.2, d-hat 1e-3 m, contacts from the host pair generator" + STEP,
    "cube": "one soft cube, 11^3 lattice (5000 tets, 1331 vertices), E 1e5 Pa, nu 0.4, dropped from 0.05 m, "
            "d-hat 1e-3 m, no contact yet" + STEP,
    "cloth_sphere": "256^2 cloth (130050 triangles, 195585 hinges) rolled in layers 0.4 mm apart over a tet "
                    "sphere (20000 tets, r 0.3 m) on the ground, d-hat 5e-4 m, mu 0.2; about a million contact "
                    "pairs from the GPU pair search, lagged friction from the GPU set-up" + STEP,
    "abd_bed": "500 affine boxes (8 points, edge 0.05 m, kappa_ABD 1e8; about a fifth resting on the bed) over "
               "a soft tet bed (100000 tets, 23409 vertices, E 1e5 Pa) on the ground, d-hat 1e-3 m, contacts from "
               "the GPU pair search; one Newton system = FEM assembly + contact class partition + ABD body "
               "terms + ABD block Jacobi + MAS build + the coupled FEM + ABD PCG to r.z <= 1e-4 r0.z0",
}
L2_FLUSH_BYTES = 256 << 20
CPU_SOLVER = ("Eigen unavailable: the oracle's OpenMP restatement of the reference's assembly and "
              "MAS-preconditioned CG (FP64 vectors, FP32 MAS inverses), not an Eigen ConjugateGradient")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=21, help="lattice vertices per cube edge (two_cubes)")
    ap.add_argument("--workload", default="two_cubes", choices=sorted(WORKLOADS),
                    help="two_cubes (the headline), cube, cloth_sphere or abd_bed")
    ap.add_argument("--cpu-sample", type=int, default=0, help="CPU baseline solves (0 = auto, about 10 s)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--timeline", action="store_true",
                    help="events after the assembly, the MAS build and the solve of each step (one GPU)")
    ap.add_argument("--pcg-phases", action="store_true",
                    help="print the per-phase profile of the persistent PCG solve instead of the bench line")
    ap.add_argument("--kernel", default=None,
                    help="only re-launch this hot kernel (sgipc_time_kernel names) on the workload and print its "
                         "time: the launch an ncu capture of the roofline kernel should see")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes from an ncu capture (profiles/traffic.json), if committed."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.gpu = gpu_index
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, power, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        loaded = [s for s, p in zip(sm, power) if p > 200.0] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "samples_under_load": len(loaded)}


# ------------------------------------------------------------------------------------------
# CPU arms (oracle = CPU FP64 restatement of the reference's formulas)
# ------------------------------------------------------------------------------------------
def make_scene(args, host_contacts=True):
    """The workload's scene.  cloth_sphere leaves its contacts to the GPU pair search (see
    gpu_contacts) unless host_contacts asks for the host generator (about two minutes)."""
    from sgipc import scenes

    if args.workload == "cube":
        return scenes.scene_cube(11, touching=False, seed=0)
    if args.workload == "cloth_sphere":
        return scenes.scene_cloth_on_sphere(256, 4000, contacts=host_contacts)
    if args.workload == "abd_bed":
        raise ValueError("the abd_bed workload runs through run_abd_bed only")
    return scenes.scene_two_cubes(args.n, seed=1)


def gpu_contacts(g, sc):
    """Contact pairs, ground pairs and lagged friction sets found on the GPU, written back
    into the scene's host arrays (the inputs of the host-state step and the CPU legs)."""
    g.buildCP()
    g.buildFrictionSets()
    t = g.tet
    sc.pairs, sc.ground_pairs = t.pairs.cpu().numpy(), t.ground_pairs.cpu().numpy()
    sc.fric_pairs, sc.fric_lambda = t.fric_pairs.cpu().numpy(), t.fric_lambda.cpu().numpy()
    sc.fric_coord, sc.fric_basis = t.fric_coord.cpu().numpy(), t.fric_basis.cpu().numpy().reshape(-1, 3, 2)
    sc.fric_gd_pairs, sc.fric_gd_lambda = t.fric_gd_pairs.cpu().numpy(), t.fric_gd_lambda.cpu().numpy()


def make_system(args, device):
    """(scene, GIPC) of the workload on one GPU, contacts in place."""
    from sgipc import system

    sc = make_scene(args, host_contacts=False)
    if args.workload == "cloth_sphere":
        g = system.GIPC(sc, device=device, max_rhs=4, pair_capacity=2_000_000)
        gpu_contacts(g, sc)
    else:
        g = system.GIPC(sc, device=device, max_rhs=4)
    return sc, g


def cpu_solves(sc, count):
    import oracle

    t0 = time.perf_counter()
    for _ in range(count):
        b, r, c, v, _ = oracle.assemble(sc)
        m = oracle.Mas(sc, r, c, v)
        oracle.pcg(r, c, v, sc.nv, m, b, 1e-4, single=True)
        del m
    return time.perf_counter() - t0


def step_accuracy(g, sc, system, N, adjoint, dLdx):
    """Errors of the timed settings against a tight FP64 solve of the same system: the
    Newton direction dx of the mixed and FP64 solves at the r.z <= 1e-4 r0.z0 stop and at the
    true-residual 1e-4 stop (relative to the tight dx, and mixed against FP64 at each stop),
    and the adjoint gradients (dL/dE, dL/dv0) of the timed adjoint setting (mixed, r.z 1e-4)
    against the adjoint of a tight FP64 solve."""
    def rel(a, b):
        return float((a - b).norm() / b.norm())

    def solve(prec, crit, tol):
        g.computeGradientAndHessian()
        st = g.calculateMovingDirection(system.PCGSolverConfig(precision=prec, criterion=crit, global_tol_rate=tol,
                                                               max_iter_ratio=1.0))
        return g.moveDir.clone(), st

    tight, st_t = solve("fp64", N.CRIT_TRUE, 1e-12)
    out = {"reference_solve": {"precision": "fp64", "criterion": "true residual", "tol": 1e-12,
                               "pcg_iters": st_t.iterations, "rel_residual": st_t.rel_residual}}
    for label, crit in (("rz_1e-4", N.CRIT_RZ), ("true_1e-4", N.CRIT_TRUE)):
        dm, sm = solve("mixed", crit, 1e-4)
        d64, s64 = solve("fp64", crit, 1e-4)
        out[label] = {"dx_rel_err_mixed_vs_fp64": rel(dm, d64), "dx_rel_err_mixed_vs_tight": rel(dm, tight),
                      "dx_rel_err_fp64_vs_tight": rel(d64, tight), "rel_residual_mixed": sm.rel_residual,
                      "rel_residual_fp64": s64.rel_residual}
    g.computeGradientAndHessian()
    dE, dv, _, _ = adjoint.adjoint(g, dLdx, precision="mixed", tol=1e-4, criterion=N.CRIT_RZ)
    g.computeGradientAndHessian()
    dE_t, dv_t, _, _ = adjoint.adjoint(g, dLdx, precision="fp64", tol=1e-12, criterion=N.CRIT_TRUE)
    out["adjoint_mixed_rz_1e-4"] = {"dLdE_rel_err_vs_tight_fp64": rel(dE, dE_t),
                                    "dLdv0_rel_err_vs_tight_fp64": rel(dv, dv_t)}
    return out


def max_over_ranks(values, world, device):
    """The job's times: every rank's device-timed values, maximum over the ranks (each rank
    runs an independent replica of the workload; the whole job takes as long as the
    slowest one)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from sgipc import scenes

    sc = make_scene(args)
    for _ in range(args.warmup):
        cpu_solves(sc, 1)
    times = []
    for _ in range(args.steps):
        times.append(cpu_solves(sc, 1))
    total = sum(times)
    value = args.steps / total
    out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice scenes)",
           "impl": "reference",
           "config": {"workload": WORKLOADS[args.workload],
                      "solver": "reference PCG, FP64 matrix/vectors, FP32 MAS inverses"},
           "cpu_baseline": {"value": value, "unit": "solves/s", "cores": oracle.num_threads(), "kind": "port",
                            "sample": "%d full Newton systems of the workload (assembly + MAS + PCG), %d OpenMP threads"
                                      % (args.steps, oracle.num_threads()), "solver": CPU_SOLVER},
           "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# ------------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from sgipc import adjoint, scenes, system
    from sgipc import _native as N

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    sc, g = make_system(args, local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    cfg = {p: system.PCGSolverConfig(precision=p) for p in ("mixed", "fp64")}
    stream = torch.cuda.current_stream()

    def step(prec):
        g.computeGradientAndHessian()
        return g.calculateMovingDirection(cfg[prec])

    def timed(fn, k):
        """Sum of per-step CUDA-event times; L2 flushed between steps (outside the events)."""
        tot, last = 0.0, None
        for _ in range(k):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            last = fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
        return tot, last

    for p in ("mixed", "fp64"):
        for _ in range(max(3, args.warmup)):
            step(p)
    host = system.HostNewtonState(sc)
    rng = torch.Generator(device="cpu").manual_seed(2)
    dLdx = torch.empty((4, 3 * sc.nv), dtype=torch.float64).uniform_(-1e-3, 1e-3, generator=rng).cuda()

    def adj_step():
        g.computeGradientAndHessian()
        return adjoint.adjoint(g, dLdx, precision="mixed", tol=1e-4, criterion=N.CRIT_RZ)

    for _ in range(max(3, args.warmup)):
        system.step_from_host(g, host, cfg["mixed"])
        adj_step()

    clocks = ClockSampler(local)
    barrier()
    l0 = g.launch_count()
    t_mixed, st_mixed = timed(lambda: step("mixed"), args.steps)
    launches = g.launch_count() - l0
    t_fp64, st_fp64 = timed(lambda: step("fp64"), args.steps)
    t_e2e, _ = timed(lambda: system.step_from_host(g, host, cfg["mixed"]), args.steps)
    t_adj, adj_out = timed(adj_step, args.steps)
    barrier()
    clk = clocks.stop()

    # the same pair of steps stopping on the true relative residual ||b - A dx|| <= 1e-4 ||b||
    # (a quarter of the steps: each takes about twice the iterations)
    k_true = max(1, args.steps // 4)
    cfg_true = {p: system.PCGSolverConfig(precision=p, criterion=N.CRIT_TRUE, max_iter_ratio=1.0)
                for p in ("mixed", "fp64")}

    def step_true(prec):
        g.computeGradientAndHessian()
        return g.calculateMovingDirection(cfg_true[prec])

    for p in ("mixed", "fp64"):
        step_true(p)
    clocks2 = ClockSampler(local)
    barrier()
    t_mixed_true, st_mixed_true = timed(lambda: step_true("mixed"), k_true)
    t_fp64_true, st_fp64_true = timed(lambda: step_true("fp64"), k_true)
    barrier()
    clk2 = clocks2.stop()

    t_mixed, t_fp64, t_e2e, t_adj, t_mixed_true, t_fp64_true = max_over_ranks(
        [t_mixed, t_fp64, t_e2e, t_adj, t_mixed_true, t_fp64_true], world, "cuda")
    units = world * args.steps
    accuracy = step_accuracy(g, sc, system, N, adjoint, dLdx)

    # roofline of the dominant kernel: per-step share = avg launch time x launches per step
    step("mixed")
    torch.cuda.synchronize()
    per_step = {"snk": 1, "gather_blocks": 1, "barrier": 1, "friction": 1, "mas_scatter": 1, "mas_invert": 1,
                "pcg32": max(1, st_mixed.refinements), "energy": 0}
    kern = {}
    for name, cnt in per_step.items():
        try:
            ms, by = g.time_kernel(name, 20)
            kern[name] = {"ms": ms, "bytes": by, "per_step": cnt, "ms_per_step": ms * cnt}
        except Exception as e:  # a kernel not used by this scene
            kern[name] = {"error": str(e)}
    valid = {k: v for k, v in kern.items() if "ms" in v}
    dom = max(valid, key=lambda k: valid[k]["ms_per_step"])
    peak, peak_src = peaks()
    ach = valid[dom]["bytes"] / (valid[dom]["ms"] * 1e-3) / 1e9
    traffic = traffic_table().get(dom)

    out = {"metric": METRIC, "value": units / t_mixed, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * t_mixed / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32",
           "data": "synthetic (seeded lattice scenes)",
           "config": {"workload": WORKLOADS[args.workload], "parallelism": "replicas x%d" % world,
                      "l2": "flushed (256 MiB write) between timed steps",
                      "solver_mixed": "FP32 BSR + FP32 MAS inner PCG, FP64 residual refinement",
                      "pcg_iters_mixed": st_mixed.iterations, "refinements_mixed": st_mixed.refinements,
                      "pcg_iters_fp64": st_fp64.iterations,
                      "rel_residual_mixed": st_mixed.rel_residual, "rel_residual_fp64": st_fp64.rel_residual},
           "fp64": {"value": units / t_fp64, "unit": "solves/s", "ms_per_step": 1e3 * t_fp64 / args.steps},
           "mixed_over_fp64": t_fp64 / t_mixed,
           "true_residual": {"criterion": "||b - A dx|| <= 1e-4 ||b||", "steps": k_true,
                             "mixed": {"value": world * k_true / t_mixed_true, "unit": "solves/s",
                                       "ms_per_step": 1e3 * t_mixed_true / k_true,
                                       "pcg_iters": st_mixed_true.iterations,
                                       "refinements": st_mixed_true.refinements,
                                       "rel_residual": st_mixed_true.rel_residual},
                             "fp64": {"value": world * k_true / t_fp64_true, "unit": "solves/s",
                                      "ms_per_step": 1e3 * t_fp64_true / k_true,
                                      "pcg_iters": st_fp64_true.iterations,
                                      "rel_residual": st_fp64_true.rel_residual},
                             "mixed_over_fp64": t_fp64_true / t_mixed_true, "clocks": clk2},
           "accuracy": accuracy,
           "adjoints": {"value": units / t_adj, "unit": "adjoints/s (4 right-hand sides each)",
                        "ms_per_step": 1e3 * t_adj / args.steps},
           "e2e": {"value": units / t_e2e, "unit": "solves/s", "h2d_bytes_per_step": host.h2d_bytes(),
                   "d2h_bytes_per_step": host.d2h_bytes()},
           "gpu_launches": int(launches),
           "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "peak_source": peak_src,
                        "unit": "GB/s", "frac": ach / peak, "traffic": traffic,
                        "bytes_per_launch": valid[dom]["bytes"], "launch_ms": valid[dom]["ms"]},
           "kernels": {k: {kk: (round(vv, 6) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                       for k, v in kern.items()},
           "clocks": clk}
    # line-search energy (not part of the Newton system): kernels alone, and the C-ABI call
    # with its readback and synchronisation, wall clock
    if "ms" in kern.get("energy", {}):
        ek = kern["energy"]
        tw = []
        for _ in range(25):
            t0 = time.perf_counter()
            g.computeEnergy()
            tw.append(time.perf_counter() - t0)
        out["line_search_energy"] = {"kernels_us": 1e3 * ek["ms"], "call_us": 1e6 * sorted(tw)[len(tw) // 2],
                                     "achieved_GBs": ek["bytes"] / (ek["ms"] * 1e-3) / 1e9}
    # line-search step bound (GIPC::self_largestFeasibleStepSize) along the solve's direction,
    # over the point-triangle and edge-edge pairs of the workload's contact list as candidates
    enc = np.asarray(sc.pairs, np.int32).reshape(-1, 4)
    pt = (enc[:, 0] < 0) & (enc[:, 2] >= 0) & (enc[:, 3] >= 0)
    ee = enc[:, 0] >= 0
    cand = enc[pt | ee].copy()
    mol = cand[:, 0] >= 0
    cand[mol, 3] = np.where(cand[mol, 3] < 0, -cand[mol, 3] - 1, cand[mol, 3])
    if len(cand):
        step("mixed")
        cand_d = torch.tensor(cand, device="cuda")
        tw = []
        for _ in range(25):
            t0 = time.perf_counter()
            alpha = g.self_largestFeasibleStepSize(0.8, g.moveDir, cand_d)
            tw.append(time.perf_counter() - t0)
        out["line_search_ccd"] = {"call_us": 1e6 * sorted(tw)[len(tw) // 2], "candidates": int(len(cand)),
                                  "alpha": alpha}
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle

        nsol = args.cpu_sample or 0
        if nsol <= 0:
            one = cpu_solves(sc, 1)
            nsol = max(1, min(20, int(10.0 / max(one, 1e-3))))
        t_cpu = cpu_solves(sc, nsol)
        out["cpu_baseline"] = {"value": nsol / t_cpu, "unit": "solves/s", "cores": oracle.num_threads(),
                               "kind": "port", "sample": "%d full Newton systems of the workload" % nsol,
                               "solver": CPU_SOLVER}
    g.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


def phase_table(stamps, phases):
    """Per-phase timing of one persistent solve from its barrier stamps: for every phase, the
    critical path (the last CTA's release from the previous barrier to the last CTA's
    arrival), the barrier latency (last arrival to last release), the mean CTA's busy time
    and the CTA that arrived last most often."""
    arrive, leave = stamps[:, :, 0], stamps[:, :, 1]
    out = {}
    for e in range(1, stamps.shape[1]):
        name = phases[e]
        crit = float(arrive[:, e].max() - leave[:, e - 1].max())
        lat = float(leave[:, e].max() - arrive[:, e].max())
        busy = float(np.mean(arrive[:, e] - leave[:, e - 1]))
        d = out.setdefault(name, {"count": 0, "crit_ns": 0.0, "barrier_ns": 0.0, "busy_ns": 0.0, "last": {}})
        d["count"] += 1
        d["crit_ns"] += crit
        d["barrier_ns"] += lat
        d["busy_ns"] += busy
        last = int(np.argmax(arrive[:, e]))
        d["last"][last] = d["last"].get(last, 0) + 1
    total = float(leave[:, -1].max() - arrive[:, 0].min())
    table = {"total_us": total / 1e3, "grid": int(stamps.shape[0]), "barriers": int(stamps.shape[1] - 1),
             "load_us": float(leave[:, 0].max() - arrive[:, 0].min()) / 1e3, "phases": {}}
    for name, d in out.items():
        n = d["count"]
        top = max(d["last"].items(), key=lambda kv: kv[1])
        table["phases"][name] = {"count": n, "crit_us": d["crit_ns"] / n / 1e3, "barrier_us": d["barrier_ns"] / n / 1e3,
                                 "busy_mean_us": d["busy_ns"] / n / 1e3, "total_us": (d["crit_ns"] + d["barrier_ns"]) / 1e3,
                                 "last_cta": top[0], "last_cta_share": top[1] / n}
    return table


def run_pcg_phases(args):
    """Barrier-stamp profile of the persistent PCG solve on the workload (one GPU)."""
    import torch

    from sgipc import system

    torch.cuda.set_device(0)
    sc, g = make_system(args, 0)
    out = {"workload": WORKLOADS[args.workload]}
    for prec, names in (("mixed", ("pcg32", "pcg32x4")), ("fp64", ("pcg64", "pcg64x4"))):
        g.computeGradientAndHessian()
        g.calculateMovingDirection(system.PCGSolverConfig(precision=prec))
        for name in names:
            for _ in range(3):  # warm-up
                g.profile_pcg(name)
            reps = [phase_table(*g.profile_pcg(name)) for _ in range(5)]
            best = min(reps, key=lambda t: t["total_us"])
            best["total_us_all"] = [round(t["total_us"], 1) for t in reps]
            out[name] = best
    g.close()
    print(json.dumps(out, indent=1))
    return 0


def run_kernel_only(args):
    """Assemble the workload, build the MAS in the precision the kernel reads, then time the
    named kernel with sgipc_time_kernel (one untimed launch, then args.steps timed ones)."""
    import torch

    from sgipc import system

    torch.cuda.set_device(0)
    sc, g = make_system(args, 0)
    g.computeGradientAndHessian()
    system.MASPreconditioner(g).setPreconditioner("fp64" if args.kernel in ("pcg64", "mas_domain64") else "mixed")
    ms, by = g.time_kernel(args.kernel, args.steps)
    g.close()
    print(json.dumps({"kernel": args.kernel, "launches": args.steps + 1, "avg_ms": ms, "bytes_per_launch": by,
                      "achieved_GBs": by / (ms * 1e-3) / 1e9}))
    return 0


def run_timeline(args):
    """Where one Newton system's time goes, on the caller's stream (one GPU): CUDA events at the
    step's start, after the assembly (the right-hand side, which joins the contact and element
    streams), after the MAS build and after the PCG solve; and the host's time inside
    sgipc_assemble.  Medians over args.steps steps, L2 flushed before each."""
    import torch

    from sgipc import system

    torch.cuda.set_device(0)
    sc, g = make_system(args, 0)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    out = {"workload": WORKLOADS[args.workload]}
    for prec in ("mixed", "fp64"):
        cfg = system.PCGSolverConfig(precision=prec)
        mas = system.MASPreconditioner(g)
        solver = system.PCGSolver(g, cfg)
        rows = []
        for k in range(args.warmup + args.steps):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            t0 = time.perf_counter()
            g.computeGradientAndHessian()
            t_host = time.perf_counter() - t0
            ev[1].record(stream)
            mas.setPreconditioner(prec)
            ev[2].record(stream)
            _, st = solver.solve(g.rhs())
            ev[3].record(stream)
            ev[3].synchronize()
            if k >= args.warmup:
                rows.append([ev[0].elapsed_time(ev[1]), ev[0].elapsed_time(ev[2]), ev[0].elapsed_time(ev[3]),
                             1e3 * t_host, st.iterations])
        r = np.median(np.array(rows), axis=0)
        out[prec] = {"assembly_end_ms": r[0], "mas_end_ms": r[1], "solve_end_ms": r[2], "assemble_host_ms": r[3],
                     "pcg_iters": int(r[4])}
        # the same step with the stream held by a ~0.5 ms spin first, so that the host has
        # enqueued the whole assembly before it starts: the device-side times alone
        gpu = []
        for k in range(args.warmup + args.steps):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            torch.cuda._sleep(1_000_000)
            ev[0].record(stream)
            g.computeGradientAndHessian()
            ev[1].record(stream)
            mas.setPreconditioner(prec)
            ev[2].record(stream)
            solver.solve(g.rhs())
            ev[3].record(stream)
            ev[3].synchronize()
            if k >= args.warmup:
                gpu.append([ev[0].elapsed_time(ev[1]), ev[0].elapsed_time(ev[2]), ev[0].elapsed_time(ev[3])])
        r = np.median(np.array(gpu), axis=0)
        out[prec]["enqueued_ahead"] = {"assembly_end_ms": r[0], "mas_end_ms": r[1], "solve_end_ms": r[2]}
    g.close()
    print(json.dumps(out))
    return 0


def run_abd_bed(args):
    """The affine-bodies-on-a-bed workload on one GPU: Newton systems per second of the coupled
    FEM + ABD system (GlobalLinearSystem), FP64 MAS inverses vs FP32 ones (the reference's
    shipping mix); the coupled solve has no FP32-vector mode."""
    import torch

    from sgipc import abd, scenes, system
    from sgipc import _native as N

    torch.cuda.set_device(0)
    sc, bodies = scenes.scene_abd_on_bed(500, contacts=False)
    g = system.GIPC(sc, device=0, pair_capacity=400_000)
    g.buildCP(body=torch.tensor(sc.body_of_vertex, dtype=torch.int32, device="cuda"))
    af = bodies["abd_first"]
    g.computeGradientAndHessian()
    part = g.contactPartition(af)
    cap = 2 * max(part["abd_blocks"][0].numel(), part["fem_blocks"][0].numel(), 1)
    sysm = abd.ABDSystem(bodies, max_abd_blocks=cap, max_fem_blocks=cap)
    q = torch.tensor(bodies["q"], device="cuda")
    qt = torch.tensor(bodies["q_tilde"], device="cuda")
    gls = abd.GlobalLinearSystem(g, sysm)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def step(prec, tol=1e-4, crit=N.CRIT_RZ, ratio=0.3):
        g.computeGradientAndHessian()
        pt = g.contactPartition(af, cap)
        sysm.setup_abd_system_gradient_hessian(q, qt, bodies["kappa"], bodies["dt"], point_grad=pt["point_grad"],
                                               abd_blocks=pt["abd_blocks"], fem_blocks=pt["fem_blocks"],
                                               fem_boundary=g.tet.BoundaryType)
        abd.ABDPreconditioner(sysm).assemble()
        system.MASPreconditioner(g).setPreconditioner(prec)
        return gls.solve_linear_system(gls.right_hand_side(), tol=tol, criterion=crit, max_iter_ratio=ratio)

    out = {"metric": METRIC, "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (MAS f64 / f32)",
           "data": "synthetic (seeded lattice bed, seeded boxes)",
           "config": {"workload": WORKLOADS["abd_bed"], "l2": "flushed (256 MiB write) between timed steps",
                      "contact_pairs": int(g.tet.pairs.shape[0]), "abd_abd_blocks": int(part["abd_blocks"][0].numel()),
                      "abd_fem_blocks": int(part["fem_blocks"][0].numel())}}
    xs = {}
    for prec in ("fp64", "ref"):
        for _ in range(max(3, args.warmup)):
            step(prec)
        tot, st = 0.0, None
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            x, _, st = step(prec)
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
        xs[prec] = x.clone()
        out[prec] = {"value": args.steps / tot, "ms_per_step": 1e3 * tot / args.steps, "pcg_iters": st.iterations,
                     "rel_residual": st.rel_residual}
    tight, _, st_t = step("fp64", 1e-10, N.CRIT_TRUE, 2.0)
    out["value"] = out["ref"]["value"]
    out["ms_per_step"] = out["ref"]["ms_per_step"]
    out["ref_over_fp64"] = out["ref"]["value"] / out["fp64"]["value"]
    out["accuracy"] = {"reference_solve": {"precision": "fp64", "criterion": "true residual", "tol": 1e-10,
                                           "pcg_iters": st_t.iterations, "rel_residual": st_t.rel_residual},
                       "dx_rel_err_ref_vs_fp64": float((xs["ref"] - xs["fp64"]).norm() / xs["fp64"].norm()),
                       "dx_rel_err_fp64_vs_tight": float((xs["fp64"] - tight).norm() / tight.norm()),
                       "dx_rel_err_ref_vs_tight": float((xs["ref"] - tight).norm() / tight.norm())}
    sysm.close()
    g.close()
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.pcg_phases:
        return run_pcg_phases(args)
    if args.kernel:
        return run_kernel_only(args)
    if args.timeline:
        return run_timeline(args)
    if args.workload == "abd_bed":
        return run_abd_bed(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
