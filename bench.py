"""Benchmark: Brownian rigid-body time steps (body-steps/s) of the FCM mobility
solve on B200, headline = mixed-precision solver, beside the plain FP64 GPU path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload clusters32768_phi0.20_g512] [--algorithm em|gdc]

Default workload: the largest single-GPU configuration, 32,768 rigid 12-blob
random clusters, each of its own shape (393,216 blobs), volume fraction 0.20,
512^3 grid, equilibrated by 10^4 Metropolis steps on the device (untimed).
One step = one Euler-Maruyama time step (main.cpp:222-451): Philox
fluctuating field, random blob velocities, steric forces, right-preconditioned
GMRES of the rigid saddle-point system to the workload's tolerance, body
update.  N > 1 runs N independent replicas, one per GPU (the solve does not
shard; no collective on the data path), value = all replicas' body-steps / the
slowest rank's time; the ensemble workload instead splits its 64 instances
across the ranks.  --impl reference times whole steps of the CPU FP64 oracle
(the reference's algorithm restated, all host threads) on the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-steps/s, mixed vs FP64 GPU at <=1e-6 rel vel error; spread/interp HBM GB/s"
UNIT = "body-steps/s"
# The mixed-precision solver refines to a 1e-8 relative residual (the FP64 path
# solves to the workload's 1e-10); its velocity error against the FP64 solve is
# measured in every run and must stay <= 1e-6.
MIXED_TOL = 1e-8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clusters32768_phi0.20_g512")
    ap.add_argument("--algorithm", default="em", choices=["em", "gdc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default kernel variants instead of fcm_autotune's choice")
    ap.add_argument("--ens-modes", default="fp64,fp64_graph,fp64_many,fp64_batch,mixed_batch,mixed",
                    help="ensemble arms to time (the JSON line needs fp64, fp64_graph and mixed)")
    ap.add_argument("--nvtx", action="store_true", help="mark the timed region with an NVTX range 'timed'")
    ap.add_argument("--mixed-tol", type=float, default=None,
                    help="refinement tolerance of the mixed-precision solver (default %g)" % MIXED_TOL)
    ap.add_argument("--step-mode", default="graph", choices=["graph", "host"],
                    help="mixed arm: device-resident graph steps (default) or host-driven fcm_step, whose "
                         "kernels a profiler can list one by one")
    ap.add_argument("--kernels-only", type=int, default=0, metavar="R",
                    help="profiling mode: R FP64 spread+interp launches and R FP32 mobility products, no steps")
    ap.add_argument("--kernels-precision", type=int, default=None, choices=[0, 1],
                    help="--kernels-only: run only this precision's grid (0 FP64, 1 FP32)")
    ap.add_argument("--variants", default=None,
                    help="--kernels-only: six comma-separated kernel variants (fcm_set_variants) to run")
    ap.add_argument("--ref-budget", type=float, default=180.0,
                    help="--impl reference: seconds of whole oracle steps to time at most (at least one step)")
    ap.add_argument("--no-step-errors", action="store_true",
                    help="skip the untimed replay that measures the mixed-vs-FP64 velocity error of every timed step")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(t, device="cuda"):
    """Slowest rank's time (all_reduce MAX); t itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(t)
    tt = torch.tensor([float(t)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(bodies_per_replica, steps, world, t_max):
    """Whole-job body-steps/s of `world` independent replicas."""
    return world * bodies_per_replica * steps / t_max


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:  # first sample before the timed region
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- ours
VARIANT_LEGEND = ("variants [FP64 spread, FP64 solve, FP32 spread, FP32 solve, FP64 interp, FP32 interp]: spread "
                  "0 persistent pipelined, 1 / 2 / 3 one CTA per tile staging 16 / 8 / 32 blobs per round, 4 "
                  "one warp per tile (two y-rows per lane), 5 one warp per tile on the tensor cores (3xTF32, FP32 "
                  "only); solve 0 cuFFT 3D + projection, 1 cuFFT (y, z) + fused x-transform, "
                  "2 library (y, z) + fused x-transform; interp 0 shuffle reduction with 64 threads per tile, 1 "
                  "one warp per tile (two y-rows per lane) with the shuffle reduction, 2 one warp per tile with "
                  "a shared-memory reduction, 3 one warp per tile on the tensor cores (3xTF32, FP32 only).  "
                  "us[16P + v]: precision P, v 0-5 spread, 6-8 solve, 9-12 interp variants, microseconds per "
                  "call, -1 not available")

AUTOTUNE = {"on": True}


def setup_suspension(p, ref, x, q, fe, stream, tune=True):
    """A context for the workload (per-body shapes with their analytic
    preconditioner blocks, or the shared shape with its probed reference
    matrices); unless --no-autotune, its kernel variants are chosen by
    fcm_autotune on the start configuration (untimed; s.tuning holds the
    variants and the microseconds per call of each candidate)."""
    from timstochrigidbodiessim_b200 import configs
    s = configs.make_suspension(p, ref, stream=stream)
    s.set_bodies(x, q)
    s.set_external_forces(fe)
    if not configs.has_body_shapes(p, ref):
        s.produce_reference_matrices()
    s.tuning = None
    if AUTOTUNE["on"] and tune:
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        v, us = s.autotune(reps=3)
        s.tuning = {"variants": v, "us": [round(float(t), 1) for t in us]}
    return s


def run_step(s, seed, index, mode):
    """One step: host-driven (fcm_step) or device-resident (fcm_step_async + wait)."""
    if mode == "graph":
        s.step_async(seed, index)
        return s.step_wait()
    return s.step(seed, index)


def timed_steps(s, K, seed, start_index, stream, mode="host"):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    iters = []
    e0.record(stream)
    for i in range(K):
        st, info = run_step(s, seed, start_index + i, mode)
        iters.append(info.gmres_iters)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, iters


def profiled_traffic(workload):
    """DRAM bytes per launch of each spread / interpolation kernel of `workload`
    from the ncu capture summarised in profiles/traffic.txt ({kernel: bytes})."""
    out = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", "traffic.txt")):
            f = line.split()
            if len(f) == 3 and not line.startswith("#") and f[0] == workload:
                out[f[1]] = float(f[2])
    except OSError:
        pass
    return out


def kernel_roofline(s, p, stream, precision, reps=20):
    """Per-launch durations of the spread and the interpolation on the grid of one
    precision (0 FP64, 1 FP32), CUDA events on the context's stream around the
    stage calls fcm_spread / fcm_interp (device F and V, no copies inside);
    algorithmic bytes 3*G*s + 6*Nb*s per launch (s = 8 or 4)."""
    import torch
    Nb = p.num_blobs
    F = torch.randn(3 * Nb, dtype=torch.float64, device="cuda")
    V = torch.empty(3 * Nb, dtype=torch.float64, device="cuda")
    s.fill_all_blob_pos()
    s.set_up_gaussians()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    for _ in range(3):
        s.spread(F, precision)
        s.interp(precision, out=V)
    torch.cuda.synchronize()
    ts, ti = [], []
    for _ in range(reps):
        ev[0].record(stream)
        s.spread(F, precision)
        ev[1].record(stream)
        s.interp(precision, out=V)
        ev[2].record(stream)
        ev[2].synchronize()
        ts.append(ev[0].elapsed_time(ev[1]) / 1e3)
        ti.append(ev[1].elapsed_time(ev[2]) / 1e3)
    G = p.nx * p.ny * p.nz
    sz = 8 if precision == 0 else 4
    bytes_ = 3 * G * sz + 6 * Nb * sz
    return bytes_, float(np.mean(ts)), float(np.mean(ti))


def rel_vel_error(p, ref, x, q, fe, stream):
    """Body (and blob) velocity error of the mixed-precision solve against the
    FP64 solve on the same deterministic right-hand side."""
    sols = []
    for prec in (0, 1):
        pp = p.copy(precision=prec, noise=0)
        if prec == 1:
            pp.gmres_tol = MIXED_TOL
        s = setup_suspension(pp, ref, x, q, fe, stream)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.calculate_forces()
        s.assemble_RHS()
        st, soln, it, rel = s.invert_saddle_point_system()
        sols.append(soln)
        s.close()
    Nb = p.num_blobs
    U64, U32 = sols[0][3 * Nb:], sols[1][3 * Nb:]
    L64, L32 = sols[0][:3 * Nb], sols[1][:3 * Nb]
    return (float(np.linalg.norm(U32 - U64) / np.linalg.norm(U64)),
            float(np.linalg.norm(L32 - L64) / np.linalg.norm(L64)))


def step_velocity_errors(p, ref, x, q, fe, seed, start, K, stream, variants=None):
    """Relative body- and blob-velocity error of the mixed-precision step against
    the FP64 step on each of K steps of the mixed trajectory, replayed untimed
    from the state the timed region started from (step indices start ..
    start + K - 1; host-driven steps reproduce the graph steps bit for bit).  At
    every step both contexts hold the same bodies and draw the same Philox noise
    (seed, index); each forms its own random velocities (FP32 grid in the mixed
    context), forces and RHS, and solves (FP64 to the workload's tolerance, mixed
    with FP64 refinement to MIXED_TOL); the mixed context then advances with its
    own solution and the FP64 context takes its bodies.  variants ({precision:
    kernel variants}) gives each context the kernels its timed arm ran with.
    Returns per-step lists (bodies, blobs)."""
    ctx = {}
    for prec in (0, 1):
        pp = p.copy(precision=prec)
        if prec == 1:
            pp.gmres_tol = MIXED_TOL
        ctx[prec] = setup_suspension(pp, ref, x, q, fe, stream, tune=False)
        if variants and variants.get(prec):
            ctx[prec].set_variants(variants[prec])
    Nb = p.num_blobs
    eU, eL = [], []
    for k in range(K):
        sol = {}
        for prec, s in ctx.items():
            s.fill_all_blob_pos()
            s.produce_random_velocity_field(seed, start + k)
            s.set_up_gaussians()
            s.calculate_random_blob_velocities()
            s.calculate_forces()
            s.assemble_RHS()
            st, soln, it, rel = s.invert_saddle_point_system()
            sol[prec] = soln
        U64, U32 = sol[0][3 * Nb:], sol[1][3 * Nb:]
        L64, L32 = sol[0][:3 * Nb], sol[1][:3 * Nb]
        eU.append(float(np.linalg.norm(U32 - U64) / np.linalg.norm(U64)))
        eL.append(float(np.linalg.norm(L32 - L64) / np.linalg.norm(L64)))
        ctx[1].end_of_step_update(U32, 1.0)
        xb, qb = ctx[1].get_bodies()
        ctx[0].set_bodies(xb, qb)
    for s in ctx.values():
        s.close()
    return eU, eL


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or None."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(p, ref, x, q, fe, gmres_iters):
    """The CPU oracle (the reference's algorithm restated, FP64) on a bounded
    sample of the same workload: one fluctuating-field solve plus one saddle-point
    product (spread, FFT solve, interpolation, K, K^T, P^-1).  A step is
    estimated as noise + (iters + 2) products, iters = the FP64 GPU path's GMRES
    iteration count on this workload."""
    from tests.oracle_lib import Oracle, lib
    from timstochrigidbodiessim_b200 import configs
    threads = os.cpu_count() or 1
    lib().orc_set_threads(threads)
    o = configs.make_suspension(p, ref, cls=Oracle)
    o.set_bodies(x, q)
    o.set_external_forces(fe)
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    n = p.system_size
    v = np.random.default_rng(0).standard_normal(n)
    t0 = time.perf_counter()
    o.produce_random_velocity_field(1234, 0)
    o.calculate_random_blob_velocities()
    o.calculate_forces()
    t1 = time.perf_counter()
    o.multiply_by_saddle_point_matrix(o.multiply_by_Pinv(v))
    t2 = time.perf_counter()
    t_step = (t1 - t0) + (gmres_iters + 2) * (t2 - t1)
    o.close()
    return {"value": p.num_bodies / t_step, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
            "sample": "bounded sample: 1 fluctuating field + forces (%.2fs) and 1 preconditioned saddle-point "
                      "product (%.2fs) of the same workload, FP64, scaled to a step as noise + (%.1f GMRES iters "
                      "+ 2) products; bench.py --impl reference times whole oracle steps" %
                      (t1 - t0, t2 - t1, gmres_iters)}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from timstochrigidbodiessim_b200 import capi, configs

    rank, world, local = dist_env()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    lib = capi.load()
    algorithm = 1 if args.algorithm == "gdc" else 2
    seed = 1234 + rank
    p, ref, x, q, fe = configs.workload(args.workload, seed=seed, algorithm=algorithm)
    mcmc = None
    steps_eq = configs.WORKLOADS[args.workload].get("mcmc_steps", 0)
    if steps_eq:  # Metropolis equilibration of the start (untimed)
        x, q, st = configs.equilibrate(p, ref, x, q, steps_eq, seed=seed, stream=stream)
        mcmc = {"steps": int(st.steps), "scale": st.scale, "acceptance_ratio": st.acceptance_ratio,
                "potential": st.potential}
    results = {}
    for tag, prec, mode in (("fp64", 0, "host"), ("fp64_graph", 0, "graph"), ("mixed", 1, args.step_mode)):
        pp = p.copy(precision=prec)
        if prec == 1:
            pp.gmres_tol = MIXED_TOL
        s = setup_suspension(pp, ref, x, q, fe, stream)
        for i in range(args.warmup):
            run_step(s, seed, i, mode)
        start_state = s.get_bodies() if tag == "mixed" else None  # for the untimed error replay
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        if tag == "mixed":
            sampler.start()
        l0 = lib.fcm_kernel_launch_count()
        t, iters = timed_steps(s, args.steps, seed, args.warmup, stream, mode)
        l1 = lib.fcm_kernel_launch_count()
        clocks = sampler.stop() if tag == "mixed" else None
        torch.cuda.synchronize()
        t = max_over_ranks(t)
        if world > 1:
            dist.barrier()
        results[tag] = dict(t=t, iters=float(np.mean(iters)), launches=l1 - l0, clocks=clocks, s=s, tuning=s.tuning,
                            start=start_state)
    # rooflines of the spread / interpolation kernels on the FP32 grid (the mixed
    # path's) and the FP64 grid
    kr = {"fp32": kernel_roofline(results["mixed"]["s"], p, stream, 1),
          "fp64": kernel_roofline(results["fp64"]["s"], p, stream, 0)}
    # end to end through the C-ABI with host buffers: H2D bodies, step, D2H bodies;
    # the timed steps replayed from their start state (same bodies, same noise
    # indices, so the same solver work as those steps)
    sm = results["mixed"]["s"]
    xs, qs = results["mixed"]["start"]
    sm.set_bodies(xs, qs)
    sm.fill_all_blob_pos()
    sm.list_populate()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    K2 = args.steps
    e2e_iters = []
    e0.record(stream)
    for i in range(K2):
        sm.set_bodies(xs, qs)
        st_, info_ = run_step(sm, seed, args.warmup + i, args.step_mode)
        e2e_iters.append(info_.gmres_iters)
        xs, qs = sm.get_bodies()
    e1.record(stream)
    e1.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    for r in results.values():  # free the grids before the replay contexts are made
        r["s"].close()
    err_U, err_l = rel_vel_error(p, ref, x, q, fe, stream) if rank == 0 else (None, None)
    step_err = None
    if rank == 0 and not args.no_step_errors:
        x0, q0 = results["mixed"]["start"]
        tuned = {prec: (results[tag]["tuning"] or {}).get("variants") for prec, tag in ((0, "fp64"), (1, "mixed"))}
        eU, eL = step_velocity_errors(p, ref, x0, q0, fe, seed, args.warmup, args.steps, stream, tuned)
        step_err = {"steps": len(eU), "bodies": {"max": max(eU), "mean": float(np.mean(eU))},
                    "blobs": {"max": max(eL), "mean": float(np.mean(eL))},
                    "variants": tuned,
                    "what": "every timed step replayed untimed with the timed arms' kernel variants: the mixed "
                            "step's body and blob velocities against the FP64 step's on the same bodies and "
                            "Philox noise"}
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured"
    if not hbm:
        hbm, peak_src = 6650.0, "fallback"
    M, K = p.num_bodies, args.steps
    value = replica_throughput(M, K, world, results["mixed"]["t"])
    fp64_value = replica_throughput(M, K, world, results["fp64"]["t"])
    fp64g_value = replica_throughput(M, K, world, results["fp64_graph"]["t"])
    if rank == 0:
        traffic = profiled_traffic(args.workload)
        kernels = []
        for tag in ("fp32", "fp64"):
            bytes_, t_spread, t_interp = kr[tag]
            for name, t_k in (("spread", t_spread), ("interp", t_interp)):
                ach = bytes_ / t_k / 1e9
                kernels.append({"kernel": "fcm %s (%s)" % (name, tag), "bytes_per_launch": bytes_,
                                "ms_per_launch": 1e3 * t_k, "achieved": ach, "frac": ach / hbm,
                                "traffic": traffic.get("%s_%s" % (name, tag)),
                                "stencil_touches_per_s": p.num_blobs * p.ngauss ** 3 / t_k})
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(p, ref, x, q, fe, results["fp64"]["iters"])
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": K,
            "warmup": args.warmup,
            "ms_per_step": 1e3 * results["mixed"]["t"] / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 grid + f64 refinement",
            "data": "synthetic (seeded random rods, Philox noise)",
            "config": {"workload": args.workload, "bodies": M, "blobs_per_body": p.blobs_per_body,
                       "grid": [p.nx, p.ny, p.nz], "box": p.box[0], "algorithm": args.algorithm,
                       "gmres_tol": p.gmres_tol, "parallelism": "replicas x%d" % world,
                       "l2": "grid fields (3x%d^3) exceed L2; no flush needed" % p.nx,
                       "mcmc_equilibration": mcmc,
                       "kernel_variants": {"legend": VARIANT_LEGEND, "fp64": results["fp64"]["tuning"],
                                           "mixed": results["mixed"]["tuning"]}},
            "fp64": {"value": fp64_value, "ms_per_step": 1e3 * results["fp64"]["t"] / K,
                     "gmres_iters": results["fp64"]["iters"], "mode": "host-driven fcm_step"},
            "fp64_graph": {"value": fp64g_value, "ms_per_step": 1e3 * results["fp64_graph"]["t"] / K,
                           "mode": "device-resident graph steps"},
            "mixed_over_fp64": value / fp64_value,
            "mixed_over_fp64_graph": value / fp64g_value,
            "gmres_iters_mixed": results["mixed"]["iters"],
            "mixed_gmres_tol": MIXED_TOL,
            "tolerances": "the FP64 arms solve to a %g relative residual, the mixed arm refines to %g "
                          "(FP32 grid GMRES inside FP64 iterative refinement)" % (p.gmres_tol, MIXED_TOL),
            "rel_vel_error_mixed_vs_fp64": {"per_step": step_err,
                                            "start_rhs": {"bodies": err_U, "blobs": err_l,
                                                          "what": "one deterministic solve of the start "
                                                                  "configuration's RHS"}},
            "roofline": dict(max((k for k in kernels if k["kernel"].endswith("(fp32)")),
                                 key=lambda k: k["ms_per_launch"]),
                             bound="hbm", peak=hbm, unit="GB/s", peak_source=peak_src,
                             note="the mixed step's longest own grid kernel; at high blob density per 8^3 "
                                  "tile it is bound by instruction issue (FMAs per (blob, tile) pair), not HBM"),
            "roofline_kernels": kernels,
            "cpu_baseline": cpu,
            "e2e": {"value": replica_throughput(M, K2, world, t_e2e), "unit": UNIT, "h2d_bytes_per_step": 7 * 8 * M,
                    "d2h_bytes_per_step": 7 * 8 * M, "steps": K2, "gmres_iters": float(np.mean(e2e_iters)),
                    "what": "the timed steps replayed from their start state through the C-ABI with host body "
                            "arrays: H2D bodies, graph step, D2H bodies"},
            "gpu_launches": results["mixed"]["launches"],
            "clocks": results["mixed"]["clocks"],
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------- reference
def run_reference(args):
    """Whole time steps of the CPU FP64 oracle (the reference's algorithm
    restated: Philox stress through the polar method, spread, FFT solve,
    interpolation, steric forces, right-preconditioned GMRES to the workload's
    tolerance, body update; main.cpp:222-451) on all host threads, from the same
    start configuration as the GPU arm before its Metropolis equilibration (that
    equilibration would take the oracle far longer than the bench may run).
    Whole steps are timed one after another until --steps are done or
    --ref-budget seconds are spent (at least one); the steps actually timed are
    in the line.  One saddle-point product is also timed on one thread and on all
    threads, and the single-thread figure (one reference MPI rank,
    run_rigid_bodies_sim.sh:15) is the whole-step figure scaled by that ratio,
    labelled as derived."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from tests.oracle_lib import Oracle, lib
    from timstochrigidbodiessim_b200 import configs
    threads = os.cpu_count() or 1
    lib().orc_set_threads(threads)
    algorithm = 1 if args.algorithm == "gdc" else 2
    seed = 1234
    p, ref, x, q, fe = configs.workload(args.workload, seed=seed, algorithm=algorithm)
    t0 = time.perf_counter()
    o = configs.make_suspension(p, ref, cls=Oracle)
    o.set_bodies(x, q)
    o.set_external_forces(fe)
    if not configs.has_body_shapes(p, ref):
        o.produce_reference_matrices()
    t_setup = time.perf_counter() - t0
    budget = max(0.0, args.ref_budget)
    # one saddle-point product on all threads sizes the run: a step is about 30
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    v = np.random.default_rng(0).standard_normal(p.system_size)
    t0 = time.perf_counter()
    o.multiply_by_saddle_point_matrix(o.multiply_by_Pinv(v))
    t_all = time.perf_counter() - t0
    # untimed warm-up steps only where they cost a small part of the budget
    warm = args.warmup if 30.0 * t_all * args.warmup < 0.25 * budget else 0
    for i in range(warm):
        o.step(seed, i)
    t_start = time.perf_counter()
    ts, iters = [], []
    for k in range(args.steps):
        if ts and time.perf_counter() - t_start + np.mean(ts) > budget:
            break
        t0 = time.perf_counter()
        st, info = o.step(seed, warm + k)
        ts.append(time.perf_counter() - t0)
        iters.append(info.gmres_iters)
    t_step = float(np.mean(ts))
    value = p.num_bodies / t_step
    # thread scaling of one saddle-point product of the same workload
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    lib().orc_set_threads(1)
    t0 = time.perf_counter()
    o.multiply_by_saddle_point_matrix(o.multiply_by_Pinv(v))
    t_one = time.perf_counter() - t0
    lib().orc_set_threads(threads)
    o.close()
    desc = ("%d whole EM step(s) of the CPU FP64 oracle timed (%d untimed warm-up), %.1f GMRES iterations per "
            "step to tol %g, %d threads; set-up (%.1fs) untimed" % (len(ts), warm, float(np.mean(iters)),
                                                                    p.gmres_tol, threads, t_setup))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": len(ts),
        "steps_requested": args.steps, "warmup": warm, "ms_per_step": 1e3 * t_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the GPU arm's workload and seed, before its Metropolis equilibration)",
        "config": {"workload": args.workload, "bodies": p.num_bodies, "blobs_per_body": p.blobs_per_body,
                   "grid": [p.nx, p.ny, p.nz], "algorithm": args.algorithm, "gmres_tol": p.gmres_tol},
        "gmres_iters": float(np.mean(iters)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
                         "cpu": cpu_model()},
        "single_thread": {"value": value * t_all / t_one, "unit": UNIT, "cores": 1,
                          "derived": "whole-step figure x (one saddle-point product on all threads %.2fs / on one "
                                     "thread %.2fs)" % (t_all, t_one)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_kernels_only(args):
    import torch
    from timstochrigidbodiessim_b200 import configs
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    p, ref, x, q, fe = configs.workload(args.workload)
    for prec in ((0, 1) if args.kernels_precision is None else (args.kernels_precision,)):
        s = configs.make_suspension(p.copy(precision=prec), ref, stream=stream)
        if args.variants:
            s.set_variants([int(v) for v in args.variants.split(",")])
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        F = torch.randn(3 * p.num_blobs, dtype=torch.float64, device="cuda")
        V = torch.empty_like(F)
        for _ in range(args.kernels_only):
            s.spread(F, prec)
            s.stokes_solve(prec)
            s.interp(prec, out=V)
        torch.cuda.synchronize()
        s.close()
    print(json.dumps({"kernels_only": args.kernels_only, "workload": args.workload}))


def ensemble_shard(n_instances, rank, world):
    """Instances of rank `rank` out of `world`: rank, rank + world, ... (every
    instance exactly once over the ranks; no data is exchanged)."""
    return list(range(rank, n_instances, world))


def run_ensemble(args):
    """Ensemble of 64 independent suspensions (seeds 0..63).  Arms, each with the
    same instances and steps:
      fp64        instances one after another on one stream, host-driven fcm_step;
      fp64_graph  instances one after another, device-resident graph steps;
      fp64_many   64 contexts on 64 streams, one graph per instance step
                  (fcm_step_many): the concurrency the mixed arm gets;
      fp64_batch  one FP64 fcm_batch (lockstep batched solves, one graph per step);
      mixed_batch the same batch with FP32 grids inside FP64 refinement;
      mixed       (the line's value) fcm_step_many over 64 mixed contexts.
    With N ranks each takes instances rank, rank + N, ... (no collective on the
    data path); value = all instances' body-steps / the slowest rank's device
    time.  Device time: events on a root stream that every instance stream joins."""
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")  # streams -> hardware queues
    from timstochrigidbodiessim_b200 import configs
    rank, world, local = dist_env()
    all_insts = configs.ensemble(64, workers=min(16, os.cpu_count() or 1))  # before any CUDA call
    mine = ensemble_shard(len(all_insts), rank, world)
    insts = [all_insts[i] for i in mine]
    import torch
    import torch.distributed as dist
    from timstochrigidbodiessim_b200 import capi
    from timstochrigidbodiessim_b200.fcm import Batch, step_many
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    lib = capi.load()
    root = torch.cuda.current_stream()
    total_bodies = sum(p.num_bodies for p, *_ in all_insts)
    seeds = [i for i in mine]
    res = {}
    modes = (("fp64", 0, "host"), ("fp64_graph", 0, "graph"), ("fp64_many", 0, "many"), ("fp64_batch", 0, "batch"),
             ("mixed_batch", 1, "batch"), ("mixed", 1, "many"))
    wanted = set(args.ens_modes.split(","))
    for tag, prec, mode in modes:
        if tag not in wanted:
            continue
        streams = [torch.cuda.Stream() for _ in insts] if mode == "many" else [torch.cuda.Stream()] * len(insts)
        batch = None
        if mode == "batch":
            pps = []
            for p, ref, x, q, fe in insts:
                pp = p.copy(precision=prec)
                if prec == 1:
                    pp.gmres_tol = MIXED_TOL
                pps.append((pp, ref))
            batch = Batch(pps, stream=streams[0])
            for m, (p, ref, x, q, fe) in zip(batch.members, insts):
                m.set_bodies(x, q)
                m.set_external_forces(fe)
                m.produce_reference_matrices()
            ss = batch.members
        else:
            ss = []
            for (p, ref, x, q, fe), st in zip(insts, streams):
                pp = p.copy(precision=prec)
                if prec == 1:
                    pp.gmres_tol = MIXED_TOL
                ss.append(setup_suspension(pp, ref, x, q, fe, st))
        for i in range(args.warmup):
            if mode == "batch":
                batch.step(seeds, i)
            elif mode == "many":
                step_many(ss, seeds, i)
            else:
                for k, s in enumerate(ss):
                    if mode == "graph":
                        s.step_async(seeds[k], i)
                        s.step_wait()
                    else:
                        s.step(seeds[k], i)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local)
        if tag == "mixed":
            sampler.start()
        l0 = lib.fcm_kernel_launch_count()
        if args.nvtx:
            torch.cuda.nvtx.range_push("timed")
        e0.record(root)
        for st in set(streams):
            st.wait_event(e0)
        iters = []
        rounds = []
        for j in range(args.steps):
            step = args.warmup + j
            if mode == "batch":
                iters += [inf.gmres_iters for inf in batch.step(seeds, step)]
                rounds.append(batch.last_rounds())
            elif mode == "many":
                iters += [inf.gmres_iters for inf in step_many(ss, seeds, step)]
            else:
                for k, s in enumerate(ss):
                    if mode == "graph":
                        s.step_async(seeds[k], step)
                        _, inf = s.step_wait()
                    else:
                        _, inf = s.step(seeds[k], step)
                    iters.append(inf.gmres_iters)
        for st in set(streams):
            ev = torch.cuda.Event()
            ev.record(st)
            root.wait_event(ev)
        e1.record(root)
        e1.synchronize()
        if args.nvtx:
            torch.cuda.nvtx.range_pop()
        clocks = sampler.stop() if tag == "mixed" else None
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        tunings = {}
        for s in ([] if batch is not None else ss):
            if s.tuning is not None:
                key = str(s.tuning["variants"])
                tunings[key] = tunings.get(key, 0) + 1
        res[tag] = dict(t=t, iters=float(np.mean(iters)) if iters else 0.0,
                        launches=lib.fcm_kernel_launch_count() - l0,
                        clocks=clocks, rounds=[float(np.mean([r[i] for r in rounds])) for i in (0, 1)] if rounds else None,
                        tunings=tunings or None)
        if batch is not None:
            batch.close()
        else:
            for s in ss:
                s.close()
    if not {"fp64", "fp64_graph", "mixed"} <= set(res):
        if rank == 0:
            print(json.dumps({"ensemble_partial": {k: {"ms_per_step": 1e3 * v["t"] / args.steps, "iters": v["iters"],
                                                        "rounds": v["rounds"]} for k, v in res.items()}}))
        if world > 1:
            dist.destroy_process_group()
        return
    # velocity error of the mixed solve against the FP64 solve, every instance of this rank
    errs = [rel_vel_error(p, ref, x, q, fe, root) for p, ref, x, q, fe in insts]
    eU = max_over_ranks(max(e[0] for e in errs) if errs else 0.0)
    eL = max_over_ranks(max(e[1] for e in errs) if errs else 0.0)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    val = {k: total_bodies * args.steps / v["t"] for k, v in res.items()}
    value = val["mixed"]
    grids = sorted({p.nx for p, *_ in all_insts})

    def arm(tag, mode):
        if tag not in res:
            return None
        out = {"value": val[tag], "ms_per_step": 1e3 * res[tag]["t"] / args.steps,
               "gmres_iters": res[tag]["iters"], "mode": mode}
        if res[tag]["rounds"]:
            out["lockstep_rounds"] = {"gmres_iters": res[tag]["rounds"][0], "sweeps": res[tag]["rounds"][1]}
        return out

    ratio = lambda a, b: val[a] / val[b] if a in val and b in val else None
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * res["mixed"]["t"] / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f32 grid + f64 refinement", "data": "synthetic (seeded random rods, Philox noise)",
        "config": {"workload": "ensemble64_rods50-500_g64-128", "instances": len(all_insts), "bodies": total_bodies,
                   "grids": grids, "gmres_tol_fp64": all_insts[0][0].gmres_tol, "mixed_gmres_tol": MIXED_TOL,
                   "seeds": "0..63",
                   "parallelism": "64 contexts on 64 streams, one CUDA graph per instance step (fcm_step_many)"
                                  + ("; instances r, r+%d, ... on rank r" % world if world > 1 else ""),
                   "kernel_variants": {"legend": VARIANT_LEGEND, "members_per_choice": {
                       k: res[k]["tunings"] for k in ("fp64", "mixed") if k in res}}},
        "fp64": arm("fp64", "instances one after another, host-driven fcm_step"),
        "fp64_graph": arm("fp64_graph", "instances one after another, device-resident graph steps"),
        "fp64_many": arm("fp64_many", "64 contexts on 64 streams, fcm_step_many (the mixed arm's concurrency)"),
        "fp64_batch": arm("fp64_batch", "one FP64 fcm_batch: lockstep batched solve, one CUDA graph per step"),
        "mixed_batch": arm("mixed_batch", "one mixed fcm_batch: lockstep batched solve, one CUDA graph per step"),
        "mixed_over_fp64_many": ratio("mixed", "fp64_many"),
        "mixed_batch_over_fp64_batch": ratio("mixed_batch", "fp64_batch"),
        "mixed_batch_over_fp64_graph": ratio("mixed_batch", "fp64_graph"),
        "mixed_over_fp64": ratio("mixed", "fp64"), "mixed_over_fp64_graph": ratio("mixed", "fp64_graph"),
        "gmres_iters_mixed": res["mixed"]["iters"],
        "rel_vel_error_mixed_vs_fp64_max": {"bodies": eU, "blobs": eL},
        "gpu_launches": res["mixed"]["launches"],
        "clocks": res["mixed"]["clocks"],
    }))


def main():
    global MIXED_TOL
    args = parse()
    AUTOTUNE["on"] = not args.no_autotune
    if args.mixed_tol:
        MIXED_TOL = args.mixed_tol
    if args.workload.startswith("ensemble"):
        run_ensemble(args)
        return
    if args.kernels_only:
        run_kernels_only(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
