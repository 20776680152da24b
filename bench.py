#!/usr/bin/env python3
"""Benchmark of the B200 Barnes-Hut step: body-updates/s of the N = 1,048,576 two-component
dwarf (TreeCode, theta 0.5, quadrupoles, Miyamoto-Nagai + Hernquist + logarithmic halo).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The input is the sample workunit's two-component Plummer dwarf (for_developers.lua: baryons
a = 0.2 kpc, M = 12; radius and mass ratios 0.2; half the bodies baryons) sampled on the GPU by
the library's port of the reference's Eddington-inversion sampler (nbGenerateDwarfCUDA, a fixed
seed, the same bodies bit for bit on every run), placed on its orbit point (l = 218, b = 53.5,
r = 28.6 kpc; v = (-156, 79, 107)); dt and eps2 from the reference's formulas.  Both arms step
the same arrays.

One step = one kick-drift-kick step of the whole dwarf: bounding box, octree build,
moments, the force walk with the external potential, both leapfrog halves.  The headline
`value` is the FP64 drop-in form (bit-exact with the reference CPU step), timed on the device
(CUDA events on the library's stream) with the bodies resident in HBM; `e2e` is the same
metric through the C ABI with host (pinned) buffers copied in and out every step.  The
mixed-precision form, the sampled accuracy of both forms against FP64 direct summation, the
roofline of the walk kernel, the CPU-runnable 20,000-body configuration (200 steps), the
8,388,608-body configuration, the adjoint cost and the batched dwarfs are reported alongside;
short top-level keys at the end of the line repeat their headline figures.

Multi-GPU (launched under torchrun): one independent dwarf per GPU, no collective on the
data path ("replicas only": a single Barnes-Hut step does not shard), weak scaling;
`value` = all ranks' body-updates / the slowest rank's device time.

--impl reference: the reference's own CPU code (oracle/_ref, built from its sources; the C
restatement in oracle/ when that is absent) on this host's cores, stepping the same dwarf
through its stock step (nbGravMap once, then nbStepSystem per step) for the W + K steps the
line claims, each timed whole; plus the 200-step run of the 20,000-body configuration.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "body-updates/s N=1M: FP64 vs mixed at stated error; adjoint/forward time"
UNIT = "body-updates/s"
N_DEFAULT = 1048576
THETA_DEFAULT = 0.5
SEED_1M, SEED_CONFIG0, SEED_CONFIG2 = 1000, 2000, 3000
WALK_FORM = -1          # the FP64 walk's form (nbSetWalkFormCUDA): -1 chosen by timing
WORKLOAD = ("sample workunit's two-component Plummer dwarf, N=1,048,576 (half baryons), "
            "TreeCode theta=0.5, quadrupoles, Miyamoto-Nagai+Hernquist+logarithmic-halo "
            "potential, KDK leapfrog")
# algorithmic flops per unit of the walk (add/mul/div/sqrt = 1): node visit test 9,
# body/monopole interaction 18, quadrupole cell 18 + 38 (nbody/src/nbody_grav.c:53-100)
FLOP_VISIT, FLOP_MONO, FLOP_QUAD = 9, 18, 56
# compulsory HBM bytes per body of the phases outside the walk, one step, from the kernels'
# inputs and outputs touched once: drift + bounding box 72 read + 48 written; keys 32 + 12;
# radix sort 8 passes x (12 read + 12 written); grid gather, run fix and parting depths ~60;
# prefix sums 8; node records ~1.5 nodes per body x 64; links 1.5 x 8; moments 1.5 x 80;
# potential + kick 72 read + 48 written
NONWALK_BYTES_PER_BODY = 120 + 44 + 192 + 60 + 8 + 96 + 12 + 120 + 120
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "walk_traffic.json")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--theta", type=float, default=THETA_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config0-steps", type=int, default=200,
                    help="steps of the 20,000-body configuration (0: skip)")
    ap.add_argument("--config2-n", type=int, default=8388608,
                    help="bodies of the large configuration (0: skip)")
    ap.add_argument("--config2-steps", type=int, default=50)
    ap.add_argument("--adjoint-n", type=int, default=131072,
                    help="bodies of the adjoint-cost measurement (0 skips it)")
    ap.add_argument("--adjoint-steps", type=int, default=1000)
    ap.add_argument("--adjoint-warmup-steps", type=int, default=64)
    ap.add_argument("--batch-dwarfs", type=int, default=256,
                    help="dwarfs of the batched workload (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--batch-theta", type=float, default=1.0)
    ap.add_argument("--batch-seed", type=int, default=2024)
    ap.add_argument("--energy-steps", type=int, default=100,
                    help="steps of the energy-drift run of both forms (0: skip)")
    ap.add_argument("--theta2", type=float, default=1.0,
                    help="second opening angle measured for both forms (0: skip)")
    ap.add_argument("--walk-form", choices=["auto", "union", "lanes", "prefetch"],
                    default="auto",
                    help="the FP64 walk: chosen by timing (default), warp union, per lane, or "
                         "per lane loading the next record early")
    ap.add_argument("--profile", choices=["fp64", "mixed", "adjoint", "batch", "config0"],
                    help="profiling entry: build the dwarf, run two force evaluations, exit")
    return ap.parse_args()


def bench_ctx(n, theta, precision="fp64"):
    from milkywayathome_client_b200 import models
    from milkywayathome_client_b200.nbody import NBodyCtx
    cfg = models.dwarf_config(n, theta=theta)
    return NBodyCtx(potential=models.sample_workunit_potential(), precision=precision, **cfg), cfg


def bench_config(n, theta):
    """The `config` of the JSON line: the same dict in both arms."""
    _, cfg = bench_ctx(n, theta)
    return {"workload": WORKLOAD, "n_bodies": n, "theta": theta, "criterion": "TreeCode",
            "quadrupole": True, "eps2": cfg["eps2"], "dt": cfg["timestep"],
            "input": "nbGenerateDwarfCUDA (the reference's two-component sampler on the GPU), "
                     "seed %d, on the orbit point l=218 b=53.5 r=28.6 v=(-156,79,107)" % SEED_1M,
            "parallelism": "replicas: one independent dwarf per GPU",
            "l2": "inputs larger than L2: ~%.1fM tree nodes (~%.0f MB) + bodies (~%.0f MB) per "
                  "step" % (1.5 * n / 1e6, 1.5 * n * 176 / 1e6, n * 120 / 1e6)}


def bench_input(n, seed, device=0):
    """The benchmark dwarf: host arrays pos, vel, mass, type (models.sampled_dwarf)."""
    from milkywayathome_client_b200 import models
    return models.sampled_dwarf(n, seed=seed, device=device)


# ---------------------------------------------------------------------------------------
class Dist:
    """torch.distributed plumbing (barrier, max/sum over ranks); a single process without it.
    NCCL between GPUs; gloo when no GPU is present (the CPU tests of the replica logic)."""

    def __init__(self, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.cuda = False
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            self.cuda = torch.cuda.is_available() if backend is None else backend == "nccl"
            if self.cuda:
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend or ("nccl" if self.cuda else "gloo"),
                                    timeout=datetime.timedelta(seconds=180))
            self.pg = dist
        else:
            try:
                import torch
                self.cuda = torch.cuda.is_available()
            except ImportError:
                self.cuda = False

    def _tensor(self, x):
        import torch
        dev = "cuda:%d" % self.local if self.cuda else "cpu"
        return torch.tensor([float(x)], device=dev, dtype=torch.float64)

    def barrier(self):
        if self.pg:
            if self.cuda:
                self.pg.barrier(device_ids=[self.local])
            else:
                self.pg.barrier()
        if self.cuda:
            import torch
            torch.cuda.synchronize()

    def max(self, x):
        if not self.pg:
            return x
        t = self._tensor(x)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        t = self._tensor(x)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def replica_throughput(dist, n_per_rank, steps, seconds_this_rank):
    """Whole-job body-updates/s of independent replicas: all ranks' updates over the slowest
    rank's time (max over ranks)."""
    t = dist.max(seconds_this_rank)
    return dist.world * n_per_rank * steps / t, t


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = max(smax, float(parts[2]))
                except ValueError:
                    continue
                for name, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def pinned_array(shape):
    import torch
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


def walk_flops(counts, use_quad=True):
    bb, bc, visits = counts[:3]
    return bb * FLOP_MONO + bc * (FLOP_QUAD if use_quad else FLOP_MONO) + visits * FLOP_VISIT


# ---------------------------------------------------------------------------------------
class RefStepper:
    """The reference's stock step on this host's cores: a reference NBodyState built from the
    arrays (oracle/_ref: setInitialNBodyState), nbGravMap once, then nbStepSystem per step
    (nbody/src/nbody.c:182-200 -> nbStepSystemPlain, nbody/src/nbody_plain.c:329-364).  Where
    the reference build is absent, the oracle's C restatement (or_grav_map + or_step)."""

    def __init__(self, ctx, pos, vel, mass, typ):
        from oracle import bindings as ob
        self.ob = ob
        self.ctx = ctx
        self.kind = "reference" if ob.ref_available() else "port"
        self.n = len(mass)
        if self.kind == "reference":
            self.r = ob.RefState.create(ctx.struct, pos, vel, mass, typ)
            self.cores = int(ob.ref().nbref_threads())
            self.status = int(self.r.gravmap())
        else:
            self.cores = int(ob.oracle().or_threads())
            self.status, self.pos, self.vel, self.acc, self.rsize = ob.steps(
                ctx.struct, pos, vel, mass, ctx.treeRSize, 0)
            self.mass = np.ascontiguousarray(mass, dtype=np.float64)

    def step(self, k=1):
        """k steps; returns their wall-clock seconds."""
        import ctypes
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.status |= int(self.r.step(k))
        else:
            rs, inc = ctypes.c_double(self.rsize), ctypes.c_int(0)
            p = lambda a: ctypes.c_void_p(a.ctypes.data)
            self.status |= int(self.ob.oracle().or_step(
                ctypes.byref(self.ctx.struct), p(self.pos), p(self.vel), p(self.mass), self.n,
                ctypes.byref(rs), p(self.acc), k, ctypes.byref(inc)))
            self.rsize = rs.value
        return time.perf_counter() - t0

    def close(self):
        if self.kind == "reference":
            self.r.close()


def config0_reference(args, dev):
    """The 20,000-body configuration's whole run (args.config0_steps steps) on the reference's
    CPU code, timed without sampling; the same input as the GPU leg."""
    n0 = 20000
    pos, vel, mass, typ = bench_input(n0, SEED_CONFIG0, dev)
    ctx0, _ = bench_ctx(n0, 1.0)
    ref = RefStepper(ctx0, pos, vel, mass, typ)
    secs = ref.step(args.config0_steps)
    ref.close()
    return {"value": n0 * args.config0_steps / secs, "unit": UNIT, "seconds": secs,
            "steps": args.config0_steps, "n_bodies": n0, "cores": ref.cores, "kind": ref.kind,
            "status": ref.status}


def cpu_baseline_step(ctx, pos, vel, mass, typ, args, dev):
    """Reference CPU code on this host's cores on the same dwarf: its initial nbGravMap
    (untimed), then one whole nbStepSystem step timed -- no sampling, no extrapolation; plus
    the 20,000-body configuration's whole run.  Returns the cpu_baseline object."""
    ref = RefStepper(ctx, pos, vel, mass, typ)
    step_s = ref.step(1)
    ref.close()
    out = {"value": len(mass) / step_s, "unit": UNIT, "cores": ref.cores, "kind": ref.kind,
           "sample": ("one whole step of the same %d-body dwarf (nbStepSystem after the initial "
                      "nbGravMap, %.2f s on %d threads), not extrapolated"
                      % (len(mass), step_s, ref.cores)) if ref.kind == "reference" else
                     ("one whole step of the oracle's C restatement (or_step) on the same dwarf "
                      "(%.2f s on %d threads)" % (step_s, ref.cores)),
           "status": ref.status, "step_seconds": step_s}
    if args.config0_steps > 0:
        out["config0"] = config0_reference(args, dev)
    return out


def adjoint_ratio(n, steps, warm_steps, dev):
    """Adjoint step / forward step time of the FP64 step with the tree frozen per step, on the
    two-component dwarf at n bodies (checkpoints every 32 steps, recomputation between them).
    Both passes are timed the same way (CUDA events on torch's stream around the whole pass,
    host sequencing included), on a run of `steps` steps after a warm-up run of `warm_steps`."""
    import torch
    from milkywayathome_client_b200 import adjoint
    pos, vel, mass, _ = bench_input(n, 4242, dev)
    ctx, _ = bench_ctx(n, 0.5)
    device = torch.device("cuda:%d" % dev)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=device)
    x0, v0, m = t(pos).requires_grad_(True), t(vel).requires_grad_(True), t(mass).requires_grad_(True)
    dt = t(ctx.timestep).requires_grad_(True)
    w = torch.randn((n, 3), dtype=torch.float64, device=device, generator=torch.Generator(device=device).manual_seed(0))
    # the warm-up run's device state (buffers and saved trees) is kept for the timed run, as in
    # an optimisation loop
    for nsteps in (warm_steps, steps):
        stats = {}
        xN, vN = adjoint.run(ctx, x0, v0, m, dt, nsteps, every=32, stats=stats)
        ((xN * w).sum() + (vN * w).sum()).backward()
    adjoint.release_states()
    return {"n_bodies": n, "steps": steps, "checkpoint_every": 32, "warmup_steps": warm_steps,
            "forward_step_ms": stats["forward_step_ms"], "adjoint_step_ms": stats["adjoint_step_ms"],
            "ratio": stats["adjoint_step_ms"] / stats["forward_step_ms"],
            "parts_device_ms": {k: stats[k] for k in ("forward_step_device_ms",
                                                      "recompute_step_device_ms",
                                                      "reverse_step_device_ms",
                                                      "vjp_walk_device_ms")},
            "how": "tree frozen per step; backward = segment recomputation (saving each step's "
                   "bodies and tree in HBM) + reverse step (nbStepAdjointCUDA: force VJP on the "
                   "saved tree and reverse leapfrog) per step; both passes timed with CUDA "
                   "events around the pass"}


def batched_run(args, dist, dev):
    """The batched-dwarfs workload (mixed form): seeded uneven dwarfs, N log-uniform in
    [4096, 65536], their parameters drawn as the workload states, started on the shared orbit
    t_forward back; plus one dwarf of a seeded reference parameter set whose final histogram is
    the likelihood target.  Dwarfs are dealt to ranks round-robin (independent units, no
    collective on the data path).  Steps run through one captured CUDA graph each, after the
    autotuner picked the walk tuning; the device time of the timed steps is the measure."""
    from milkywayathome_client_b200 import (NBodyBatch, NBodyCtx, HistogramParams,
                                            data_from_counts, models)
    pot = models.sample_workunit_potential()          # the CPU-runnable configuration's
    draws = models.dwarf_parameter_draws(args.batch_dwarfs, seed=args.batch_seed)
    mine = draws[dist.rank::dist.world]
    ref_draw = models.dwarf_parameter_draws(1, seed=args.batch_seed + 1)[0]
    t0 = time.perf_counter()
    # the workload's 500 steps span each dwarf's 3.5-4.5 Gyr forward time: dt = t_forward / 500
    spec, structs = models.batched_dwarf_structs([ref_draw] + mine, pot, seed=args.batch_seed * 1000,
                                                 device=dev, nsteps=args.batch_steps)
    t_setup = time.perf_counter() - t0
    n_total = int(sum(s[0] for s in spec))
    # the config-0 tree settings: TreeCode, theta = 1.0, quadrupoles; mixed precision
    ctx = NBodyCtx(potential=pot, precision="mixed", timestep=spec[0][2], eps2=spec[0][1],
                   theta=args.batch_theta, criterion="TreeCode", useQuad=True)
    hp = HistogramParams(lambdaStart=-150.0, lambdaEnd=150.0, lambdaBins=50, betaStart=-15.0,
                         betaEnd=15.0, betaBins=1)
    with NBodyBatch(spec, device=dev) as bt:
        t0 = time.perf_counter()
        bt.generate(structs)                 # all dwarfs' initial conditions on the GPU
        t_ic = time.perf_counter() - t0
        bt.check("nbBatchGravMap", bt.gravMap(ctx))
        tune = bt.autotune(ctx)
        bt.check("nbBatchRunSteps", bt.run_steps(ctx, 6, graph=True))
        timed = max(args.batch_steps - 6, 1)         # the 6 warm-up steps count towards the run
        dist.barrier()
        w0 = time.perf_counter()
        rc = bt.run_steps(ctx, timed, graph=True)
        wall = time.perf_counter() - w0
        bt.check("nbBatchRunSteps", rc)
        step_ms = bt.step_time_ms()
        status, rsize, _, nodes = bt.dwarf_info()
        counts, totals, mpp, comps = bt.histogram(hp, components=True)
        data = data_from_counts(hp, counts[0], totals[0, 1], mpp[0], comps[0])
        lik = bt.likelihood(hp, data)
        # after the run: the same state stepped with and without the captured graph
        cmp_ms = {}
        for name, g in (("graph", True), ("plain", False), ("graph_again", True)):
            bt.check("nbBatchRunSteps", bt.run_steps(ctx, 4, graph=g))
            cmp_ms[name] = bt.step_time_ms()
    dev_s = step_ms * timed / 1e3
    t = dist.max(dev_s)
    updates = dist.sum(float(n_total - spec[0][0]) * timed)   # the reference dwarf excluded
    lk = lik[1:, 0]
    return {
        "workload": "%d seeded dwarfs, N log-uniform in [4096, 65536] (%d bodies on this rank), "
                    "mixed form, TreeCode theta=%g, quadrupoles, %d steps spanning each dwarf's "
                    "forward time, one captured CUDA graph per step" % (
                        args.batch_dwarfs, n_total, args.batch_theta, args.batch_steps),
        "value": updates / t, "unit": UNIT, "ms_per_step": step_ms,
        "graph_vs_plain_ms_per_step": cmp_ms, "timed_steps": timed, "wall_s": wall,
        "ic_seconds": t_ic, "ic": "nbBatchGenerateDwarfsCUDA: the reference's two-component "
                                  "sampler for all dwarfs on the GPU",
        "setup_seconds": t_setup,
        "dwarfs_per_rank": len(mine), "bodies_per_rank": n_total - spec[0][0],
        "tuning": {"group_max": tune[0], "list_cap": tune[1], "blocks_per_sm": tune[2],
                   "walk_ms": tune[3]},
        "statuses_nonzero": int(np.count_nonzero(status)),
        "likelihood": {"target": "final histogram of a seeded reference parameter set (50 x 1 "
                                 "Lambda bins over [-150, 150] deg, counts and beta "
                                 "dispersions; EMD + cost + beta-dispersion terms)",
                       "min": float(np.nanmin(lk)), "median": float(np.nanmedian(lk)),
                       "finite": int(np.isfinite(lk).sum()),
                       "reference_self": float(lik[0, 0])},
    }


def run_reference(args, dist):
    """--impl reference: the reference's stock step on the host, rank 0 only."""
    if dist.rank != 0:
        return 0
    n, K, W = args.n, args.steps, args.warmup
    # the same arrays as the GPU arm's rank 0 (generated on the GPU, outside the timed steps)
    pos, vel, mass, typ = bench_input(n, SEED_1M)
    ctx, _ = bench_ctx(n, args.theta)
    ref = RefStepper(ctx, pos, vel, mass, typ)
    times = [ref.step(1) for _ in range(W + K)][W:]
    ref.close()
    step_s = float(np.mean(times))
    value = n * K / float(np.sum(times))
    c0 = config0_reference(args, 0) if args.config0_steps > 0 else None
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: the sample workunit's two-component dwarf (seeded; no dataset)",
        "config": bench_config(n, args.theta),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.cores, "kind": ref.kind,
                         "sample": ("none: %d warm-up + %d timed whole steps of the %d-body dwarf "
                                    "(nbGravMap once, then nbStepSystem per step), each timed "
                                    "with the host clock" % (W, K, n))},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "status": ref.status,
        "step_seconds": times,
        "config0": c0,
        "config0_value": c0["value"] if c0 else None,
    }
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
def form_accuracy(pos, vel, mass, c_cfg, dev, seed=4096):
    """Relative acceleration error of the FP64 walk, the mixed walk (exact sets) and the mixed
    group mode against FP64 direct summation, self-gravity only, on a seeded 4,096-body
    sample."""
    from milkywayathome_client_b200.nbody import NBodyCtx, NBodyState
    n = len(mass)
    rng = np.random.default_rng(seed)
    sample = np.sort(rng.choice(n, size=min(4096, n), replace=False)).astype(np.int32)
    c_self = NBodyCtx(potential=None, **c_cfg)
    rel = {}
    with NBodyState.create(c_self, pos, vel, mass, device=dev, gravmap=False) as sa:
        direct = sa.direct_sample(c_cfg["eps2"], sample)
        cm = c_self.with_precision("mixed")
        for name, c, exact in (("fp64", c_self, True), ("mixed", cm, True),
                               ("mixed_group_mode", cm, False)):
            sa.set_mixed_mode(exact)
            sa.check("nbGravMap", sa.gravMap(c))
            a = sa.accels()[sample]
            rel[name] = np.linalg.norm(a - direct, axis=1) / np.linalg.norm(direct, axis=1)
    out = {"sample": "4,096 seeded bodies, self-gravity only, vs FP64 direct summation"}
    for name in ("fp64", "mixed", "mixed_group_mode"):
        out[name] = {p: float(np.percentile(rel[name], q)) for p, q in
                     (("p50", 50), ("p90", 90), ("p99", 99), ("max", 100))}
    for form, tag in (("mixed", "mixed"), ("mixed_group_mode", "group_mode")):
        for p in ("p50", "p99", "max"):
            out["%s_added_error_%s_pct" % (tag, p)] = 100.0 * (
                out[form][p] - out["fp64"][p]) / out["fp64"][p]
    return out


WALK_FORM_NAMES = {0: "warp union", 1: "per lane", 2: "per lane, next record loaded early"}


def settle_walk_form(st, c):
    """Untimed force evaluations at the current positions (each recomputes the same
    accelerations) until the FP64 walk's automatic form choice is made, so that no timed step
    runs a candidate form; a no-op for the mixed form and once a form is set."""
    from milkywayathome_client_b200 import _lib
    if c.precision != _lib.PRECISION_FP64 or c.criterion == _lib.EXACT:
        return                          # only FP64 tree walks choose a form
    for _ in range(8):
        if st.walk_form() >= 0:
            return
        st.check("nbGravMap", st.gravMap(c))


def run_steps_timed(c, pos, vel, mass, dev, warm, steps, exact=True):
    """A fresh state of the arrays, `warm` untimed steps, then `steps` steps each timed with
    CUDA events; returns (step ms list, walk ms list, tree info)."""
    from milkywayathome_client_b200.nbody import NBodyState
    with NBodyState(len(mass), dev) as st:
        st.set_walk_form(WALK_FORM)
        st.set_bodies(pos, vel, mass, c.treeRSize)
        st.check("nbGravMap", st.gravMap(c))
        st.set_mixed_mode(exact)
        for _ in range(warm):
            st.check("nbStepSystem", st.step(c))
        if warm:
            settle_walk_form(st, c)
        ms, walk = [], []
        for _ in range(steps):
            st.check("nbStepSystem", st.step(c))
            ms.append(st.step_time_ms())
            walk.append(st.walk_time_ms()[0])
        return ms, walk, st.tree_info()


def config0_run(args, dist, dev):
    """The CPU-runnable configuration on the GPU: the sample workunit's dwarf at 20,000 bodies,
    TreeCode theta = 1.0 with quadrupoles, its whole run of args.config0_steps steps (the
    reference's dt and eps2), FP64 and mixed, after one warm-up run on another state."""
    n0, S = 20000, args.config0_steps
    pos, vel, mass, _ = bench_input(n0, SEED_CONFIG0 + dist.rank, dev)
    ctx0, _ = bench_ctx(n0, 1.0)
    out = {"workload": "sample workunit's two-component dwarf, N=20,000, TreeCode theta=1.0, "
                       "quadrupoles, %d steps (nbGenerateDwarfCUDA seed %d)" % (S, SEED_CONFIG0),
           "n_bodies": n0, "steps": S}
    for name, c in (("fp64", ctx0), ("mixed", ctx0.with_precision("mixed"))):
        run_steps_timed(c, pos, vel, mass, dev, 0, max(args.warmup, 3))
        ms, _, _ = run_steps_timed(c, pos, vel, mass, dev, 0, S)
        v, t = replica_throughput(dist, n0, S, sum(ms) / 1e3)
        out[name] = {"value": v, "unit": UNIT, "ms_per_step": 1e3 * t / S, "run_ms": 1e3 * t}
    return out


def config2_run(args, dist, dev):
    """The large configuration: the sample workunit's dwarf at args.config2_n bodies, TreeCode
    theta = 0.5 with quadrupoles, args.config2_steps steps of each form after W warm-up steps;
    sampled direct-sum error; HBM throughput of the phases outside the walk (their compulsory
    bytes over their device time)."""
    n2, S, W = args.config2_n, args.config2_steps, args.warmup
    pos, vel, mass, _ = bench_input(n2, SEED_CONFIG2 + dist.rank, dev)
    ctx2, cfg2 = bench_ctx(n2, 0.5)
    out = {"workload": "sample workunit's two-component dwarf, N=%d, TreeCode theta=0.5, "
                       "quadrupoles, %d steps (nbGenerateDwarfCUDA seed %d)" % (n2, S, SEED_CONFIG2),
           "n_bodies": n2, "steps": S}
    for name, c in (("fp64", ctx2), ("mixed", ctx2.with_precision("mixed"))):
        ms, walk, info = run_steps_timed(c, pos, vel, mass, dev, W, S)
        v, t = replica_throughput(dist, n2, S, sum(ms) / 1e3)
        nonwalk = float(np.mean(ms) - np.mean(walk))
        out[name] = {"value": v, "unit": UNIT, "ms_per_step": 1e3 * t / S,
                     "walk_ms": float(np.mean(walk)), "nonwalk_ms": nonwalk,
                     "nonwalk_hbm_gbs": NONWALK_BYTES_PER_BODY * n2 / (nonwalk * 1e-3) / 1e9}
        out["tree"] = {"nodes": info.nNodes, "max_depth": info.maxDepth, "rsize": info.rsize}
    out["mixed_speedup"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["nonwalk_bytes_per_body"] = NONWALK_BYTES_PER_BODY
    out["accuracy"] = form_accuracy(pos, vel, mass, cfg2, dev)
    return out


def run_ours(args, dist):
    from milkywayathome_client_b200.nbody import NBodyState, kernel_launches, peak_fma_tflops
    n, K, W = args.n, args.steps, args.warmup
    dev = dist.local
    pos, vel, mass, typ = bench_input(n, SEED_1M + dist.rank, dev)
    ctx, cfg = bench_ctx(n, args.theta)
    ctx_mixed = ctx.with_precision("mixed")
    notes = []

    def timed_run(c, exact=True):
        st = NBodyState(n, dev)
        st.set_walk_form(WALK_FORM)
        st.set_bodies(pos, vel, mass, c.treeRSize)
        st.check("nbGravMap", st.gravMap(c))
        st.set_mixed_mode(exact)
        for _ in range(W):              # the automatic walk form is chosen here
            st.check("nbStepSystem", st.step(c))
        settle_walk_form(st, c)
        # the interaction counts of the walk in use (a force evaluation at the same positions)
        st.set_counting(True)
        st.check("nbGravMap", st.gravMap(c))
        counts = st.walk_stats()
        st.set_counting(False)
        dist.barrier()
        l0 = kernel_launches()
        clocks = ClockSampler(dev)
        clocks.start()
        step_ms, walk_ms = [], []
        for _ in range(K):
            st.check("nbStepSystem", st.step(c))
            step_ms.append(st.step_time_ms())
            walk_ms.append(st.walk_time_ms()[0])
        clk = clocks.stop()
        launches = kernel_launches() - l0
        dist.barrier()
        info = st.tree_info()
        info.walkForm = st.walk_form()
        return st, counts, step_ms, walk_ms, launches, clk, info

    # ---- FP64 drop-in (headline) ----
    st, counts, step_ms, walk_ms, launches, clk, info = timed_run(ctx)
    value, t_dev = replica_throughput(dist, n, K, sum(step_ms) / 1e3)
    flops_per_walk = walk_flops(counts)
    mean_walk = float(np.mean(walk_ms))

    # ---- accuracy against FP64 direct summation on a seeded 4,096-body sample ----
    accuracy = form_accuracy(pos, vel, mass, cfg, dev)

    # ---- e2e through the C ABI with pinned host buffers ----
    hp = pinned_array((n, 3)); hv = pinned_array((n, 3)); hm = pinned_array((n,))
    hp[:] = pos; hv[:] = vel; hm[:] = mass
    st.set_bodies(hp, hv, hm, ctx.treeRSize)
    st.check("nbGravMap", st.gravMap(ctx))
    for _ in range(min(W, 2)):
        st.set_bodies(hp, hv, hm, ctx.treeRSize)
        st.check("nbStepSystem", st.step(ctx))
        st.bodies(out=(hp, hv))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        st.set_bodies(hp, hv, hm, ctx.treeRSize)       # pinned host -> HBM
        st.check("nbStepSystem", st.step(ctx))
        st.bodies(out=(hp, hv))                        # HBM -> pinned host
    dist.barrier()
    e2e_value, t_e2e = replica_throughput(dist, n, K, time.perf_counter() - t0)
    e2e = {"value": e2e_value, "unit": UNIT,
           "h2d_bytes_per_step": int(n * (3 + 3 + 1) * 8), "d2h_bytes_per_step": int(n * 6 * 8),
           "how": ("per step: nbSetBodiesCUDA (pinned pos/vel/mass -> HBM), nbStepSystemCUDA, "
                   "nbGetBodiesCUDA (HBM -> pinned pos/vel); host wall clock, max over ranks")}
    st.close()

    # ---- mixed form ----
    stm, counts_m, step_ms_m, walk_ms_m, launches_m, clk_m, _ = timed_run(ctx_mixed)
    stm.close()
    mixed_value, t_mixed = replica_throughput(dist, n, K, sum(step_ms_m) / 1e3)
    mixed = {"value": mixed_value, "unit": UNIT,
             "ms_per_step": 1e3 * t_mixed / K, "walk_ms": float(np.mean(walk_ms_m)),
             "speedup_vs_fp64": t_dev / t_mixed,
             "interaction_sets": "exact (nbSetMixedModeCUDA 1, the default): every body takes "
                                 "its own FP64 interaction set"}
    # the group mode (every body of a walk group takes the group's set): faster, heavier tail
    stg, _, step_ms_g, walk_ms_g, _, _, _ = timed_run(ctx_mixed, exact=False)
    stg.close()
    group_value, t_group = replica_throughput(dist, n, K, sum(step_ms_g) / 1e3)
    mixed["group_mode"] = {"value": group_value, "unit": UNIT,
                           "ms_per_step": 1e3 * t_group / K,
                           "walk_ms": float(np.mean(walk_ms_g)),
                           "speedup_vs_fp64": t_dev / t_group}

    # ---- energy drift of both forms over the configuration's step count ----
    energy = None
    if args.energy_steps > 0:
        energy = {"steps": args.energy_steps,
                  "how": "total energy (kinetic + softened self-gravity + external potential) "
                         "by FP64 direct summation on the GPU (nbEnergyCUDA) before and after "
                         "the run; rel_drift = (E1 - E0) / |E0|; the external potential "
                         "dominates E, so the drift is also given over |W0|, the dwarf's "
                         "self-gravity energy"}
        for name, c in (("fp64", ctx), ("mixed", ctx_mixed)):
            with NBodyState.create(c, pos, vel, mass, device=dev) as se:
                e0 = se.energy(c)
                se.check("nbRunSteps", se.run_steps(c, args.energy_steps))
                e1 = se.energy(c)
            energy[name] = {"E0": sum(e0), "E1": sum(e1),
                            "rel_drift": (sum(e1) - sum(e0)) / abs(sum(e0)),
                            "drift_over_self_energy": (sum(e1) - sum(e0)) / abs(e0[1]),
                            "components_E0": list(e0)}

    # ---- the configuration's second opening angle: both forms, speed and accuracy ----
    theta2 = None
    if args.theta2 > 0:
        ctx2, cfg2 = bench_ctx(n, args.theta2)
        theta2 = {"theta": args.theta2}
        for name, c in (("fp64", ctx2), ("mixed", ctx2.with_precision("mixed"))):
            ms, _, _ = run_steps_timed(c, pos, vel, mass, dev, W, K)
            v2, t2 = replica_throughput(dist, n, K, sum(ms) / 1e3)
            theta2[name] = {"value": v2, "unit": UNIT, "ms_per_step": 1e3 * t2 / K}
        theta2["speedup_mixed_vs_fp64"] = theta2["mixed"]["value"] / theta2["fp64"]["value"]
        theta2["accuracy"] = form_accuracy(pos, vel, mass, cfg2, dev)

    # ---- roofline of the walk kernels (FP64 pipe; FP32 pipe for the mixed walk) ----
    peak64 = peak_fma_tflops(True, dev)
    peak32 = peak_fma_tflops(False, dev)
    achieved = flops_per_walk / (mean_walk * 1e-3) / 1e12
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        try:
            with open(PROFILE_TRAFFIC) as f:
                prof = json.load(f)
            rec = prof["fp64_walk_lanes" if info.walkForm >= 1 else "fp64_walk"]
            per_body = rec["dram_bytes"] / rec["n_bodies"]
            traffic = per_body * n
        except (OSError, KeyError, ValueError):
            traffic = None
    roofline = {"bound": "fp64",
                "kernel": "k_walk_fp64_lanes" if info.walkForm >= 1 else "k_walk_fp64",
                "achieved": achieved,
                "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                "traffic": traffic,
                "peak_source": "measured DFMA throughput on this GPU (nbPeakFmaCUDA, in this run)",
                "flops_per_launch": flops_per_walk, "walk_ms": mean_walk,
                "interactions_per_body": {"body": counts[0] / n, "cell": counts[1] / n,
                                          "visits": counts[2] / n},
                "lane_utilisation": counts[2] / (32.0 * max(counts[3], 1)),
                "walk_form": WALK_FORM_NAMES.get(info.walkForm, "undecided")}
    # the exact-set mixed walk evaluates every body's own FP64 interaction set, so its
    # algorithmic work is the FP64 walk's count; issued work (list entries x 32 lanes, masked
    # lanes included) is given beside it
    mixed["roofline"] = {"bound": "fp32", "kernel": "k_walk_mixed",
                         "achieved": flops_per_walk / (mixed["walk_ms"] * 1e-3) / 1e12,
                         "peak": peak32, "unit": "TFLOP/s",
                         "peak_source": "measured FFMA throughput (nbPeakFmaCUDA)",
                         "flops_per_launch": flops_per_walk,
                         "issued_flops_per_launch": walk_flops(counts_m)}
    mixed["roofline"]["frac"] = mixed["roofline"]["achieved"] / peak32

    # ---- the CPU-runnable and the large configurations ----
    config0 = None
    if args.config0_steps > 0:
        try:
            config0 = config0_run(args, dist, dev)
        except Exception as e:
            notes.append("config0 measurement failed: %r" % (e,))
    config2 = None
    if args.config2_n > 0:
        try:
            config2 = config2_run(args, dist, dev)
        except Exception as e:
            notes.append("config2 measurement failed: %r" % (e,))

    # ---- adjoint step cost (the adjoint configuration's dwarf) ----
    adj = None
    if args.adjoint_n > 0:
        try:
            adj = adjoint_ratio(args.adjoint_n, args.adjoint_steps, args.adjoint_warmup_steps, dev)
        except Exception as e:
            notes.append("adjoint measurement failed: %r" % (e,))

    # ---- batched uneven dwarfs (mixed form, graph-captured steps, autotuned walk) ----
    batched = None
    if args.batch_dwarfs > 0:
        try:
            batched = batched_run(args, dist, dev)
        except Exception as e:
            notes.append("batched measurement failed: %r" % (e,))

    # ---- CPU baseline (rank 0, single GPU only) ----
    cpu = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_step(ctx, pos, vel, mass, typ, args, dev)
        except Exception as e:  # the baseline is reported, never the target
            notes.append("cpu_baseline failed: %r" % (e,))

    if dist.rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": K,
            "warmup": W, "ms_per_step": 1e3 * t_dev / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: the sample workunit's two-component dwarf per GPU (seeded; no dataset)",
            "form": "fp64 drop-in (bit-exact with the reference)",
            "config": bench_config(n, args.theta),
            "roofline": roofline, "mixed": mixed, "accuracy": accuracy, "energy": energy,
            "theta2": theta2, "e2e": e2e,
            "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk, "adjoint": adj,
            "batched": batched, "config0": config0, "config2": config2,
            "tree": {"nodes": info.nNodes, "cells": info.cellUsed, "max_depth": info.maxDepth,
                     "rsize": info.rsize},
        }
        if notes:
            out["notes"] = notes
        # the headline figures of every configuration once more, short, at the end of the line
        out["summary"] = {
            "fp64_value": value,
            "mixed_speedup": mixed["speedup_vs_fp64"],
            "mixed_added_error_p99_pct": accuracy["mixed_added_error_p99_pct"],
            "mixed_added_error_max_pct": accuracy["mixed_added_error_max_pct"],
            "theta1_mixed_speedup": theta2["speedup_mixed_vs_fp64"] if theta2 else None,
            "walk_fp64_frac": roofline["frac"],
            "walk_mixed_frac": mixed["roofline"]["frac"],
            "config0_value": config0["fp64"]["value"] if config0 else None,
            "config0_reference_value": (cpu["config0"]["value"]
                                        if cpu and "config0" in cpu else None),
            "config2_fp64_value": config2["fp64"]["value"] if config2 else None,
            "config2_mixed_speedup": config2["mixed_speedup"] if config2 else None,
            "config2_mixed_added_error_p99_pct": (
                config2["accuracy"]["mixed_added_error_p99_pct"] if config2 else None),
            "adjoint_ratio": adj["ratio"] if adj else None,
            "adjoint_steps": adj["steps"] if adj else None,
            "batched_value": batched["value"] if batched else None,
            "cpu_baseline_value": cpu["value"] if cpu else None,
        }
        print(json.dumps(out), flush=True)
    return 0


def run_profile(args):
    """Small committed entry for ncu: the dwarf, one warm-up and one profiled gravMap (or, for
    --profile adjoint, one force evaluation followed by one force VJP at --adjoint-n bodies)."""
    from milkywayathome_client_b200 import models
    if args.profile == "batch":
        from milkywayathome_client_b200 import NBodyBatch, NBodyCtx
        pot = models.sample_workunit_potential()
        draws = models.dwarf_parameter_draws(args.batch_dwarfs, seed=args.batch_seed)
        spec, structs = models.batched_dwarf_structs(draws, pot, seed=args.batch_seed * 1000,
                                                     nsteps=args.batch_steps)
        ctx = NBodyCtx(potential=pot, precision="mixed", timestep=spec[0][2], eps2=spec[0][1],
                       theta=args.batch_theta)
        with NBodyBatch(spec) as bt:
            bt.generate(structs)
            bt.check("nbBatchGravMap", bt.gravMap(ctx))
            bt.check("nbBatchRunSteps", bt.run_steps(ctx, 2, graph=False))
            print(json.dumps({"profile": "batch", "dwarfs": len(spec), "bodies": bt.nbody,
                              "step_ms": bt.step_time_ms()}))
        return 0
    if args.profile == "config0":
        # the 20,000-body configuration: a few whole steps (launch lists of the small case)
        from milkywayathome_client_b200.nbody import NBodyState
        pos, vel, mass, _ = bench_input(20000, SEED_CONFIG0)
        ctx, _ = bench_ctx(20000, 1.0)
        with NBodyState(20000, 0) as st:
            st.set_walk_form(WALK_FORM)
            st.set_bodies(pos, vel, mass, ctx.treeRSize)
            st.check("nbGravMap", st.gravMap(ctx))
            ms = []
            for _ in range(5):
                st.check("nbStepSystem", st.step(ctx))
                ms.append(st.step_time_ms())
            print(json.dumps({"profile": "config0", "n": 20000, "step_ms": ms}))
        return 0
    if args.profile == "adjoint":
        import torch
        from milkywayathome_client_b200.adjoint import DeviceState
        n = args.adjoint_n
        pos, vel, mass, _ = bench_input(n, 4242)
        ctx, _ = bench_ctx(n, args.theta)
        dev = torch.device("cuda:0")
        t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
        ds = DeviceState(n, dev)
        ds.set(t(pos), t(vel), t(mass), ctx.treeRSize)
        ds.gravmap(ctx)
        fwd_walk = ds.st.walk_time_ms()[0]
        abar = torch.randn((n, 3), dtype=torch.float64, device=dev,
                           generator=torch.Generator(device=dev).manual_seed(0))
        ds.vjp(ctx, abar)
        print(json.dumps({"profile": "adjoint", "n": n, "forward_walk_ms": fwd_walk,
                          "vjp_walk_ms": ds.st.walk_time_ms()[0], "vjp_ms": ds.st.step_time_ms()}))
        ds.close()
        return 0
    from milkywayathome_client_b200.nbody import NBodyState
    pos, vel, mass, _ = bench_input(args.n, SEED_1M)
    ctx, _ = bench_ctx(args.n, args.theta, precision=args.profile)
    with NBodyState(args.n, 0) as st:
        st.set_walk_form(WALK_FORM if WALK_FORM >= 0 else 0)
        st.set_bodies(pos, vel, mass, ctx.treeRSize)
        st.check("nbGravMap", st.gravMap(ctx))
        st.check("nbGravMap", st.gravMap(ctx))
        print(json.dumps({"profile": args.profile, "n": args.n, "walk_ms": st.walk_time_ms()[0],
                          "step_ms": st.step_time_ms()}))
    return 0


def main():
    args = parse_args()
    global WALK_FORM
    WALK_FORM = {"auto": -1, "union": 0, "lanes": 1, "prefetch": 2}[args.walk_form]
    if args.impl == "reference":
        # the reference arm is host-only: rank 0 runs it, other ranks exit without work
        os.environ.setdefault("WORLD_SIZE", "1")
        dist = Dist.__new__(Dist)
        dist.world, dist.rank = 1, int(os.environ.get("RANK", "0"))
        dist.local, dist.pg = int(os.environ.get("LOCAL_RANK", "0")), None
        return run_reference(args, dist)
    if args.profile:
        return run_profile(args)
    dist = Dist()
    try:
        return run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    sys.exit(main())
