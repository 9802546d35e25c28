#!/usr/bin/env python
"""Benchmark: exact poses/s of the batched scorer on synthetic complexes.

Workload (default): the batched exact-scorer configuration — 64 synthetic
complexes (receptors log-uniform 2k-40k atoms, ligands 300-5k atoms; 32 dna,
32 pydock), 20 swarms x 300 glowworms each = 384,000 poses per step, seed 11.
One step = one scoring pass over every pose of every complex, issued as ONE
launch group (``lkg_score_multi_device``).  ``--workload config0`` runs the
plain dna configuration (1 x 200 poses) instead.

Reported (one JSON line on rank 0):
  value     poses/s with poses resident in HBM, CUDA events on the context's
            stream, max over ranks (weak scaling: every rank scores its own
            copy of the workload; with ``--partition`` the complexes are
            split over the ranks instead, strong scaling, and the scores are
            gathered after the timed region)
  e2e       the same through the C ABI with host buffers (``lkg_score_multi``:
            page-locked poses in, scores out, every step)
  roofline  FP32 work of the dominant kernel (near pairs x FLOPs per pair
            from the reference formulas + 30 FLOPs per charged ligand atom
            for the far field) per launch / launch time, against the FP32
            peak 148 SMs x 128 lanes x 2 FLOPs x max SM clock
  cpu_baseline  the oracle (C++ restatement of the reference's CPU grid
            path, OpenMP over poses, all host cores) on a bounded sample
``--impl reference`` times that CPU path alone as the reference arm.
"""
import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

FLOPS_PER_PAIR = {"dna": 24, "pydock": 23, "vdw": 19, "cpydock": 25}
# DRAM bytes per pose of the fast kernel (56.8 MB per 24,000-pose launch of
# the 4-complex profiling case under ncu, at tile 256, groups of 16, cell 7 A)
TRAFFIC_PER_POSE = 56.8e6 / 24000
FAR_FLOPS = 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lkg", choices=["lkg", "reference"])
    ap.add_argument("--workload", default="config2",
                    choices=["config2", "config0", "config1", "config3", "config4", "config4-gso",
                             "restraints"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--gso-loop-steps", type=int, default=100,
                    help="GSO steps of the step-loop measurement (batched workload; 0: skip it)")
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--cell", type=float, default=0.0)
    ap.add_argument("--group", type=int, default=0)
    ap.add_argument("--xsub", type=int, default=0)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--stage", default="l1", choices=["l1", "tma"],
                    help="how the plain kernel loads candidate receptor atoms: through L1 (default) or staged in "
                         "shared memory by bulk copies")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--gso-steps", type=int, default=200)
    ap.add_argument("--seeds", type=int, default=1,
                    help="screened workloads: GSO seeds over which the screened run, the random-rank ablation and "
                         "the plain run with the next seed are compared with the plain run (mean and spread)")
    ap.add_argument("--complexes", type=int, default=0,
                    help="score only the first K complexes of the workload (profiling-size cases)")
    ap.add_argument("--partition", action="store_true",
                    help="under torchrun: split the workload's complexes over the ranks (strong scaling, scores "
                         "gathered after the timed region) instead of one replica of the workload per rank")
    return ap.parse_args()


def workload(name, gen=None):
    """The workload's complexes with their setup poses.  gen: the chain and
    StdRng generators (None: liblkg's; the CPU reference arm passes the
    oracle's, so that it never loads the product library)."""
    synth = importlib.import_module("lklight-gpu_b200.synth")
    if gen is not None and name not in ("config0", "config2"):
        raise SystemExit("the CPU reference arm covers the config0 and config2 workloads")
    if name == "config0":
        c0 = synth.config0(gen=gen)
        items = [dict(rec=c0["rec"], lig=c0["lig"], family="dna", swarms=1, glowworms=200, seed=42)]
    elif name == "config1":
        base = synth.config0()
        items = []
        for fam in ("vdw", "pydock", "cpydock"):
            c1 = synth.config1(fam, base=base)
            items.append(dict(rec=c1["rec"], lig=c1["lig"], family=fam, swarms=6, glowworms=300, seed=7))
    elif name == "config4":
        c4 = synth.config4()
        items = [dict(rec=c4["rec"], lig=c4["lig"], family="cpydock", swarms=50, glowworms=500, seed=19)]
    elif name == "restraints":
        # the config-0 complex (dna) at the config-3 swarm layout, with active
        # restraints and a membrane: runs the reference scores on its CPU path only
        c0 = synth.config0()
        items = [dict(rec=c0["rec"], lig=c0["lig"], family="dna", swarms=10, glowworms=1000, seed=3)]
    else:
        items = synth.config2(gen=gen)
    for it in items:
        it["poses"] = synth.to_kernel_poses(
            synth.setup_poses(it["rec"]["coords"], it["swarms"], it["glowworms"], it["seed"], gen=gen))
    if name == "restraints":
        it = items[0]
        centres = it["poses"][::it["glowworms"], 4:7]
        it["restraints"] = synth.restraints(it["rec"]["coords"], len(it["lig"]["coords"]), centres, 23)
    return items


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(k)
            except (ValueError, IndexError):
                pass
        load = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_models(items):
    """Oracle models of every complex with their far fields built (set-up,
    as the reference builds its ReceptorField once per receptor)."""
    import oracle
    models = []
    for it in items:
        m = oracle.Model(it["family"], it["rec"], it["lig"])
        m.field()
        if "restraints" in it:
            rr, lr, mem = it["restraints"]
            m.set_restraints(rr, int(rr.max()) + 1, lr, int(lr.max()) + 1, mem)
        models.append(m)
    return models


def cpu_sample(items, models, min_seconds=10.0, threads=0, per_complex=32):
    """The oracle (the reference's CPU grid path) on a bounded sample of the
    workload itself: rounds that take `per_complex` poses from every complex
    in turn (every complex has the same number of poses in the step, so each
    round has the step's mix), until min_seconds pass.  Returns poses/s,
    near pairs/s (pairs counted by the oracle), the cores used and the
    sample's description."""
    done, pairs, off = 0, 0.0, 0
    t0 = time.perf_counter()
    while True:
        for it, m in zip(items, models):
            p = it["poses"]
            sel = p[(off + np.arange(per_complex)) % len(p)]
            _, parts = m.batch_energy_grid(sel, threads=threads, parts=True)
            pairs += float(parts[:, 4].sum())
            done += len(sel)
        off += per_complex
        el = time.perf_counter() - t0
        if el >= min_seconds:
            break
    cores = threads if threads > 0 else os.cpu_count()
    sample = "%d poses, %d from each of the %d complexes in turn (the step's mix), %.1f s" % (
        done, done // len(items), len(items), el)
    return dict(value=done / el, pairs_per_s=pairs / el, cores=cores, sample=sample)


def parity_sample(items, models, scores, counts, pairs, per_complex=4, fp64_every=4, seed=23):
    """Parity of the timed step's own scores, computed after the timed
    region: from every complex, `per_complex` seeded random poses and the
    pose with the most near pairs (the most crowded interface), against the
    oracle (the reference's CPU grid path: f32 far field) and, for every
    `fp64_every`-th complex, against the oracle's FP64 evaluation of the
    same function (far field accumulated and stored in f64).  Relative error
    with denominator max(|E|, 1), as the reference's grid-vs-exact test
    (src/dna.rs:1155-1179)."""
    rng = np.random.default_rng(seed)
    off = np.concatenate([[0], np.cumsum(counts)])
    e_grid, e_fp64, n_fp64 = [], [], 0
    for k, (it, m) in enumerate(zip(items, models)):
        n = counts[k]
        sel = np.unique(np.concatenate([rng.choice(n, min(per_complex, n), replace=False),
                                        [int(np.argmax(pairs[off[k]:off[k + 1]]))]]))
        got = scores[off[k] + sel]
        ref = m.batch_energy_grid(it["poses"][sel])
        e_grid.append(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0))
        if k % fp64_every == 0:
            r64 = m.batch_energy_grid(it["poses"][sel], fp64=True)
            e_fp64.append(np.abs(got - r64) / np.maximum(np.abs(r64), 1.0))
            n_fp64 += len(sel)
    eg, ef = np.concatenate(e_grid), np.concatenate(e_fp64)
    return {"vs_oracle": {"max_rel": float(eg.max()), "median_rel": float(np.median(eg)), "poses": int(len(eg))},
            "vs_fp64": {"max_rel": float(ef.max()), "median_rel": float(np.median(ef)), "poses": int(n_fp64)},
            "tolerance": 1e-5, "denominator": "max(|E|, 1)",
            "sample": "from every complex %d seeded random poses of the timed step plus its most crowded pose; "
                      "FP64 on every %d-th complex" % (per_complex, fp64_every)}


def workload_config(args, items, world):
    """The workload definition (identical on both arms of the comparison);
    items: the whole job's complexes."""
    return {"workload": args.workload, "complexes": len(items),
            "poses_per_step": int(sum(len(it["poses"]) for it in items)),
            "families": sorted(set(it["family"] for it in items)),
            "receptor_atoms": int(sum(len(it["rec"]["coords"]) for it in items)),
            "ligand_atoms": int(sum(len(it["lig"]["coords"]) for it in items)),
            "l2": "inputs larger than L2 (receptor arrays and far-field grids of all complexes)",
            "parallelism": "single" if world == 1 else
            ("partitioned by complex" if getattr(args, "partition", False) else "replicas")}


def max_over_ranks(v, dist, device):
    """The slowest rank's value: every multi-rank time is the max over ranks."""
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_items(items, world):
    """Complexes to ranks for a partitioned run: greedy, largest estimated
    work first (poses x ligand atoms, the near scan's cost driver), each to
    the rank with the least work so far.  Returns one list of item indices
    per rank, each in workload order."""
    order = sorted(range(len(items)), key=lambda i: -len(items[i]["poses"]) * len(items[i]["lig"]["coords"]))
    load, out = [0.0] * world, [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += len(items[i]["poses"]) * len(items[i]["lig"]["coords"])
    return [sorted(o) for o in out]


def gather_scores(local, dist):
    """Per-complex score arrays of every rank, merged on every rank
    ({item index: scores}); a single process returns its own."""
    if not dist:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    merged = {}
    for p in parts:
        merged.update(p)
    return merged


def sum_over_ranks(v, dist, device):
    """The sum of a per-rank count over all ranks."""
    if not dist:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank, world, ms_max):
    """Whole-job throughput: every rank processes units_per_rank (replicas,
    weak scaling), the job takes the slowest rank's time."""
    return units_per_rank * world / (ms_max / 1e3)


def run_reference(args, rank, world):
    """The reference's CPU grid path (the oracle port: the reference is Rust
    and cannot be built here) on the host cores, all threads, over bounded
    samples of the same workload: every step takes poses from every complex.
    Inputs come from the oracle's generators, so this arm never loads
    liblkg.  Rank 0 alone runs (the other ranks exit)."""
    if rank != 0:
        return
    import oracle
    items = workload(args.workload, gen=oracle.Generators)
    if args.complexes:
        items = items[:args.complexes]
    models = cpu_models(items)
    vals, prs = [], []
    for s in range(args.warmup + args.steps):
        r = cpu_sample(items, models, min_seconds=1.0 if s < args.warmup else 3.0)
        if s >= args.warmup:
            vals.append(r["value"])
            prs.append(r["pairs_per_s"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "exact poses/s on 1 B200 (dna); surrogate-screened at >=95% top-5 overlap",
            "value": v, "unit": "poses/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(args, items, world),
            "pair_rate": {"value": statistics.median(prs), "unit": "near pairs/s"},
            "cpu_baseline": {"value": v, "unit": "poses/s", "cores": r["cores"], "kind": "port",
                             "sample": r["sample"] + " per step (median of %d steps)" % args.steps},
            "e2e": {"value": v, "unit": "poses/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    ref_gpu = reference_cuda_per_swarm(items, models)
    if ref_gpu:
        line["reference_cuda_kernel"] = ref_gpu
    print(json.dumps(line), flush=True)


# cuda_batch_score (full_score.cu:359-371) as the reference's Rust bridge binds it
_REF_SIG = ("PiiiffffPPPPPiPPiiiffffPPPPPPiiIP")


def reference_cuda_per_swarm(items, models):
    """The reference's own GPU scorer, src/cuda/full_score.cu compiled
    unmodified for sm_100a (oracle/_ref, built where the reference tree is
    present), called the way the reference's GSO calls it: one
    cuda_batch_score per swarm and step (swarm.rs:70-100, gpu_family.rs:
    196-262), host buffers, on every swarm of the workload, each complex's
    first call (the upload into its buffer cache) untimed.  The far field
    is the oracle's grid (bitwise the reference builder's), in place.
    None when there is no CUDA device or the library was not built."""
    import ctypes as C
    path = os.path.join(REPO, "oracle", "_ref", "libref_cuda.so")
    try:
        import torch
        if not torch.cuda.is_available() or not os.path.exists(path):
            return None
    except ImportError:
        return None
    compat = importlib.import_module("lklight-gpu_b200.compat")
    L = C.CDLL(path)
    T = {"P": C.c_void_p, "i": C.c_int, "f": C.c_float, "I": C.c_uint}
    L.cuda_batch_score.argtypes = [T[ch] for ch in _REF_SIG]
    L.cuda_batch_score.restype = C.c_int
    flags = {"dna": 7, "pydock": 3}   # full_score.cu:21-22, gpu_family.rs:187-194
    keep, t_total, poses_done, calls = [], 0.0, 0, 0
    for it, m in zip(items, models):
        if it["family"] not in flags:
            return None
        rec, lig = it["rec"], it["lig"]
        crec = compat.CudaReceptor(rec["coords"], rec["ele"], np.sqrt(rec["vdw"]), rec["radius"], rec["heavy"])
        clig = compat.CudaLigand(lig["coords"], lig["ele"], np.sqrt(lig["vdw"]), lig["radius"], lig["heavy"])
        f = m.field()
        field = dict(phi=f.phi_view(), dims=f.dims, origin=f.origin, spacing=f.spacing)
        # the reference caches device copies by host pointer: every complex's
        # arrays stay alive (and so at distinct addresses) until the end
        keep.append((crec, clig, f, field))
        g = it["glowworms"]
        pos = it["poses"]
        compat.batch_raw(field, crec, clig, pos[:g], flags[it["family"]], library=L)
        t0 = time.perf_counter()
        for s in range(it["swarms"]):
            compat.batch_raw(field, crec, clig, pos[s * g:(s + 1) * g], flags[it["family"]], library=L)
        t_total += time.perf_counter() - t0
        poses_done += it["swarms"] * g
        calls += it["swarms"]
    return {"value": poses_done / t_total, "unit": "poses/s", "calls": calls, "poses_per_call": items[0]["glowworms"],
            "seconds": t_total,
            "what": "the reference's src/cuda/full_score.cu compiled unmodified for sm_100a, one cuda_batch_score per "
                    "swarm (as its GSO calls it), host buffers, every swarm of the workload once, buffer cache warm"}


def pick_shape(args, items, local):
    """The warp kernel's tile shape: the command line's, else the
    autotuner's (CUDA-graph replays of a sample of the workload's complexes
    and poses per candidate shape; cached per device and batch signature)."""
    shape = dict(tile=args.tile, group=args.group, cell=args.cell, xsub=args.xsub, source="command line")
    if not (args.tile or args.group or args.cell or args.xsub):
        if args.no_autotune:
            shape["source"] = "library default"
        else:
            autotune = importlib.import_module("lklight-gpu_b200.autotune")
            shape = autotune.autotune(items, device=local)
    return shape


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lkg = importlib.import_module("lklight-gpu_b200")

    if args.workload in ("config3", "config4-gso"):
        return run_screened(args, lkg, torch, local, rank, world, dist)
    items = workload(args.workload)
    if args.complexes:
        items = items[:args.complexes]
    job_items, mine = items, list(range(len(items)))
    partitioned = args.partition and world > 1
    if partitioned:
        if world > len(items):
            raise SystemExit("--partition needs at least one complex per rank (%d complexes, %d ranks)"
                             % (len(items), world))
        mine = shard_items(items, world)[rank]
        items = [items[i] for i in mine]
    shape = pick_shape(args, items, local)
    ctx = lkg.Context(device=local, tile=shape["tile"], cell=shape["cell"], group=shape["group"], xsub=shape["xsub"],
                      stage=args.stage)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ids = [ctx.add_complex(it["family"], it["rec"], it["lig"]) for it in items]
    for cid, it in zip(ids, items):
        if "restraints" in it:
            ctx.set_restraints(cid, *it["restraints"])
    counts = [len(it["poses"]) for it in items]
    npose = int(sum(counts))
    allp = np.vstack([it["poses"] for it in items])
    d_poses = torch.tensor(allp, dtype=torch.float64, device="cuda")
    d_scores = torch.zeros(npose, dtype=torch.float64, device="cuda")
    d_parts = torch.zeros((npose, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    # algorithmic work: near pairs counted by the exact path (equal to the
    # oracle's count), charged ligand atoms for the far field
    ctx.set_precision("exact")
    ctx.score_multi_device(ids, counts, d_poses.data_ptr(), d_scores.data_ptr(), d_parts.data_ptr())
    stream.synchronize()
    pairs = d_parts[:, 3].cpu().numpy()
    ctx.set_precision("fast")
    flops, off = 0.0, 0
    fam_pairs = {}
    for it, n in zip(items, counts):
        p = float(pairs[off:off + n].sum())
        fam_pairs[it["family"]] = fam_pairs.get(it["family"], 0.0) + p
        charged = int(np.count_nonzero(it["lig"]["ele"])) if it["family"] != "vdw" else 0
        flops += p * FLOPS_PER_PAIR[it["family"]] + FAR_FLOPS * charged * n
        off += n

    # one persistent launch group per step, captured once in a CUDA graph
    plan = lkg.Plan(ctx, ids, counts)
    if args.no_graph:
        def step():
            plan.launch(d_poses.data_ptr(), d_scores.data_ptr())
    else:
        plan.capture(d_poses.data_ptr(), d_scores.data_ptr(), n_launches=1)

        def step():
            plan.replay()

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    l0 = ctx.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launches - l0
    ms = ev0.elapsed_time(ev1) / args.steps
    timed_scores = d_scores.cpu().numpy()   # the last timed step's scores (read after the timed region)
    ms_max = max_over_ranks(ms, dist, "cuda")
    # replicas: every rank scores npose; partitioned: the ranks' shares sum
    # to the workload's poses
    npose_job = sum_over_ranks(npose, dist, "cuda") if partitioned else npose * world

    def rate(ms_):
        return npose_job / (ms_ / 1e3)
    value = rate(ms_max)
    gathered = None
    if partitioned:
        # the one collective of a partitioned run: every complex's scores of
        # the last timed step, gathered on every rank for ranking
        offs = np.concatenate([[0], np.cumsum(counts)])
        merged = gather_scores({mine[k]: timed_scores[offs[k]:offs[k + 1]] for k in range(len(items))}, dist)
        gathered = {"complexes": len(merged), "poses": int(sum(len(v) for v in merged.values())),
                    "complexes_on_rank0": len(mine), "how": "all_gather_object after the timed region"}

    # e2e: host buffers through the C ABI, copies inside the timed region
    h_poses = torch.from_numpy(allp).pin_memory()
    h_scores = torch.zeros(npose, dtype=torch.float64).pin_memory()
    for _ in range(max(1, args.warmup)):
        ctx.score_multi(ids, counts, h_poses, h_scores)
    if dist:
        dist.barrier()
    # device-timed on the context stream: the events bracket every call's
    # H2D of poses, the launch group and the D2H of scores (and any host
    # gap between calls)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for _ in range(args.steps):
        ctx.score_multi(ids, counts, h_poses, h_scores)
    ev3.record(stream)
    ev3.synchronize()
    e2e_ms_max = max_over_ranks(ev2.elapsed_time(ev3) / args.steps, dist, "cuda")
    e2e_value = rate(e2e_ms_max)

    # plain single-complex scorer: one host-buffer call (one launch) per complex
    plain = None
    if not args.no_plain and len(items) > 1:
        for k, cid in enumerate(ids):
            ctx.score(cid, items[k]["poses"])
        t0 = time.perf_counter()
        reps = max(1, min(3, args.steps))
        for _ in range(reps):
            for k, cid in enumerate(ids):
                ctx.score(cid, items[k]["poses"])
        pms = (time.perf_counter() - t0) * 1e3 / reps
        plain = {"value": npose / (pms / 1e3), "unit": "poses/s", "ms_per_step": pms,
                 "what": "lkg_score per complex, host buffers, one launch and sync per complex"}
        # the same kernel launched once per complex on device buffers (no
        # persistent batch, no graph, one wait per step), device-timed
        offs = np.concatenate([[0], np.cumsum(counts)])
        def per_complex():
            for k, cid in enumerate(ids):
                ctx.score_device(cid, counts[k], d_poses.data_ptr() + 56 * int(offs[k]),
                                 d_scores.data_ptr() + 8 * int(offs[k]))
        per_complex()
        stream.synchronize()
        e6, e7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e6.record(stream)
        for _ in range(reps):
            per_complex()
        e7.record(stream)
        e7.synchronize()
        dms = e6.elapsed_time(e7) / reps
        plain["device_buffers"] = {"value": npose / (dms / 1e3), "unit": "poses/s", "ms_per_step": dms,
                                   "what": "lkg_score_device per complex (one launch each), device buffers"}

    # the whole GSO step loop of the batched workload: every swarm of every
    # complex as one device-resident GSO (one persistent scoring launch of
    # the moved glowworms per step plus the GSO kernels, graph-replayed);
    # exact poses / s over the loop, wall time including set-up and the
    # state's read-back
    gso_loop = None
    if args.workload == "config2" and args.gso_loop_steps > 0:
        groups = [(cid, it["swarms"], it["glowworms"]) for cid, it in zip(ids, items)]
        host_pos = np.hstack([allp[:, 4:7], allp[:, 0:4]])   # (tx, ty, tz, qw, qx, qy, qz)
        g = lkg.GSO(ctx, groups, host_pos, [it["seed"] for it in items])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.run(args.gso_loop_steps, device=True)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        t_gso = max_over_ranks(el, dist, "cuda")
        scored_job = sum_over_ranks(g.scored, dist, "cuda") if partitioned else g.scored * world
        gso_loop = {"value": scored_job / t_gso, "unit": "exact poses/s",
                    "steps": args.gso_loop_steps, "seconds": t_gso, "exact_evals_per_rank": int(g.scored),
                    "glowworms": int(len(host_pos)),
                    "what": "device-resident GSO over every swarm of every complex: per step one persistent "
                            "scoring launch of the moved glowworms plus the GSO kernels, replayed from one CUDA "
                            "graph; wall time including set-up and read-back"}
        del g

    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = flops / (ms / 1e3) / 1e12

    line = {"metric": "exact poses/s on 1 B200 (dna); surrogate-screened at >=95% top-5 overlap",
            "value": value, "unit": "poses/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "strong" if partitioned else "weak",
            "vs_baseline": None, "dtype": "f32 pair math, f64 transform and sums", "data": "synthetic",
            "config": workload_config(args, job_items, world),
            "work": {"near_pairs_per_step": float(pairs.sum()), "near_pairs_by_family": fam_pairs,
                     "counted_by": "the exact (f64) path's near-pair counts, equal to the oracle's by test",
                     "tile_shape": {k: shape.get(k) for k in ("tile", "group", "cell", "xsub", "source")}},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak,
                         "traffic": TRAFFIC_PER_POSE * npose if args.workload == "config2" else None,
                         "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of "
                                           "k_score_warp<16> (tile 256, cell 7 A) on the first 4 complexes "
                                           "(24,000 poses), scaled by poses to this launch",
                         "peak_source": "148 SMs x 128 FP32 lanes x 2 x sm_max_mhz of MEASURED_PEAKS.json",
                         "work": "near pairs x FLOPs/pair (dna 24, pydock 23, vdw 19) + 30 per charged ligand "
                                 "atom (far field), counted per launch"},
            "pair_rate": {"value": float(pairs.sum()) / (ms / 1e3), "unit": "near pairs/s"},
            "e2e": {"value": e2e_value, "unit": "poses/s", "ms_per_step": e2e_ms_max,
                    "h2d_bytes_per_step": npose * 7 * 8, "d2h_bytes_per_step": npose * 8,
                    "api": "lkg_score_multi (host page-locked buffers)"},
            "gpu_launches": int(launches), "clocks": clk,
            "step": "CUDA graph replay of one persistent launch group" if not args.no_graph else "plan launch",
            "candidate_loads": args.stage}
    if gathered:
        line["gathered"] = gathered
    if plain:
        line["plain_single_complex"] = plain
    if gso_loop:
        line["gso_step_loop"] = gso_loop
    if any("restraints" in it for it in items):
        # the same poses without restraints / membrane: the cost of the
        # interface bits; and the fractions seen, to show they were exercised
        h_iface = ctx.score_interface(ids[0], items[0]["poses"])[1]
        rr, lr, mem = items[0]["restraints"]
        line["work"]["restraints"] = {
            "receptor_residues": int(rr.max()) + 1, "ligand_residues": int(lr.max()) + 1, "membrane_beads": len(mem),
            "poses_with": {k: int((h_iface[:, i] > 0).sum()) for i, k in enumerate(("rec", "lig", "membrane"))}}
        plan.close()
        for cid in ids:
            ctx.set_restraints(cid)
        plan = lkg.Plan(ctx, ids, counts)
        plan.capture(d_poses.data_ptr(), d_scores.data_ptr(), n_launches=1)
        for _ in range(args.warmup):
            plan.replay()
        e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        for _ in range(args.steps):
            plan.replay()
        e5.record(stream)
        e5.synchronize()
        pms = e4.elapsed_time(e5) / args.steps
        line["without_restraints"] = {"value": npose / (pms / 1e3), "unit": "poses/s", "ms_per_step": pms,
                                      "restraint_overhead": ms / pms - 1.0}
        for cid, it in zip(ids, items):
            ctx.set_restraints(cid, *it["restraints"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        models = cpu_models(items)
        line["parity"] = parity_sample(items, models, timed_scores, counts, pairs)
        r = cpu_sample(items, models)
        line["cpu_baseline"] = {"value": r["value"], "unit": "poses/s", "cores": r["cores"], "kind": "port",
                                "sample": r["sample"], "pair_rate": {"value": r["pairs_per_s"],
                                                                     "unit": "near pairs/s"}}
        r1 = cpu_sample(items, models, min_seconds=5.0, threads=1, per_complex=4)
        line["cpu_baseline_single_thread"] = {"value": r1["value"], "unit": "poses/s", "cores": 1, "kind": "port",
                                              "sample": r1["sample"],
                                              "pair_rate": {"value": r1["pairs_per_s"], "unit": "near pairs/s"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()


def top5_overlap(tr_a, sc_a, tr_b, sc_b, tol=2.0):
    """Share of run A's top-5 poses (engine rank order: descending scoring)
    within tol A on every axis of some top-5 pose of run B
    (tools/analyze_perf3.py:50-55)."""
    ta = tr_a[np.argsort(-sc_a, kind="stable")[:5]]
    tb = tr_b[np.argsort(-sc_b, kind="stable")[:5]]
    return sum(1 for a in ta if any(np.all(np.abs(a - b) <= tol) for b in tb)) / 5.0


def run_screened(args, lkg, torch, local, rank, world, dist):
    """Surrogate-screened GSO against the plain GSO on the same complex and
    start, both ending with an exact rescoring of the final poses; wall time
    of the whole run (device scoring, surrogate training / inference, host
    movement).  config3: the config-0 complex (dna), 10 swarms x 1,000
    glowworms, seed 3.  config4-gso: the config-4 complex (cpydock, 101k-atom
    receptor, 12k-atom ligand), 50 x 500, seed 19, 100 steps."""
    synth = importlib.import_module("lklight-gpu_b200.synth")
    if args.workload == "config4-gso":
        c = synth.config4()
        family, swarms, glow, steps, seed = "cpydock", 50, 500, min(args.gso_steps, 100), 19
    else:
        c = synth.config0()
        family, swarms, glow, steps, seed = "dna", 10, 1000, args.gso_steps, 3
    pos = synth.setup_poses(c["rec"]["coords"], swarms, glow, seed)
    shape = pick_shape(args, [dict(family=family, rec=c["rec"], lig=c["lig"], poses=synth.to_kernel_poses(pos))],
                       local)
    ctx = lkg.Context(device=local, tile=shape["tile"], cell=shape["cell"], group=shape["group"], xsub=shape["xsub"])
    cid = ctx.add_complex(family, c["rec"], c["lig"])
    res = {}
    clocks = Clocks(local)   # sampled over every timed run below
    for mode in ("plain", "device", "screened", "screened_device", "ablation", "screened_carry"):
        g = lkg.GSO(ctx, [(cid, swarms, glow)], pos, [seed])
        if mode != "plain" and mode != "device":
            g.set_screen(candidates=4, exact_fraction=0.25, rescore_every=10, train_steps=20, train_epochs=20,
                         finetune_epochs=2, lr=1e-3, seed=seed, random_rank=(mode == "ablation"), batch=1024,
                         carry_prediction=(mode == "screened_carry"))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.run(steps, device=mode in ("device", "screened_device"))
        g.finalize()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        st = g.state()
        res[mode] = dict(seconds=el, scored=g.scored, predicted=g.predicted, st=st, phases=g.timing())
        del g
    clk = clocks.stop()
    # the GSO's own spread: the plain run from the same start with the next
    # seed; its top-5 overlap with the plain run bounds what any run with a
    # different random stream can reach
    g = lkg.GSO(ctx, [(cid, swarms, glow)], pos, [seed + 1])
    g.run(steps)
    g.finalize()
    res["plain_next_seed"] = dict(st=g.state())
    del g
    ov = {}
    for mode in ("screened", "screened_device", "ablation", "screened_carry", "plain_next_seed"):
        o = []
        for k in range(swarms):
            sl = slice(k * glow, (k + 1) * glow)
            a, b = res[mode]["st"], res["plain"]["st"]
            o.append(top5_overlap(a["translation"][sl], a["scoring"][sl], b["translation"][sl], b["scoring"][sl]))
        ov[mode] = float(np.mean(o))
    best = {m: float(np.mean(res[m]["st"]["scoring"].reshape(swarms, glow).max(axis=1))) for m in res}
    t_plain = min(res["plain"]["seconds"], res["device"]["seconds"])
    t_scr = min(res["screened"]["seconds"], res["screened_device"]["seconds"])
    line = {"metric": "surrogate-screened GSO speedup over the plain GSO (e2e, same complex and start)",
            "value": t_plain / t_scr, "unit": "x", "n_gpus": world,
            "what": "the faster plain GSO (host or device steps) over the faster screened GSO",
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": args.workload, "family": family, "swarms": swarms, "glowworms": glow, "steps": steps,
                       "candidates": 4, "exact_fraction": 0.25, "rescore_every": 10, "train_steps": 20,
                       "tile_shape": {k: shape.get(k) for k in ("tile", "group", "cell", "xsub", "source")}},
            "plain": {"seconds": res["plain"]["seconds"], "exact_evals": res["plain"]["scored"],
                      "mean_best_score": best["plain"], "phases_s": res["plain"]["phases"]},
            "plain_device_gso": {"seconds": res["device"]["seconds"], "exact_evals": res["device"]["scored"],
                                 "mean_best_score": best["device"], "speedup_over_host_gso":
                                 res["plain"]["seconds"] / res["device"]["seconds"],
                                 "what": "the plain GSO with whole steps on the device (graph replays)"},
            "screened": {"seconds": res["screened"]["seconds"], "exact_evals": res["screened"]["scored"],
                         "surrogate_evals": res["screened"]["predicted"], "mean_best_score": best["screened"],
                         "top5_overlap_with_plain": ov["screened"], "phases_s": res["screened"]["phases"]},
            "screened_device": {"seconds": res["screened_device"]["seconds"],
                                "speedup_over_host_gso": res["plain"]["seconds"] / res["screened_device"]["seconds"],
                                "exact_evals": res["screened_device"]["scored"],
                                "surrogate_evals": res["screened_device"]["predicted"],
                                "mean_best_score": best["screened_device"],
                                "top5_overlap_with_plain": ov["screened_device"],
                                "phases_s": res["screened_device"]["phases"],
                                "what": "the screened GSO with its steps after training on the device"},
            "ablation_no_network": {"seconds": res["ablation"]["seconds"], "exact_evals": res["ablation"]["scored"],
                                    "mean_best_score": best["ablation"], "top5_overlap_with_plain": ov["ablation"],
                                    "phases_s": res["ablation"]["phases"],
                                    "what": "the screened search with seeded random ranks instead of the network"},
            "screened_carry_prediction": {"seconds": res["screened_carry"]["seconds"],
                                          "exact_evals": res["screened_carry"]["scored"],
                                          "mean_best_score": best["screened_carry"],
                                          "top5_overlap_with_plain": ov["screened_carry"],
                                          "what": "the screened GSO whose unscored moves take current score + "
                                                  "predicted gain (the default keeps the last exact score)"},
            "plain_next_seed": {"mean_best_score": best["plain_next_seed"],
                                "top5_overlap_with_plain": ov["plain_next_seed"],
                                "what": "the plain GSO from the same start with GSO seed + 1: the overlap two "
                                        "plain runs reach"},
            "clocks": clk}
    if args.seeds > 1:
        line["seeds"] = seed_spread(lkg, ctx, cid, pos, swarms, glow, steps, seed, args.seeds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def seed_spread(lkg, ctx, cid, pos, swarms, glow, steps, seed0, n_seeds):
    """The screened run (device steps), the random-rank ablation and the
    plain run with the next GSO seed, each against the plain run of the same
    seed, over GSO seeds seed0 .. seed0 + n_seeds - 1 from the same start:
    mean and standard deviation of the top-5 overlap and of the mean best
    score per swarm, and the per-seed values."""
    def run(seed, mode):
        g = lkg.GSO(ctx, [(cid, swarms, glow)], pos, [seed])
        if mode in ("screened", "ablation"):
            g.set_screen(candidates=4, exact_fraction=0.25, rescore_every=10, train_steps=20, train_epochs=20,
                         finetune_epochs=2, lr=1e-3, seed=seed, random_rank=(mode == "ablation"), batch=1024)
        g.run(steps, device=(mode == "screened"))
        g.finalize()
        st = g.state()
        del g
        return st

    def overlap(a, b):
        o = []
        for k in range(swarms):
            sl = slice(k * glow, (k + 1) * glow)
            o.append(top5_overlap(a["translation"][sl], a["scoring"][sl], b["translation"][sl], b["scoring"][sl]))
        return float(np.mean(o))

    def best(st):
        return float(np.mean(st["scoring"].reshape(swarms, glow).max(axis=1)))

    plain = [run(seed0 + i, "plain") for i in range(n_seeds + 1)]
    per = {"screened": [], "ablation": [], "plain_next_seed": []}
    for i in range(n_seeds):
        s = seed0 + i
        for mode in ("screened", "ablation"):
            st = run(s, mode)
            per[mode].append({"seed": s, "top5_overlap": overlap(st, plain[i]), "mean_best_score": best(st)})
        per["plain_next_seed"].append({"seed": s + 1, "top5_overlap": overlap(plain[i + 1], plain[i]),
                                       "mean_best_score": best(plain[i + 1])})
    out = {"seeds": [seed0 + i for i in range(n_seeds)],
           "plain_mean_best_score": [best(p) for p in plain[:n_seeds]]}
    for mode, rows in per.items():
        ov = np.array([r["top5_overlap"] for r in rows])
        bs = np.array([r["mean_best_score"] for r in rows])
        out[mode] = {"top5_overlap_mean": float(ov.mean()), "top5_overlap_std": float(ov.std()),
                     "mean_best_score_mean": float(bs.mean()), "mean_best_score_std": float(bs.std()),
                     "per_seed": rows}
    return out


if __name__ == "__main__":
    main()
