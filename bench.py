#!/usr/bin/env python
"""Throughput of the TSR volumetric core (octree + occupancy field + dual
marching cells) on B200, in samples/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload csg4m|sphere|heldout16m]

A step is one reconstruction of the workload's samples: tree build, both
cone-kernel passes, priors, occupancy values and DMC.

* ``value``  -- samples resident in HBM when the timed region starts
  (tsr_tree_build_device), CUDA events on the launching stream.
* ``e2e``    -- the same step through the public API (tsr_b200.core.Tree /
  Occupancy / extractCrust) from pinned host buffers: H2D of the samples and
  the cameras, and the mesh (case codes, vertices, triangles) copied back,
  every step.
* ``--impl reference`` -- the FP64 CPU oracle (a restatement of the reference's
  C++ path, which cannot be built here) on the host cores, same metric.
* ``next_rows`` (1 GPU, not timed into the headline) -- the paths either side
  of the hot path with the CPU restatement timed beside each: the crust's
  post-processing, depth-map triangulation, the incremental field update
  and the tree/field files (``--no-next-rows`` skips them).

Multi-GPU: replicas only (each rank reconstructs its own seeded scene; there
is no data-path collective); value = all ranks' samples / max rank time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "samples/s (octree+occupancy+DMC) MLP-pruned vs plain FP32 on B200, fixed mesh error"
UNIT = "samples/s"
L2_BYTES = 126 * 1024 * 1024
# DRAM bytes per unit (per link for the cone passes, per leaf for the priors),
# from the ncu capture summarised in profiles/occupancy_kernels_csg1m.md
TRAFFIC_PER_UNIT = {"occ.sampleness": 161.0, "occ.emptiness": 163.5, "occ.priors": 197.2}
CPU_SAMPLE_N = 60_000


WORKLOADS = {
    "csg4m": ("csg: 2 mm plate + cylinder r=0.3 + torus R=0.5/r=0.1, 120 cameras at 1.5-12, 4M samples",
              4_000_000),
    "csg1m": ("csg (as csg4m) subsampled to 1M samples, for profiling", 1_000_000),
    "sphere": ("unit sphere, 24 cameras, ~250k samples", 250_000),
    "heldout16m": ("held-out random CSG scene, 16M samples", 16_000_000),
}


def make_scene(workload, seed):
    from tsr_b200 import scenes
    desc = WORKLOADS[workload][0]
    if workload == "csg4m":
        return scenes.csg_scene(seed=seed, n_target=4_000_000), desc
    if workload == "csg1m":
        return scenes.csg_scene(seed=seed, n_target=1_000_000), desc
    if workload == "sphere":
        return scenes.sphere_scene(seed=seed, stride=3), desc
    if workload == "heldout16m":
        return scenes.random_csg_scene(seed=999 + seed, n_target=16_000_000, width=2200, height=1650,
                                       f=1650.0), desc
    raise SystemExit("unknown workload " + workload)


def cpu_scene(workload):
    from tsr_b200 import scenes
    if workload == "sphere":
        return scenes.sphere_scene(stride=9)
    return scenes.csg_scene(seed=0, n_target=CPU_SAMPLE_N)


def run_oracle_once(scene, threads):
    from oracle.pyoracle import Oracle
    t0 = time.perf_counter()
    o = Oracle(scene)
    o.build_tree()
    o.occupancy(nthreads=threads)
    o.dmc()
    return time.perf_counter() - t0


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = ROOT / "gpurun_out" / ("clocks_%d.csv" % index)

    def start(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.close()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def replica_throughput(samples_this_rank, seconds_this_rank, steps, dist=None):
    """Whole-job samples/s of N independent replicas: every rank's samples
    over the slowest rank's time (max over ranks)."""
    if dist is None:
        return samples_this_rank * steps / seconds_this_rank
    import torch
    t = torch.tensor([seconds_this_rank, float(samples_this_rank)], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(tot[1]) * steps / float(mx[0])


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    scene = cpu_scene(args.workload)
    for _ in range(args.warmup):
        run_oracle_once(scene, threads)
    times = [run_oracle_once(scene, threads) for _ in range(args.steps)]
    t = sum(times)
    value = scene.n * args.steps / t
    sample = "each step: the oracle's full pipeline (tree, occupancy, priors, DMC) on %d samples of the " \
             "same geometry and cameras, a bounded sample of the workload" % scene.n
    desc, full_n = WORKLOADS[args.workload]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "samples": full_n, "samples_per_timed_step": scene.n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def our_arm(args):
    import ctypes

    import numpy as np
    import torch
    from tsr_b200 import core

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    scene, desc = make_scene(args.workload, seed=rank)
    n = scene.n
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    params = core.params_default()
    cams = core.Cameras(scene.cams)

    # ---- device-resident inputs for the `value` leg
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
           dict(pos=scene.pos, nrm=scene.nrm, scale=scene.scale, conf=scene.conf,
                links=scene.links.astype(np.int32)).items()}
    dview = core.tsr_samples_view(n, scene.k, dev["pos"].data_ptr(), dev["nrm"].data_ptr(), dev["scale"].data_ptr(),
                                  dev["conf"].data_ptr(), dev["links"].data_ptr())

    pruner_view = None

    def device_step(pruned=False):
        tree = ctypes.c_void_p()
        core._check(core.lib.tsr_tree_build_device(ctypes.byref(dview), ctypes.byref(params), sptr,
                                                   ctypes.byref(tree)))
        occ = ctypes.c_void_p()
        if pruned:
            core._check(core.lib.tsr_occupancy_compute_pruned(tree, ctypes.byref(cams.view()), ctypes.byref(params),
                                                              ctypes.byref(pruner_view), sptr, ctypes.byref(occ)))
        else:
            core._check(core.lib.tsr_occupancy_compute(tree, ctypes.byref(cams.view()), ctypes.byref(params), 0,
                                                       sptr, ctypes.byref(occ)))
        mesh = ctypes.c_void_p()
        core._check(core.lib.tsr_dmc_extract(tree, occ, sptr, ctypes.byref(mesh)))
        tc = core.tsr_tree_counts()
        core._check(core.lib.tsr_tree_get_counts(tree, ctypes.byref(tc)))
        mc = core.tsr_mesh_counts()
        core._check(core.lib.tsr_mesh_get_counts(mesh, ctypes.byref(mc)))
        tms = np.zeros(8, np.float32)
        oms = np.zeros(8, np.float32)
        core.lib.tsr_tree_stage_ms(tree, core._ptr(tms), 8)
        core.lib.tsr_occupancy_stage_ms(occ, core._ptr(oms), 8)
        oc = core.tsr_occupancy_counts()
        core._check(core.lib.tsr_occupancy_get_counts(occ, ctypes.byref(oc)))
        core.lib.tsr_mesh_free(mesh)
        core.lib.tsr_occupancy_free(occ)
        core.lib.tsr_tree_free(tree)
        return tc, mc, tms, oms, oc

    # ---- host buffers (pinned) for the e2e leg
    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True)
        t.numpy()[...] = a
        return t

    host = {k: pinned(np.ascontiguousarray(v)) for k, v in
            dict(pos=scene.pos, nrm=scene.nrm, scale=scene.scale, conf=scene.conf,
                 links=scene.links.astype(np.int32)).items()}

    def e2e_step():
        # the samples stay in the caller's pinned buffers; the tree keeps its
        # reordered copy in HBM (reorder_samples=False), the mesh comes back
        s = core.Samples(host["pos"].numpy(), host["nrm"].numpy(), host["scale"].numpy(), host["conf"].numpy(),
                         host["links"].numpy().view(np.uint32))
        tree = core.Tree(s, params, stream=stream, reorder_samples=False)
        occ = core.Occupancy(tree, cams, params, stream=stream)
        mesh = occ.extractCrust(stream=stream)
        return tree, mesh

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # the clock sampler starts before the warm-up: its start-up (nvidia-smi
    # initialising NVML) stalls CUDA calls briefly and must not land in a
    # timed step; it keeps sampling through the timed region
    clocks = Clocks(local)
    clocks.start()
    for _ in range(args.warmup):
        device_step()
    # ---- timed: value (device-resident inputs)
    barrier()
    l0 = core.kernel_launches()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage_sum = np.zeros(16)
    for i in range(args.steps):
        ev[i][0].record(stream)
        tc, mc, tms, oms, oc = device_step()
        ev[i][1].record(stream)
        stage_sum += np.concatenate([tms, oms])
    barrier()
    launches = core.kernel_launches() - l0
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_value = sum(step_ms) / 1e3
    t_value = max_over_ranks(t_value)

    # ---- timed: e2e through the public API from pinned host buffers
    h2d = n * (24 + 24 + 8 + 8 + 4 * scene.k) + scene.cams.nbytes
    t_e2e, d2h, e2e_step_ms = None, 0, []
    if not args.value_only:
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
        barrier()
        eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for i in range(args.steps):
            eev[i][0].record(stream)
            tree, mesh = e2e_step()
            eev[i][1].record(stream)
        barrier()
        e2e_step_ms = [a.elapsed_time(b) for a, b in eev]
        t_e2e = max_over_ranks(sum(e2e_step_ms) / 1e3)
        d2h = mesh.cases.nbytes + mesh.positions.nbytes + mesh.scales.nbytes + mesh.edge_keys.nbytes + \
            mesh.triangles.nbytes

    # ---- roofline of the dominant kernel (per-launch algorithmic bytes / event time)
    stage_ms = stage_sum / args.steps
    names = ["tree.containment", "tree.sampling", "tree.balance", "tree.relayout", "tree.neighbors",
             "tree.dual_cells", "sub.sampling_eval", "sub.sampling_resolve", "occ.sampleness", "occ.flags", "occ.emptiness", "occ.priors", "occ.finalize",
             "", "", ""]
    stages = {nm: float(v) for nm, v in zip(names, stage_ms) if nm}
    K = scene.k
    Nn, Nl = tc.nodes, tc.leaves
    per_pass = n * (32 + 4 * K) + Nn * 8 + Nl * 16       # per cone pass
    alg = {"occ.sampleness": per_pass, "occ.emptiness": per_pass, "occ.priors": Nl * (16 + 8),
           "occ.finalize": Nl * (32 + 8)}
    dom = max(alg, key=lambda k: stages[k])
    # DRAM bytes (read + write) per unit from one ncu capture of each kernel on
    # the csg1m workload (profiles/occupancy_kernels_csg1m.md), scaled by the
    # units of this run: links for the cone passes, leaves for the priors
    units = {"occ.sampleness": n * K, "occ.emptiness": n * K, "occ.priors": Nl}
    traffic = None
    if dom in TRAFFIC_PER_UNIT:
        traffic = int(TRAFFIC_PER_UNIT[dom] * units[dom])
    hbm, src = peaks()
    achieved = alg[dom] / (stages[dom] / 1e3) / 1e9
    total_ms = sum(v for k, v in stages.items() if not k.startswith("sub."))

    world_samples = n * world
    line = {
        "metric": METRIC, "value": world_samples * args.steps / t_value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_value / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": desc, "samples": n, "cameras": int(scene.cams.shape[0]), "k": K,
                   "mode": "plain path: FP32 kernel evaluation with FP64 per-leaf accumulation, FP64 topology",
                   "l2": "inputs %d MB > 126 MB L2; all buffers re-allocated each step" % (h2d // 2**20),
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "nodes": Nn, "leaves": Nl, "dual_cells": tc.dual_cells, "triangles": mc.triangles,
                   "accepted_pairs": {"sampleness": oc.accepted_sampleness, "emptiness": oc.accepted_emptiness},
                   "nodes_visited": {"sampleness": oc.visited_sampleness, "emptiness": oc.visited_emptiness,
                                     "priors": oc.visited_priors},
                   "sampling": {"rounds": tc.sampling_rounds, "waves": tc.sampling_waves,
                                "writers": tc.sampling_writers}},
        "e2e": None if t_e2e is None else {"value": world_samples * args.steps / t_e2e, "unit": UNIT,
                                            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                                            "step_ms": [round(x, 3) for x in e2e_step_ms]},
        "gpu_launches": int(launches),
        "step_ms": [round(x, 3) for x in step_ms],
        "stage_ms": {k: round(v, 3) for k, v in stages.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_source": src + " (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes": int(alg[dom]), "kernel_ms": stages[dom],
                     "share_of_step": stages[dom] / total_ms if total_ms else None, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per unit on csg1m, "
                                       "scaled to this run's units"},
        # the survey's secondary figures: the traversals' work rates (what bounds them, not HBM)
        "secondary": {
            "node_tests_per_s": {"sampleness": oc.visited_sampleness / (stages["occ.sampleness"] / 1e3),
                                 "emptiness": oc.visited_emptiness / (stages["occ.emptiness"] / 1e3),
                                 "priors": oc.visited_priors / (stages["occ.priors"] / 1e3)},
            "accepted_pairs_per_s": {"sampleness": oc.accepted_sampleness / (stages["occ.sampleness"] / 1e3),
                                     "emptiness": oc.accepted_emptiness / (stages["occ.emptiness"] / 1e3)}},
        "clocks": clk,
    }
    # ---- the learned pruner's field (same workload, same timing), judged by
    # the plain method on this scene
    if not args.no_pruned:
        pr = core.Pruner.load()
        pruner_view = pr.view()
        for _ in range(max(1, args.warmup // 2)):
            device_step(pruned=True)
        barrier()
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        pstage = np.zeros(16)
        for i in range(args.steps):
            pev[i][0].record(stream)
            _, _, ptms, poms, poc = device_step(pruned=True)
            pev[i][1].record(stream)
            pstage += np.concatenate([ptms, poms])
        barrier()
        p_step_ms = [a.elapsed_time(b) for a, b in pev]
        t_pruned = max_over_ranks(sum(p_step_ms) / 1e3)
        from tsr_b200 import pruner as pruner_mod
        jt = core.Tree(core.Samples(scene.pos, scene.nrm, scene.scale, scene.conf, scene.links), params,
                       stream=stream, reorder_samples=False)
        j = pruner_mod.judge(jt, cams, pr, params, stream=stream)
        del jt
        line["pruned"] = {
            "value": world_samples * args.steps / t_pruned, "unit": UNIT, "ms_per_step": 1e3 * t_pruned / args.steps,
            "step_ms": [round(x, 3) for x in p_step_ms],
            "speedup_vs_plain": t_value / t_pruned,
            "skipped_prior_queries": poc.pruned_leaves, "repaired_leaves": poc.repaired_leaves, "leaves": int(Nl),
            "stage_ms": {k: round(float(v), 3) for k, v in zip(names, pstage / args.steps) if k},
            "judge": {"sign_agreement": j["sign_agreement"], "case_agreement": j["case_agreement"],
                      "vertex_hausdorff": j["vertex_hausdorff"], "finest_leaf_size": j["finest_leaf_size"],
                      "triangles_plain_pruned": j["triangles"]},
            "network": "tsr_b200/pruner_weights.npz (trained on 7 random CSG scenes of 1M samples, seeds 1-7)",
        }
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cs = cpu_scene(args.workload)
        tcpu = run_oracle_once(cs, threads)
        line["cpu_baseline"] = {"value": cs.n / tcpu, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": "FP64 oracle full pipeline on the same geometry and cameras at %d samples"
                                % cs.n}
    if rank == 0 and world == 1 and not args.no_next_rows:
        line["next_rows"] = next_rows(core, scene, cams, params, stream, line["ms_per_step"],
                                      cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def next_rows(core, scene, cams, params, stream, ms_per_step, cpu=True):
    """Measurements of the paths either side of the hot path, on this GPU with
    the CPU restatement timed beside each: the crust's post-processing
    (DualMarchingCells.cpp:31-36), depth-map triangulation (the samples'
    source, DepthImage::triangulate), the incremental field update
    (Occupancy::eraseSamples) and the tree/field files.  Each entry is
    independent and reports an error instead of failing the run."""
    import ctypes
    import tempfile

    import numpy as np
    import torch
    from oracle import pyoracle
    from tsr_b200 import scenes

    hbm, src = peaks()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    out = {}

    def ev_ms(fn, reps):
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            prep = fn(None)
            a.record(stream)
            fn(prep)
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return ms

    samples = core.Samples(scene.pos, scene.nrm, scene.scale, scene.conf, scene.links)
    tree = core.Tree(samples, params, stream=stream, reorder_samples=False)
    occ = core.Occupancy(tree, cams, params, stream=stream)
    try:
        raw = occ.extractCrust(stream=stream)
        holder = {}

        def post(prep):
            if prep is None:   # a fresh raw mesh, untimed
                h = ctypes.c_void_p()
                core._check(core.lib.tsr_dmc_extract(tree.handle, occ.handle, sptr, ctypes.byref(h)))
                holder["h"] = h
                return h
            pc = core.tsr_mesh_post_counts()
            core._check(core.lib.tsr_mesh_postprocess(prep, 1000, ctypes.byref(pc)))
            holder["pc"] = pc
            core.lib.tsr_mesh_free(prep)

        post(post(None))
        ms = ev_ms(post, 5)
        pc = holder["pc"]
        nv, nt = raw.positions.shape[0], raw.triangles.shape[0]
        oc, tcpu = None, None
        if cpu:
            t0 = time.perf_counter()
            oc = pyoracle.mesh_postprocess(raw.positions, raw.triangles, raw.scales, 1000)[0]
            tcpu = time.perf_counter() - t0
        alg = nt * 12 * 2 + nv * 24 * 3     # triangles read twice; positions read twice, normals written
        gpu_ms = statistics.median(ms)
        out["mesh_postprocess"] = {
            "what": "isle deletion (min 1000 vertices), hole filling, angle-weighted normals of this workload's "
                    "crust", "vertices": nv, "triangles": nt,
            "isle_vertices": pc.isle_vertices, "holes": pc.holes, "hole_triangles": pc.hole_triangles,
            "gpu_ms": gpu_ms, "cpu_ms": None if tcpu is None else 1e3 * tcpu,
            "cpu": "CPU restatement, 1 thread (kind: port)",
            "same_counts_as_cpu": None if oc is None else bool(
                oc["triangles"] == nt - pc.isle_triangles + pc.hole_triangles),
            "roofline": {"bound": "hbm", "algorithmic_bytes": alg, "achieved": alg / gpu_ms / 1e6, "peak": hbm,
                         "unit": "GB/s", "frac": alg / gpu_ms / 1e6 / hbm, "peak_source": src,
                         "note": "sorts, scans and one-thread ring search over a small mesh: launch-bound"}}
    except Exception as e:   # pragma: no cover - reported, not fatal
        out["mesh_postprocess"] = {"error": repr(e)}
    try:
        views = scenes.sphere_depth_views(width=1280, height=960, f=600.0, n_cams=4)

        def tri(prep, v=views[0]):
            if prep is None:
                return True
            core.DepthImage(v["depths"]).triangulate(v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"],
                                                     stream=stream)

        tri(True)
        ms = ev_ms(tri, 4)
        v = views[0]
        g = core.DepthImage(v["depths"]).triangulate(v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"],
                                                     stream=stream)
        tcpu = None
        if cpu:
            t0 = time.perf_counter()
            pyoracle.depth_triangulate(v["depths"], v["hps_to_ray_vs"], v["hps_to_ray_ws"], v["center"])
            tcpu = time.perf_counter() - t0
        npx = v["depths"].size
        nv, nt = g.positions.shape[0], g.triangles.shape[0]
        alg = npx * (8 + 4) + nv * (24 * 4 + 8) + nt * 12
        gpu_ms = statistics.median(ms)
        out["depth_triangulate"] = {
            "what": "DepthImage::triangulate of a 1280x960 depth map (sphere and plate), through the C ABI "
                    "from host memory (H2D of the map, mesh read back)",
            "pixels": npx, "vertices": nv, "triangles": nt, "gpu_ms": gpu_ms,
            "cpu_ms": None if tcpu is None else 1e3 * tcpu,
            "pixels_per_s_gpu": npx / gpu_ms * 1e3, "pixels_per_s_cpu": None if tcpu is None else npx / tcpu,
            "cpu": "CPU restatement, 1 thread (kind: port)",
            "roofline": {"bound": "hbm", "algorithmic_bytes": alg, "achieved": alg / gpu_ms / 1e6, "peak": hbm,
                         "unit": "GB/s", "frac": alg / gpu_ms / 1e6 / hbm, "peak_source": src}}
    except Exception as e:   # pragma: no cover
        out["depth_triangulate"] = {"error": repr(e)}
    try:
        rng = np.random.default_rng(7)
        chosen = np.sort(rng.choice(tree.sample_count, size=tree.sample_count // 100, replace=False))

        def upd(prep):
            if prep is None:
                holder["o"] = core.Occupancy(tree, cams, params, stream=stream)
                return True
            holder["o"].eraseSamples(chosen, cams, params)

        upd(upd(None))
        ms = ev_ms(upd, 3)
        out["occupancy_update"] = {
            "what": "Occupancy::eraseSamples of 1% of the samples (both cone passes over their links with "
                    "negated values, then priors and values of every leaf)",
            "samples_removed": int(chosen.shape[0]), "gpu_ms": statistics.median(ms),
            "full_step_ms": ms_per_step}
    except Exception as e:   # pragma: no cover
        out["occupancy_update"] = {"error": repr(e)}
    try:
        with tempfile.TemporaryDirectory() as d:
            prefix = os.path.join(d, "scene.octree")
            t0 = time.perf_counter()
            tree.saveToFiles(prefix)
            occ.saveToFile(os.path.join(d, "scene.occupancy"))
            tsave = time.perf_counter() - t0
            nbytes = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
            ordered = core.Samples(*_tree_samples(core, tree, scene.k))
            t0 = time.perf_counter()
            t2 = core.Tree.fromFiles(prefix, ordered, params=params, stream=stream)
            core.Occupancy.fromFile(t2, os.path.join(d, "scene.occupancy"), params, stream=stream)
            tload = time.perf_counter() - t0
        out["files"] = {"what": "tree (.nodes/.leaves/.dualCells) and field (.occupancy) of this workload: "
                                "save, then load with full validation (host I/O and checks)",
                        "bytes": nbytes, "save_s": tsave, "load_s": tload,
                        "save_gb_s": nbytes / tsave / 1e9, "load_gb_s": nbytes / tload / 1e9}
    except Exception as e:   # pragma: no cover
        out["files"] = {"error": repr(e)}
    return out


def _tree_samples(core, tree, k):
    """The tree's samples in tree order (what a .samples file holds)."""
    import numpy as np
    n = tree.sample_count
    pos, nrm, sc, cf = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n)
    links = np.zeros((n, k), np.uint32)
    core._check(core.lib.tsr_tree_copy_samples(tree.handle, core._ptr(pos), core._ptr(nrm), core._ptr(sc),
                                               core._ptr(cf), core._ptr(links)))
    return pos, nrm, sc, cf, links


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="csg4m", choices=["csg4m", "csg1m", "sphere", "heldout16m"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--value-only", action="store_true", help="skip the e2e leg (profiling runs)")
    ap.add_argument("--no-pruned", action="store_true", help="skip the learned pruner's leg")
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the measurements of post-processing, depth maps, updates and files")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
