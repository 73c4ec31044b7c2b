#!/usr/bin/env python
"""Throughput of the TSR volumetric core (octree + occupancy field + dual
marching cells) on B200, in samples/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload heldout16m|csg4m|csg1m|sphere|cluttered60m|vase100m]

A step is one reconstruction of the workload's samples: tree build, both
cone-kernel passes, priors, occupancy values and DMC.  The default workload
is the held-out 16M-sample random CSG scene, the size the pruned-vs-plain
target is stated at; its samples are rendered on the GPU before timing.

* ``value``  -- samples resident in HBM when the timed region starts
  (tsr_tree_build_device), CUDA events on the launching stream: the plain
  FP32 path.
* ``pruned`` -- the same steps with the learned pruner's field
  (tsr_occupancy_compute_pruned), compared with the plain field on this scene.
* ``e2e``    -- the plain step through the C ABI from pinned host buffers:
  H2D of the samples and the cameras, the tree build, the reordered samples
  copied back (the reference reorders Samples in place), the field, DMC and
  the mesh (case codes, vertices, scales, edge keys, triangles) copied back,
  every handle freed inside its step.
* ``cpu_baseline`` -- the reference's own hot path (oracle/_ref: its sources
  built against the BaseProject shim) on a 3k-sample version of the
  workload's scene, with the FP64 oracle port's time on 60k samples beside it.
* ``fp64_check`` -- the GPU's field and mesh (plain and pruned) against the
  FP64 oracle's on the 60k-sample scene: per-field error, sign flips, case
  codes, mesh Hausdorff.
* ``--impl reference`` -- the reference build on the host cores, same metric
  (the oracle port where the reference build is absent).
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
# DRAM bytes (read + write) per unit of the occupancy kernels -- per link for
# the cone passes, per leaf for the priors -- from one ncu capture of each
# kernel on the 1M-sample CSG workload; the per-unit traffic is flat in the
# size (one read of the per-link records and of the prior table)
TRAFFIC_PER_UNIT = {"occ.sampleness": 160.0, "occ.emptiness": 161.1, "occ.priors": 158.3}
CPU_SAMPLE_N = 60_000     # the oracle port's sample (fp64_check)
REF_SAMPLE_N = 3_000      # the reference build's sample per timed step (~4-6 s on 8-16 host threads)


WORKLOADS = {
    "heldout16m": ("held-out random CSG scene (seed 999: 3-8 spheres/boxes/cylinders/thin plates, 64-160 cameras "
                   "at 1.5-8, 2200x1650, f=1650), 16M samples, depth noise 0.5%, normal jitter 8 deg", 16_000_000),
    "csg4m": ("csg: 2 mm plate + cylinder r=0.3 + torus R=0.5/r=0.1, 120 cameras at 1.5-12, 4M samples",
              4_000_000),
    "csg1m": ("csg (as csg4m) subsampled to 1M samples, for profiling", 1_000_000),
    "sphere": ("unit sphere, 24 cameras, ~250k samples", 250_000),
    "cluttered60m": ("cluttered scene: 24 random primitives on a ground plate, 400 cameras at 1920x1080, f=1400, "
                     "60M samples, 5% outliers uniform in the bounding box, depth noise 1%, confidence U[0.2,1]",
                     60_000_000),
    "vase100m": ("density stress: vase with a 1 mm wall on a ground plane, 1000 cameras at 0.3-300 "
                 "(log-uniform), 1024x768, f=900, 100M samples", 100_000_000),
}


def make_scene(workload, seed):
    """The workload's samples, generated on the current CUDA device (a
    DeviceScene) or on the host for the small ones (a Scene)."""
    from tsr_b200 import scenes
    desc = WORKLOADS[workload][0]
    if workload == "heldout16m":
        return scenes.random_csg_scene_device(999 + seed, 16_000_000, 2200, 1650, 1650.0), desc
    if workload == "csg4m":
        return scenes.csg_scene_device(seed=seed, n_target=4_000_000), desc
    if workload == "csg1m":
        return scenes.csg_scene_device(seed=seed, n_target=1_000_000), desc
    if workload == "sphere":
        return scenes.sphere_scene(seed=seed, stride=3), desc
    if workload == "cluttered60m":
        return scenes.cluttered_scene_device(seed=seed), desc
    if workload == "vase100m":
        return scenes.vase_scene_device(seed=seed), desc
    raise SystemExit("unknown workload " + workload)


def cpu_scene(workload, n=CPU_SAMPLE_N):
    """A bounded sample of the workload for the CPU paths: the same geometry,
    cameras and image resolution (so the same sample scales), n samples
    (rendered with torch on the host)."""
    import numpy as np
    from tsr_b200 import scenes
    if workload == "sphere":
        sc = scenes.sphere_scene(stride=3)
        return sc.subset(np.sort(np.random.default_rng(0).choice(sc.n, size=min(n, sc.n), replace=False)))
    if workload == "heldout16m":
        return scenes.random_csg_scene_device(999, n, 2200, 1650, 1650.0, device="cpu").host()
    if workload == "cluttered60m":
        return scenes.cluttered_scene_device(n_target=n, device="cpu").host()
    if workload == "vase100m":
        return scenes.vase_scene_device(n_target=n, device="cpu").host()
    return scenes.csg_scene_device(seed=0, n_target=n, device="cpu").host()


def run_oracle_once(scene, threads, keep=False):
    from oracle.pyoracle import Oracle
    t0 = time.perf_counter()
    o = Oracle(scene)
    o.build_tree()
    o.occupancy(nthreads=threads)
    o.mesh = o.dmc()
    t = time.perf_counter() - t0
    return (t, o) if keep else t


def reference_available():
    try:
        from oracle import refpy
        return refpy.available()
    except Exception:
        return False


def run_reference_once(scene, threads):
    """The reference's own hot path (its Scene/Tree and SurfaceExtraction
    sources built against the BaseProject shim, oracle/_ref): Tree::Tree(),
    Occupancy(tree) and extractCrust() on `threads` OpenMP threads."""
    from oracle import refpy
    t0 = time.perf_counter()
    refpy.run(scene, threads=threads, outputs=False)
    return time.perf_counter() - t0


class Clocks:
    """nvidia-smi sampling during the timed region (into a temporary file)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, path=None):
        import tempfile
        self.index = index
        self.p = None
        self.path = Path(path) if path else Path(tempfile.gettempdir()) / ("tsr_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
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
                "samples": len(rows), "log": str(self.path)}


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
    if reference_available():
        kind = "reference"
        scene = cpu_scene(args.workload, REF_SAMPLE_N)
        once = run_reference_once
        what = ("the reference's own Tree::Tree(), Occupancy(tree) and extractCrust() (its sources built "
                "unmodified against the BaseProject shim, oracle/_ref)")
    else:
        kind = "port"
        scene = cpu_scene(args.workload)
        once = run_oracle_once
        what = "the oracle's full pipeline (the C++ restatement, bit-exact with the reference's build)"
    for _ in range(args.warmup):
        once(scene, threads)
    times = [once(scene, threads) for _ in range(args.steps)]
    t = sum(times)
    value = scene.n * args.steps / t
    sample = "each step: %s on %d samples of the same geometry, cameras and image resolution, a bounded " \
             "sample of the workload, %d host threads" % (what, scene.n, threads)
    desc, full_n = WORKLOADS[args.workload]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "samples": full_n, "samples_per_timed_step": scene.n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def fp64_check(core, scene, oracle, cams_np, params, pruner, stream):
    """The GPU field and mesh of `scene` (plain and pruned) against the FP64
    oracle's on the same scene: per-field max / mean relative error, sign
    flips, case-code mismatches, and the symmetric vertex Hausdorff distance
    of the meshes in units of the finest leaf size."""
    import numpy as np
    from tsr_b200 import pruner as pruner_mod
    f = oracle.fields()
    om = oracle.mesh
    tree = core.Tree(core.Samples.from_scene(scene), params, stream=stream)
    cams = core.Cameras(cams_np)
    finest = float(tree.getLeaves().scopes[:, 3].min())
    out = {"samples": scene.n, "leaves": tree.counts["leaves"], "finest_leaf_size": finest}
    for label, pr in (("plain", None), ("pruned", pruner)):
        occ = core.Occupancy(tree, cams, params, stream=stream, pruner=pr)
        mesh = occ.extractCrust(stream=stream)
        errs = {}
        for name, key in [("emptiness_sum", "e_sum"), ("sampleness_sum", "s_sum"),
                          ("emptiness_length", "e_len"), ("sampleness_length", "s_len"),
                          ("prior_emptiness", "prior"), ("occupancy", "occ")]:
            a, b = occ.field(name), f[key]
            ok = np.isfinite(a) & np.isfinite(b)   # the pruned field has no prior where it skipped the query
            if not ok.any():
                continue
            d = np.abs(a[ok] - b[ok])
            rel = d / np.maximum(np.abs(b[ok]), 1e-300)
            errs[name] = {"max_abs": float(d.max()), "mean_abs": float(d.mean()),
                          "max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "compared": int(ok.sum())}
        occ_g, occ_o = occ.getOccupancy(), f["occ"]
        entry = {"field_error": errs, "sign_flips": int(((occ_g > 0) != (occ_o > 0)).sum())}
        entry["case_mismatches"] = int((mesh.cases != om["cases"]).sum())
        entry["hausdorff_vs_fp64"] = pruner_mod.vertex_hausdorff(mesh.positions, om["vpos"])
        entry["hausdorff_vs_fp64_finest_leaves"] = entry["hausdorff_vs_fp64"] / finest
        entry["triangles_gpu_fp64"] = [int(mesh.triangles.shape[0]), int(om["tris"].shape[0])]
        out[label] = entry
    return out


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

    t_gen = time.perf_counter()
    scene, desc = make_scene(args.workload, seed=rank)
    n = scene.n
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    params = core.params_default()
    cams = core.Cameras(scene.cams)

    # ---- device-resident inputs for the `value` leg
    if isinstance(scene.pos, np.ndarray):
        dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
               dict(pos=scene.pos, nrm=scene.nrm, scale=scene.scale, conf=scene.conf,
                    links=scene.links.view(np.int32)).items()}
    else:
        dev = dict(pos=scene.pos, nrm=scene.nrm, scale=scene.scale, conf=scene.conf, links=scene.links)
    dview = core.tsr_samples_view(n, scene.k, dev["pos"].data_ptr(), dev["nrm"].data_ptr(), dev["scale"].data_ptr(),
                                  dev["conf"].data_ptr(), dev["links"].data_ptr())

    # ---- pinned host inputs for the e2e leg (what a caller holds)
    def pinned_like(t):
        return torch.empty(t.shape, dtype=t.dtype, pin_memory=True)

    host = {}
    for k, v in dev.items():
        h = pinned_like(v)
        h.copy_(v)
        host[k] = h
    torch.cuda.synchronize()
    torch.cuda.empty_cache()   # the renderer's temporaries go back to the device for the library's pool
    gen_s = time.perf_counter() - t_gen

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

    # ---- the e2e step: the C ABI from the caller's pinned host buffers, as
    # the reference's callers use it -- Tree::Tree() (H2D of the samples, the
    # build, and the in-place sample reorder: the reordered samples copied
    # back into host buffers, Nodes.cpp:630), Occupancy(tree), extractCrust()
    # with the mesh (case codes, vertices, scales, edge keys, triangles) read
    # back into host buffers.  Every handle is freed inside its step.
    hview = core.tsr_samples_view(n, scene.k, host["pos"].data_ptr(), host["nrm"].data_ptr(),
                                  host["scale"].data_ptr(), host["conf"].data_ptr(), host["links"].data_ptr())
    reordered = {k: pinned_like(v) for k, v in host.items()}
    mesh_out = {}

    def mesh_buffers(tc, mc):
        need = {"cases": (tc.dual_cells, np.uint8), "positions": (mc.vertices * 3, np.float64),
                "scales": (mc.vertices, np.float64), "edge_keys": (mc.vertices * 2, np.uint32),
                "triangles": (mc.triangles * 3, np.uint32)}
        for k, (cnt, dt) in need.items():
            if k not in mesh_out or mesh_out[k].numel() < cnt:
                mesh_out[k] = torch.empty(max(1, int(cnt * 1.25)), dtype=torch.from_numpy(np.zeros(1, dt)).dtype,
                                          pin_memory=True)
        return sum(int(cnt) * np.dtype(dt).itemsize for cnt, dt in need.values())

    def e2e_step():
        tree = ctypes.c_void_p()
        occ = ctypes.c_void_p()
        mesh = ctypes.c_void_p()
        try:
            core._check(core.lib.tsr_tree_build(ctypes.byref(hview), ctypes.byref(params), sptr, ctypes.byref(tree)))
            core._check(core.lib.tsr_tree_copy_samples(tree, *[ctypes.c_void_p(reordered[k].data_ptr()) for k in
                                                                ("pos", "nrm", "scale", "conf", "links")]))
            core._check(core.lib.tsr_occupancy_compute(tree, ctypes.byref(cams.view()), ctypes.byref(params), 0,
                                                       sptr, ctypes.byref(occ)))
            core._check(core.lib.tsr_dmc_extract(tree, occ, sptr, ctypes.byref(mesh)))
            tc = core.tsr_tree_counts()
            core._check(core.lib.tsr_tree_get_counts(tree, ctypes.byref(tc)))
            mc = core.tsr_mesh_counts()
            core._check(core.lib.tsr_mesh_get_counts(mesh, ctypes.byref(mc)))
            d2h = mesh_buffers(tc, mc)
            core._check(core.lib.tsr_mesh_copy(mesh, *[ctypes.c_void_p(mesh_out[k].data_ptr()) for k in
                                                       ("cases", "positions", "scales", "edge_keys", "triangles")]))
            return d2h + sum(v.numel() * v.element_size() for v in reordered.values())
        finally:
            if mesh:
                core.lib.tsr_mesh_free(mesh)
            if occ:
                core.lib.tsr_occupancy_free(occ)
            if tree:
                core.lib.tsr_tree_free(tree)

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
    # timed step; it keeps sampling through the timed regions
    clocks = Clocks(local, args.clock_log)
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
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_value = sum(step_ms) / 1e3
    t_value = max_over_ranks(t_value)

    # ---- timed: e2e through the C ABI from pinned host buffers
    h2d = sum(v.numel() * v.element_size() for v in host.values()) + scene.cams.nbytes
    t_e2e, d2h, e2e_step_ms = None, 0, []
    if not args.value_only:
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
        barrier()
        eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for i in range(args.steps):
            eev[i][0].record(stream)
            d2h = e2e_step()
            eev[i][1].record(stream)
        barrier()
        e2e_step_ms = [a.elapsed_time(b) for a, b in eev]
        t_e2e = max_over_ranks(sum(e2e_step_ms) / 1e3)

    # ---- roofline of the dominant kernel (per-launch algorithmic bytes / event time)
    stage_ms = stage_sum / args.steps
    names = ["tree.containment", "tree.sampling", "tree.balance", "tree.relayout", "tree.neighbors",
             "tree.dual_cells", "sub.sampling_eval", "sub.sampling_resolve", "occ.sampleness", "occ.flags",
             "occ.emptiness", "occ.priors", "occ.finalize", "", "", ""]
    stages = {nm: float(v) for nm, v in zip(names, stage_ms) if nm}
    K = scene.k
    Nn, Nl = tc.nodes, tc.leaves
    per_pass = n * (32 + 4 * K) + Nn * 8 + Nl * 16       # per cone pass
    alg = {"occ.sampleness": per_pass, "occ.emptiness": per_pass, "occ.priors": Nl * (16 + 8),
           "occ.finalize": Nl * (32 + 8)}
    dom = max(alg, key=lambda k: stages[k])
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
                   "mode": "plain path: FP32 kernel evaluation with FP64 per-leaf accumulation (FP64 atomics "
                           "instead of Kahan-compensated FP32), FP64 topology",
                   "l2": "inputs %d MB > 126 MB L2; all buffers re-allocated each step" % (h2d // 2**20),
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "scene_generation_s": round(gen_s, 2),
                   "nodes": Nn, "leaves": Nl, "dual_cells": tc.dual_cells, "triangles": mc.triangles,
                   "accepted_pairs": {"sampleness": oc.accepted_sampleness, "emptiness": oc.accepted_emptiness},
                   "nodes_visited": {"sampleness": oc.visited_sampleness, "emptiness": oc.visited_emptiness,
                                     "priors": oc.visited_priors},
                   "sampling": {"rounds": tc.sampling_rounds, "waves": tc.sampling_waves,
                                "writers": tc.sampling_writers}},
        "e2e": None if t_e2e is None else {"value": world_samples * args.steps / t_e2e, "unit": UNIT,
                                            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                                            "ms_per_step": 1e3 * t_e2e / args.steps,
                                            "what": "C ABI from pinned host buffers: H2D of samples and cameras, "
                                                    "tree build, reordered samples copied back (the in-place "
                                                    "reorder), field, DMC, mesh copied back; handles freed in-step",
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
        # secondary figures: the traversals' work rates (what bounds them, not HBM)
        "secondary": {
            "node_tests_per_s": {"sampleness": oc.visited_sampleness / (stages["occ.sampleness"] / 1e3),
                                 "emptiness": oc.visited_emptiness / (stages["occ.emptiness"] / 1e3),
                                 "priors": oc.visited_priors / (stages["occ.priors"] / 1e3)},
            "accepted_pairs_per_s": {"sampleness": oc.accepted_sampleness / (stages["occ.sampleness"] / 1e3),
                                     "emptiness": oc.accepted_emptiness / (stages["occ.emptiness"] / 1e3)}},
    }
    # ---- the learned pruner's field (same workload, same timing), compared with
    # the plain method on this scene
    pr = None
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
        clk = clocks.stop()
        from tsr_b200 import pruner as pruner_mod
        jt = core.Tree(core.Samples(host["pos"].numpy(), host["nrm"].numpy(), host["scale"].numpy(),
                                    host["conf"].numpy(), host["links"].numpy().view(np.uint32)), params,
                       stream=stream, reorder_samples=False)
        j = pruner_mod.compare_with_plain(jt, cams, pr, params, stream=stream)
        del jt
        line["pruned"] = {
            "value": world_samples * args.steps / t_pruned, "unit": UNIT, "ms_per_step": 1e3 * t_pruned / args.steps,
            "step_ms": [round(x, 3) for x in p_step_ms],
            "speedup_vs_plain": t_value / t_pruned,
            "skipped_prior_queries": poc.pruned_leaves, "repaired_leaves": poc.repaired_leaves,
            "certified_skips": poc.certified_leaves, "leaves": int(Nl),
            "stage_ms": {k: round(float(v), 3) for k, v in zip(names, pstage / args.steps) if k},
            "vs_plain": {"sign_agreement": j["sign_agreement"], "case_agreement": j["case_agreement"],
                         "vertex_hausdorff": j["vertex_hausdorff"], "finest_leaf_size": j["finest_leaf_size"],
                         "triangles_plain_pruned": j["triangles"], "visited_plain_pruned": j["visited"]},
            "network": pr.describe(),
        }
    else:
        clk = clocks.stop()
    line["clocks"] = clk
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        if reference_available():
            rs = cpu_scene(args.workload, REF_SAMPLE_N)
            tref = run_reference_once(rs, threads)
            line["cpu_baseline"] = {"value": rs.n / tref, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": "the reference's own tree, field and DMC (oracle/_ref: its sources "
                                              "built against the BaseProject shim) on %d samples of the same "
                                              "geometry, cameras and image resolution" % rs.n}
        cs = cpu_scene(args.workload)
        tcpu, orc = run_oracle_once(cs, threads, keep=True)
        port = {"value": cs.n / tcpu, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": "FP64 oracle (C++ restatement, bit-exact with the reference build; -O3 "
                          "-march=x86-64-v3, OpenMP) full pipeline on %d samples of the same geometry, cameras "
                          "and image resolution" % cs.n}
        if "cpu_baseline" in line:
            line["cpu_baseline"]["port"] = port
        else:
            line["cpu_baseline"] = port
        try:
            line["fp64_check"] = fp64_check(core, cs, orc, cs.cams, params, pr, stream)
            line["fp64_check"]["what"] = ("GPU field and mesh vs the FP64 oracle's (bit-exact with the reference "
                                          "build) on a %d-sample version of the workload's scene; the oracle "
                                          "cannot run the full workload in bench time" % cs.n)
        except Exception as e:   # pragma: no cover - reported, not fatal
            line["fp64_check"] = {"error": repr(e)}
        del orc
    if rank == 0 and world == 1 and not args.no_next_rows:
        hs = scene if isinstance(scene.pos, np.ndarray) else None
        if hs is None:
            from tsr_b200 import scenes as scenes_mod
            hs = scenes_mod.Scene(host["pos"].numpy(), host["nrm"].numpy(), host["scale"].numpy(),
                                  host["conf"].numpy(), host["links"].numpy().view(np.uint32), scene.cams, desc)
        line["next_rows"] = next_rows(core, hs, cams, params, stream, line["ms_per_step"],
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
    ap.add_argument("--workload", default="heldout16m", choices=list(WORKLOADS))
    ap.add_argument("--clock-log", default=None, help="file for the nvidia-smi clock samples (default: a temp file)")
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
