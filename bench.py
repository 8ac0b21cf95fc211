"""Benchmark of the closest-hit ray query on the 1,048,576-triangle heightfield.

Workload (synthetic, seeded - the reference ships no scenes): a 1024 x 512
cell heightfield over [0,1]^2 (value-noise fBm, amplitude 0.2, seed 1), with
4,194,304 coherent primary rays (2048^2 pinhole, 60 deg, eye (0.5,-0.6,0.8))
and 4,194,304 incoherent rays (origins on random triangles, cosine-hemisphere
directions). One step = one closest-hit pass over both ray sets, as one
batch of 8,388,608 rays (one ilg_intersect call: the coherent rays, then
the incoherent ones).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0. `value` is device-resident throughput (rays
already in HBM, hits left in HBM); `e2e` is the same query through the public
C ABI from pinned host buffers, copies included. Under torchrun each rank
traces its own full replica of the workload (weak scaling, no collective on
the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s closest-hit"
UNIT = "Mrays/s"
WORKLOAD = "ray batch: 1,048,576-tri heightfield, 4,194,304 coherent + 4,194,304 incoherent rays, FP32"
NODE_BYTES, TRI_BYTES, RAY_IN, HIT_OUT = 80, 48, 32, 16


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling around the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    from illuminaprt_b200 import replicas
    return replicas.rank_info()


def run_reference(args, world, rank):
    """The reference's own CPU path (compiled from its sources) on this host's cores."""
    if rank != 0:
        return
    from illuminaprt_b200 import scenes
    from oracle import bindings
    pos, idx, (co, cd), (io, idr) = scenes.ray_batch_workload()
    nthreads = os.cpu_count() or 1
    kind = "reference"
    try:
        ref = bindings.RefLib()
        mesh = ref.mesh(pos, idx, "bvh")
        build_s = mesh.build_seconds
        tracer = lambda o, d: mesh.intersect(o, d, nthreads)
        what = "reference BasicSpace->BVHMesh (Core/Space/BasicSpace.cpp:58-73, Core/Shape/BVHMesh.cpp:169-198)"
    except FileNotFoundError:
        kind = "port"
        bvh = bindings.Oracle().bvh(pos, idx)
        build_s = None
        tracer = lambda o, d: bvh.intersect(o, d, nthreads)
        what = "C restatement of the reference query (oracle/ilg_oracle.c)"
    # size the per-step sample so the whole run stays within a few minutes
    probe = 4096 * max(1, nthreads)
    t0 = time.perf_counter()
    tracer(co[:probe // 2], cd[:probe // 2])
    tracer(io[:probe // 2], idr[:probe // 2])
    rate = probe / max(time.perf_counter() - t0, 1e-6)
    per_step = int(min(co.shape[0], max(8192, rate * args.ref_seconds / max(1, args.steps + args.warmup)))) // 2 * 2
    rng = np.random.default_rng(11)
    half = per_step // 2
    for _ in range(args.warmup):
        pick = rng.choice(co.shape[0], half, replace=False)
        tracer(co[pick], cd[pick])
        tracer(io[pick], idr[pick])
    t_total = 0.0
    for _ in range(args.steps):
        pick = rng.choice(co.shape[0], half, replace=False)
        oc, dc, oi, di = co[pick], cd[pick], io[pick], idr[pick]
        t0 = time.perf_counter()
        tracer(oc, dc)
        tracer(oi, di)
        t_total += time.perf_counter() - t0
    value = per_step * args.steps / t_total / 1e6
    extra = {}
    if kind == "reference":
        box = scenes.box_scene()
        spp = 4
        t0 = time.perf_counter()
        ref.render_box(box, 256, 256, spp, seed=1, nthreads=nthreads)
        dt = time.perf_counter() - t0
        extra = {"pt_box_msamples_s": round(256 * 256 * spp / dt / 1e6, 4),
                 "pt_box_sample": f"256x256 at {spp} spp of the box scene through the reference's PathIntegrator"}
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_total / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_rays_per_step": per_step, **extra},
        "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": nthreads, "kind": kind,
                         "sample": f"{per_step} random rays per step (half coherent, half incoherent) of the "
                                   f"8,388,608-ray workload; {what}; tree build {build_s} s not timed"},
        "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(pos, idx, co, cd, io, idr, seconds=10.0, gpu_out=None):
    """The reference's CPU path on a bounded random sample (about `seconds` of
    work on all host cores), for the cpu_baseline key. With gpu_out (the
    device results of both ray sets), the sample's reference answers are
    also compared ray by ray with the device's: hit ids must agree except at
    near ties (two valid hits of the reference's test less than 1e-5 apart,
    which the reference decides by visit order), and agreeing hits must agree
    bit for bit in t, u and v."""
    from oracle import bindings
    nthreads = os.cpu_count() or 1
    try:
        mesh = bindings.RefLib().mesh(pos, idx, "bvh")
        kind, tracer = "reference", (lambda o, d: mesh.intersect(o, d, nthreads))
        what = "reference BasicSpace->BVHMesh (Core/Space/BasicSpace.cpp:58-73, Core/Shape/BVHMesh.cpp:169-198)"
    except FileNotFoundError:
        bvh = bindings.Oracle().bvh(pos, idx)
        kind, tracer = "port", (lambda o, d: bvh.intersect(o, d, nthreads))
        what = "oracle C restatement"
    rng = np.random.default_rng(11)
    probe = rng.choice(co.shape[0], 4096 * nthreads, replace=False)
    t0 = time.perf_counter()
    tracer(co[probe], cd[probe])
    tracer(io[probe], idr[probe])
    rate = 2 * len(probe) / max(time.perf_counter() - t0, 1e-6)
    half = int(min(co.shape[0], max(16384, rate * seconds / 2)))
    pick = rng.choice(co.shape[0], half, replace=False)
    oc, dc, oi, di = co[pick], cd[pick], io[pick], idr[pick]
    t0 = time.perf_counter()
    rc = tracer(oc, dc)
    ri = tracer(oi, di)
    dt = time.perf_counter() - t0
    res = {"value": round(2 * half / dt / 1e6, 4), "unit": UNIT, "cores": nthreads, "kind": kind,
           "sample": f"{half} random coherent + {half} random incoherent rays of the workload through the {what}, "
                     f"{dt:.1f} s on {nthreads} threads"}
    if gpu_out is not None:
        from tests.parity import classify_rates
        orc = bindings.Oracle()
        n_same = n_tie = n_rel = n_bad = 0
        bits = True
        for (o4, d4, ref), dev in ((oc, dc, rc), gpu_out["coherent"]), ((oi, di, ri), gpu_out["incoherent"]):
            got = tuple((x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x))[pick] for x in dev)
            r = classify_rates(pos, idx, o4, d4, got, ref, orc)
            n_same, n_tie, n_rel = n_same + r["same_id"], n_tie + r["near_ties"], n_rel + r["near_ties_relative"]
            n_bad, bits = n_bad + len(r["bad"]), bits and r["bits_ok"]
        n = 2 * half
        res["parity"] = {"rays": n, "same_id": n_same, "near_ties": n_tie, "other_mismatches": n_bad,
                         "near_tie_rate": round(n_tie / n, 9),
                         "near_ties_relative": n_rel, "near_tie_rate_relative": round(n_rel / n, 9),
                         "mismatch_rate_outside_relative_window": round((n - n_same - n_rel) / n, 9),
                         "tie_rules": "near_ties: both ids valid hits of the reference's test with |dt| < 1e-5 "
                                      "(its absolute window, IndexedTriangle.cpp:115); near_ties_relative: those "
                                      "with |dt| < 1e-5 * t",
                         "t_u_v_bit_equal_on_same_id": bits,
                         "note": "the reference's own KD-tree and BVH meshes disagree at near ties on this "
                                 "workload at 1.34e-5 (112 of 8,388,608 rays, measured once with both trees "
                                 "of the compiled reference): ties are decided by visit order"}
    return res


def bench_path_tracer(dev, local, legs=("box", "field", "mlp", "batch", "cache"), cache_budgets=(0.5, 2.0)):
    """Samples/s of the wavefront path tracer on the box scene (256^2, 16 spp,
    depth 6) and on the icosphere field (1920x1080, 64 spp, depth 12;
    64 spheres x 327,680 triangles + ground + 4 lights = 20,971,530 triangles)."""
    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace
    res = {}
    sp = GpuSpace(device=local)
    box = scenes.load_box_scene(sp)
    out = torch.empty((256, 256, 3), dtype=torch.float32, device=dev)
    st = torch.cuda.ExternalStream(sp.stream, device=dev)
    sp.render(box["camera"], 256, 256, 16, seed=1, out=out)
    sp.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    e0.record(st)
    for r in range(reps):
        sp.render(box["camera"], 256, 256, 16, seed=2 + r, out=out)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    res["pt_box_256x256x16spp_ms"] = round(ms, 3)
    res["pt_box_msamples_s"] = round(256 * 256 * 16 / (ms / 1e3) / 1e6, 3)
    # progressive display on the device: accumulate a 1080p frame and tone-map it
    frame = torch.rand((1080, 1920, 3), device=dev)
    avg, shown = torch.empty_like(frame), torch.empty_like(frame)
    sp.accumulate(frame, out=avg)
    sp.tonemap(avg, "drago", out=shown)
    sp.sync()
    e0.record(st)
    for _ in range(10):
        sp.accumulate(frame, out=avg)
        sp.tonemap(avg, "drago", out=shown)
    e1.record(st)
    e1.synchronize()
    pms = e0.elapsed_time(e1) / 10
    res["post_1080p_accumulate_drago_ms"] = round(pms, 4)
    # bytes: accumulate reads frame + sum, writes sum + out (48 B/px); Drago reads twice, writes once (36 B/px)
    res["post_1080p_gbs"] = round(1920 * 1080 * 84 / (pms / 1e3) / 1e9, 1)
    sp.close()
    if "field" in legs:
        bench_field(res, dev, local, e0, e1)
    if "mlp" in legs:
        bench_mlp(res, dev, local, e0, e1)
    if "batch" in legs:
        bench_batch(res, local)
    if "cache" in legs:
        bench_cache(res, local, budgets=cache_budgets)
    return res


def bench_cache(res, local, budgets=(0.5, 2.0)):
    """The radiance cache at equal wall time on the 1080p workload: the
    20,971,530-triangle icosphere field at 1920x1080, depth 12, against a
    16384-spp plain ground truth (64 renders of 256 spp averaged, untimed).
    At each budget, plain path tracing renders in calls that fill the
    wavefront (4 spp at 1080p, full throughput), and each cached arm renders
    1-spp frames trained on right after each one (the first 8 frames not
    averaged, their time counted): the network as the workload specifies it
    (12-band frequency encoding, 1 path in 16 traced to full depth as the
    training target, cache at the first or second bounce), this project's
    hash-grid network with 1-vertex self-training tails, and the non-learned
    hash-grid cache. Frames accumulate on the device in every arm."""
    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.cache_experiment import ARMS, gain_versus_budget
    from illuminaprt_b200.ilg import GpuSpace
    w, h = 1920, 1080
    field = scenes.sphere_field(8, 7, seed=3, width=w, height=h)
    sp = GpuSpace(device=local)
    scenes.load_sphere_field(sp, field)
    cam = dict(field["camera"], aspect=w / h)
    out = torch.empty((h, w, 3), dtype=torch.float32, device=f"cuda:{local}")
    acc = torch.zeros((h, w, 3), dtype=torch.float64, device=out.device)
    t0 = time.perf_counter()
    for k in range(64):
        sp.render(cam, w, h, 256, max_depth=12, seed=424242 + k, sky=field["sky"], out=out)
        acc.add_(out)
    sp.sync()
    gt = (acc / 64).cpu().numpy()
    gt_s = time.perf_counter() - t0
    del acc, out
    r = gain_versus_budget(sp, field, w, h, gt, budgets=budgets, arms=ARMS)
    r.update({"scene": "icosphere field 1920x1080, depth 12, ground truth 16384 spp",
              "ground_truth_seconds": round(gt_s, 1), "plain_spp_per_call": 4, "cached_spp_per_frame": 1,
              "cached_warmup_frames": 8, "accumulation": "device"})
    res["cache_equal_time_1080p"] = r
    sp.close()
    try:
        r["cpu_baseline"] = ic_cpu_baseline()
    except (FileNotFoundError, OSError, RuntimeError) as e:
        r["cpu_baseline"] = {"unavailable": str(e)[:200]}
    res["cache_matte_field"] = cache_matte_field(local)


def cache_matte_field(local, gpu_size=(960, 540), cpu_size=(240, 135), gpu_budgets=(0.25, 1.0), ic_spp=4):
    """The reference's irradiance cache and this project's learned caches on
    one scene the reference can render (scenes.matte_field: the icosphere
    field with every sphere Lambertian, 81,924 triangles, one quad light).
    On the device: plain path tracing against the hash-grid network with
    self-training tails and against the hash-grid cache, at equal wall time
    (gpu_budgets, 960x540, 16384-spp ground truth of this renderer). On the
    host (one thread: the reference's ICIntegrator shares one octree of
    records and is not thread-safe): the reference's ICIntegrator (factory
    defaults, ic_spp samples per pixel) against its PathIntegrator at equal
    CPU time (time of the integrators' Initialise to Commit, scene loading
    excluded), both through its BasicRenderer from a scene script, relMSE
    against this renderer's 16384-spp image at the same size."""
    import tempfile

    from illuminaprt_b200 import scenes
    from illuminaprt_b200.cache_experiment import ARMS, gain_versus_budget, rel_mse
    from illuminaprt_b200.ilg import GpuSpace
    gw, gh = gpu_size
    sc = scenes.matte_field(width=gw, height=gh)
    sp = GpuSpace(device=local)
    scenes.load_box_scene(sp, sc)
    cam = dict(sc["camera"], aspect=gw / gh)
    gt = sp.render(cam, gw, gh, 16384, max_depth=12, seed=424242)
    arms = {k: ARMS[k] for k in ("hashgrid_self_training", "hash_grid_cache")}
    out = {"scene": f"matte icosphere field ({sc['prim_of_tri'].size} triangles, one quad light)",
           "device": gain_versus_budget(sp, sc, gw, gh, gt, budgets=gpu_budgets, arms=arms)}
    out["device"]["size"] = f"{gw}x{gh}"
    cw, ch = cpu_size
    gt_small = sp.render(dict(sc["camera"], aspect=cw / ch), cw, ch, 16384, max_depth=12, seed=424243)
    sp.close()
    try:
        from oracle import bindings
        ref = bindings.RefLib()
        with tempfile.TemporaryDirectory() as tmp:
            def run(integrator, spp):
                script = scenes.write_box_script(os.path.join(tmp, f"{integrator}{spp}"), scene=sc, width=cw,
                                                 height=ch, spp=spp, space="Basic", renderer="Basic",
                                                 integrator=integrator)
                img, _, _, info = ref.render_script(script, cw, ch)
                return img, float(info.rsplit("render_s=", 1)[1])
            ic, t_ic = run("IC", ic_spp)
            _, t_pt1 = run("PathTracing", 1)
            pt_spp = max(1, int(round(t_ic / t_pt1)))
            pt, t_pt = run("PathTracing", pt_spp)
        e_ic, e_pt = rel_mse(ic, gt_small), rel_mse(pt, gt_small)
        out["reference_ic"] = {
            "kind": "reference", "cores": 1, "size": f"{cw}x{ch}", "gain": round(e_pt / e_ic, 3),
            "relmse_ic": round(e_ic, 5), "relmse_plain": round(e_pt, 5),
            "bias_ic": [round(b, 4) for b in (ic.mean((0, 1)) / gt_small.mean((0, 1)) - 1.0).tolist()],
            "bias_plain": [round(b, 4) for b in (pt.mean((0, 1)) / gt_small.mean((0, 1)) - 1.0).tolist()],
            "sample": f"ICIntegrator {ic_spp} spp in {t_ic:.2f} s vs PathIntegrator {pt_spp} spp in {t_pt:.2f} s, "
                      f"one thread, {cw}x{ch}"}
    except (FileNotFoundError, OSError, RuntimeError, ValueError, IndexError) as e:
        out["reference_ic"] = {"unavailable": str(e)[:200]}
    return out


def ic_cpu_baseline(width=64, ic_spp=16):
    """The reference's own caching method as the baseline of the cache leg:
    its irradiance-cache integrator (Core/Integrator/ICIntegrator.cpp, factory
    defaults) against its PathIntegrator at equal CPU time, both driven by
    its BasicRenderer over BasicSpace from a scene script (the box scene at
    64x64; error against the reference's 4096-spp image of the same scene).
    The reference renders on one thread."""
    import tempfile

    from illuminaprt_b200 import scenes
    from oracle import bindings
    from tests.test_scene_script import GOLDEN, coarse_expectation, rel_mse
    ref = bindings.RefLib()
    expected = coarse_expectation(np.load(GOLDEN)["image"], width)
    with tempfile.TemporaryDirectory() as tmp:
        def run(integrator, spp):
            script = scenes.write_box_script(os.path.join(tmp, f"{integrator}{spp}"), width=width, height=width,
                                             spp=spp, space="Basic", renderer="Basic", integrator=integrator)
            t0 = time.perf_counter()
            img = ref.render_script(script, width, width)[0]
            return img, time.perf_counter() - t0
        ic, t_ic = run("IC", ic_spp)
        _, t_pt4 = run("PathTracing", 4)
        pt_spp = max(1, int(round(4 * t_ic / t_pt4)))
        pt, t_pt = run("PathTracing", pt_spp)
    e_ic, e_pt = rel_mse(ic, expected), rel_mse(pt, expected)
    bias = (ic.mean((0, 1)) / expected.mean((0, 1)) - 1.0).tolist()
    return {"kind": "reference", "cores": 1, "gain": round(e_pt / e_ic, 3), "relmse_ic": round(e_ic, 5),
            "relmse_plain": round(e_pt, 5), "bias_ic": [round(b, 4) for b in bias],
            "sample": f"box scene {width}x{width}: ICIntegrator {ic_spp} spp in {t_ic:.2f} s vs PathIntegrator "
                      f"{pt_spp} spp in {t_pt:.2f} s, one thread"}


def pt_bytes_per_sample(counts, samples):
    """Algorithmic bytes per path sample from a counted render: every
    closest-hit ray reads its 32-byte ray, the node and triangle records its
    traversal visits (80 and 48 bytes) and moves ~64 bytes of path state
    (hit, throughput, next queue entry); every shadow ray reads its 48-byte
    segment and its records and adds a 16-byte contribution."""
    cr, cn, ct, sr, sn, st = counts
    total = cr * (32 + 64) + cn * NODE_BYTES + ct * TRI_BYTES + sr * (48 + 16) + sn * NODE_BYTES + st * TRI_BYTES
    return total / samples


def bench_field(res, dev, local, e0, e1):
    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace
    field = scenes.sphere_field(8, 7, seed=3)
    sp = GpuSpace(device=local)
    scenes.load_sphere_field(sp, field)
    W, H, spp = field["width"], field["height"], field["spp"]
    out = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    st = torch.cuda.ExternalStream(sp.stream, device=dev)
    sp.render(field["camera"], W, H, 1, max_depth=12, seed=1, sky=field["sky"], out=out)
    sp.sync()
    e0.record(st)
    sp.render(field["camera"], W, H, spp, max_depth=12, seed=2, sky=field["sky"], out=out)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    # traversal work of the same frame (a counted render, untimed) -> algorithmic bytes per sample
    sp.render(field["camera"], W, H, spp, max_depth=12, seed=2, sky=field["sky"], out=out, count=True)
    sp.sync()
    bps = pt_bytes_per_sample(sp.render_counts(), W * H * spp)
    hbm, _ = load_peaks()
    res["pt_field_alg_bytes_per_sample"] = round(bps, 1)
    res["pt_field_alg_gbs"] = round(bps * W * H * spp / (ms / 1e3) / 1e9, 1)
    res["pt_field_roofline_frac"] = round(res["pt_field_alg_gbs"] / hbm, 4)
    res["pt_field_triangles"] = int(field["idx"].shape[0])
    res["pt_field_bvh_build_ms"] = round(sp.stats()["build_ms"], 2)
    res["pt_field_1080p_64spp_ms"] = round(ms, 2)
    res["pt_field_msamples_s"] = round(W * H * spp / (ms / 1e3) / 1e6, 3)
    st_ = sp.stats()
    scene_mb = (st_["node_bytes"] + st_["tri_bytes"]) / 1e6
    res["pt_field_roofline"] = {
        "bound": "hbm", "achieved": res["pt_field_alg_gbs"], "peak": hbm, "unit": "GB/s",
        "frac": res["pt_field_roofline_frac"], "alg_bytes_per_sample": round(bps, 1),
        "note": f"scene {scene_mb:.0f} MB of node and triangle records exceeds L2: HBM level"}
    sp.close()
    res["pt_field_cpu_baseline"] = field_cpu_baseline(field)


def field_cpu_baseline(field, width=320, height=180, spp=16):
    """The field's CPU baseline: this project's C restatement of the path
    tracer (oracle/pt_oracle.c, the reference's PathIntegrator bounce loop
    with the GGX conductor and the sky added, over a binary BVH) on all host
    cores, on a bounded sample of the workload. The reference's own
    PathIntegrator cannot render this scene (it has no GGX conductor and its
    sky is inconsistent), so the baseline is the port."""
    from oracle.bindings import Oracle
    orc = Oracle()
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    orc.render(field["pos"], field["idx"], field["mat_ids"], field["materials"], field["lights"],
               dict(field["camera"], aspect=width / height), width, height, spp, max_depth=12, seed=3,
               sky=field["sky"], nthreads=nthreads)
    total = time.perf_counter() - t0
    dt = orc.last_render_seconds()
    return {"value": round(width * height * spp / max(dt, 1e-9) / 1e6, 4), "unit": "Msamples/s", "cores": nthreads,
            "kind": "port",
            "sample": f"{width}x{height} at {spp} spp of the field (depth 12) through oracle/pt_oracle.c on "
                      f"{nthreads} threads: {dt:.2f} s of paths; its tree build ({total - dt:.1f} s) not counted"}


def bench_mlp(res, dev, local, e0, e1):
    """Cache-network inference, 2,097,152 queries: the tcgen05 kernel and the
    mma.sync one, with the hash-grid encoding (grid gathers in k_grid_encode
    first) and with the frequency-only one (the network alone, its encoding
    computed in the kernel). 45,440 useful FLOP per query (2 x (96 x 64 +
    4 x 64 x 64 + 64 x 3)); the fraction is of the measured dense BF16 peak."""
    import torch
    from illuminaprt_b200.ilg import GpuSpace
    nq = 1 << 21
    q = torch.rand((nq, 16), device=dev)
    yq = torch.empty((nq, 3), device=dev)
    sp = GpuSpace(device=local)
    st = torch.cuda.ExternalStream(sp.stream, device=dev)
    peak = None
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            peak = float(json.load(f)["bf16_tflops"])
    for enc in ("hashgrid", "freq12"):
        sp.mlp_init(seed=1, encoding=enc)
        for flag, key in ((0, "tcgen05"), (0x10, "mma_sync")):
            sp.L.ilg_mlp_infer(sp.h, q.data_ptr(), nq, yq.data_ptr(), 0x1 | flag)
            sp.sync()
            e0.record(st)
            for _ in range(10):
                sp.L.ilg_mlp_infer(sp.h, q.data_ptr(), nq, yq.data_ptr(), 0x1 | flag)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / 10
            tag = key if enc == "hashgrid" else f"{key}_{enc}"
            res[f"mlp_infer_{tag}_mqueries_s"] = round(nq / (ms / 1e3) / 1e6, 1)
            res[f"mlp_infer_{tag}_tflops"] = round(nq * 45440 / (ms / 1e3) / 1e12, 2)
    # training step (forward, loss, backward, weight gradients) on 16384
    # rows: 3 x 45,440 FLOP per row
    nt = 16384
    tq = torch.rand((nt, 16), device=dev)
    tt = torch.rand((nt, 3), device=dev)
    g = torch.empty(23040, device=dev)
    loss = torch.empty(1, device=dev)
    for enc in ("hashgrid", "freq12"):
        sp.mlp_init(seed=1, encoding=enc)
        for flag, key in ((0, "tcgen05"), (0x10, "mma_sync")):
            sp.L.ilg_mlp_grads(sp.h, tq.data_ptr(), tt.data_ptr(), nt, g.data_ptr(), loss.data_ptr(), 0x1 | flag)
            sp.sync()
            e0.record(st)
            for _ in range(10):
                sp.L.ilg_mlp_grads(sp.h, tq.data_ptr(), tt.data_ptr(), nt, g.data_ptr(), loss.data_ptr(), 0x1 | flag)
            e1.record(st)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / 10
            res[f"mlp_train_{key}_{enc}_16384_rows_us"] = round(ms * 1e3, 1)
            res[f"mlp_train_{key}_{enc}_tflops"] = round(nt * 3 * 45440 / (ms / 1e3) / 1e12, 2)
    if peak:
        t = res["mlp_infer_tcgen05_freq12_tflops"]
        res["mlp_infer_roofline"] = {"bound": "tensor", "achieved": t, "peak": peak, "unit": "TFLOP/s",
                                     "frac": round(t / peak, 4), "kernel": "k_mlp_infer_tc (frequency encoding, "
                                     "network alone)", "peak_source": "measured bf16_tflops (burst)"}
    sp.close()


def bench_batch(res, local):
    """32 independent scenes of uneven size in one wavefront, autotuned."""
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace
    from illuminaprt_b200.autotune import tune_batch
    items = scenes.batch_workload(32, seed=9)
    spaces, batch = [], []
    for i, s in enumerate(items):
        sp_i = GpuSpace(device=local)
        scenes.load_sphere_field(sp_i, s)
        spaces.append(sp_i)
        batch.append({"space": sp_i, "camera": s["camera"], "width": s["width"], "height": s["height"],
                      "spp": s["spp"], "max_depth": s["max_depth"], "seed": 7 + i, "sky": s["sky"]})
    runner = GpuSpace(device=local)
    choice, sweep = tune_batch(runner, batch, waves=(1 << 21, 1 << 22, 1 << 23), blocks=(128, 256))
    kw = {k: choice[k] for k in ("paths_per_wave", "block", "one_launch")}
    runner.render_batch(batch, **kw)  # this setting's graph
    t0 = time.perf_counter()
    runner.render_batch(batch, **kw)
    dt = time.perf_counter() - t0
    best_wave = min((r for r in sweep if not r["one_launch"]), key=lambda r: r["seconds"])
    one = [r for r in sweep if r["one_launch"]]
    res["pt_batch32_schedules_msamples_s"] = {
        "wavefront_best": round(sum(b["width"] * b["height"] * b["spp"] for b in batch) / best_wave["seconds"] / 1e6, 3),
        "one_launch": round(sum(b["width"] * b["height"] * b["spp"] for b in batch) / one[0]["seconds"] / 1e6, 3)
        if one else None}
    samples = sum(b["width"] * b["height"] * b["spp"] for b in batch)
    res["pt_batch32_triangles"] = int(sum(s["idx"].shape[0] for s in items))
    res["pt_batch32_samples"] = int(samples)
    res["pt_batch32_ms"] = round(dt * 1e3, 2)
    res["pt_batch32_msamples_s"] = round(samples / dt / 1e6, 3)
    res["pt_batch32_autotuned"] = kw
    # traversal work of the same batch (a counted render, untimed) -> algorithmic bytes per sample
    runner.render_batch(batch, paths_per_wave=choice["paths_per_wave"] or (1 << 22), block=choice["block"], count=True)
    bps = pt_bytes_per_sample(runner.render_counts(), samples)
    hbm, _ = load_peaks()
    gbs = bps * samples / dt / 1e9
    res["pt_batch32_roofline"] = {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s",
                                  "frac": round(gbs / hbm, 4), "alg_bytes_per_sample": round(bps, 1),
                                  "note": "wall time of the whole batch call (host preparation included)"}
    for sp_i in spaces:
        sp_i.close()
    runner.close()
    return res


PROFILE_CASES = ("trace_heightfield", "mlp_infer_freq12", "mlp_infer_hashgrid", "mlp_train_hashgrid",
                 "mlp_train_freq12", "field_frame", "field_frame_one_launch", "cache_frames_1080p")


def profile_case(name):
    """Small fixed workloads for kernel profiles (one process, cuda:0):
    trace_heightfield: two coherent then two incoherent closest-hit launches
    on the 1 M-triangle heightfield; mlp_infer_*: three inference launches
    of 2,097,152 random queries; mlp_train_*: three training steps of
    16,384 random rows; field_frame(_one_launch): two 960x540 1-spp frames
    of the 20,971,530-triangle icosphere field (wavefront, or the one-launch
    renderer); cache_frames_1080p: eight 1920x1080 1-spp frames of that
    field with the radiance cache (hash-grid network, cache at the first
    bounce, 1-vertex self-training tails, two passes of 4 Adam steps of 16,384
    records: the equal-time comparison's best arm), then eight plain ones."""
    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace
    sp = GpuSpace(device=0)
    if name == "trace_heightfield":
        pos, idx, rays_c, rays_i = scenes.ray_batch_workload()
        sp.initialise(pos, idx)
        sp.build()
        for o, d in (rays_c, rays_i):
            O, D = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
            out = (torch.empty(O.shape[0], dtype=torch.int32, device="cuda"),
                   *(torch.empty(O.shape[0], device="cuda") for _ in range(3)))
            for _ in range(2):
                sp.intersects_into(O, D, *out, device_ptrs=True)
            sp.sync()
    elif name.startswith("mlp_infer_"):
        nq = 1 << 21
        q = torch.rand((nq, 16), device="cuda:0")
        y = torch.empty((nq, 3), device="cuda:0")
        sp.mlp_init(seed=1, encoding=name[len("mlp_infer_"):])
        for _ in range(3):
            sp._check(sp.L.ilg_mlp_infer(sp.h, q.data_ptr(), nq, y.data_ptr(), 0x1))
        sp.sync()
    elif name.startswith("mlp_train_"):
        n = 16384
        q = torch.rand((n, 16), device="cuda:0")
        t = torch.rand((n, 3), device="cuda:0")
        g = torch.empty(23040, device="cuda:0")
        loss = torch.empty(1, device="cuda:0")
        sp.mlp_init(seed=1, encoding=name[len("mlp_train_"):])
        for _ in range(3):
            sp._check(sp.L.ilg_mlp_grads(sp.h, q.data_ptr(), t.data_ptr(), n, g.data_ptr(), loss.data_ptr(), 0x1))
        sp.sync()
    elif name == "cache_frames_1080p":
        f = scenes.sphere_field(8, 7, seed=3)
        scenes.load_sphere_field(sp, f)
        cam = dict(f["camera"], aspect=1920 / 1080)
        sp.mlp_init(seed=1, lr=1e-2)
        for k in range(8):
            sp.render(cam, 1920, 1080, 1, max_depth=12, seed=k, sky=f["sky"], cache_depth=1, train_steps=4,
                      train_batch=16384, train_tail=1, train_epochs=2)
        for k in range(8):
            sp.render(cam, 1920, 1080, 1, max_depth=12, seed=k, sky=f["sky"])
        sp.sync()
    elif name.startswith("field_frame"):
        f = scenes.sphere_field(8, 7, seed=3)
        scenes.load_sphere_field(sp, f)
        cam = dict(f["camera"], aspect=960 / 540)
        for k in range(2):
            sp.render(cam, 960, 540, 1, max_depth=12, seed=1 + k, sky=f["sky"],
                      one_launch=name.endswith("one_launch"))
        sp.sync()
    sp.close()
    print(f"{name}: ok", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=PROFILE_CASES,
                    help="run one small profiling workload on cuda:0 and exit (no JSON line)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=120.0,
                    help="reference arm: seconds of CPU work over all steps (sizes each step's sample)")
    ap.add_argument("--no-path-tracer", action="store_true")
    ap.add_argument("--cache-budgets", default="0.5,2",
                    help="wall-time budgets (s) of the equal-time cache comparison")
    ap.add_argument("--legs", default="box,field,mlp,batch,cache",
                    help="extra measurements after the ray query: box,field,mlp,batch")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case)
        return
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    from illuminaprt_b200 import scenes
    from illuminaprt_b200.ilg import GpuSpace

    from illuminaprt_b200 import replicas
    torch.cuda.set_device(local)
    replicas.init("nccl")

    pos, idx, (co, cd), (io, idr) = scenes.ray_batch_workload()
    n_co, n_in = co.shape[0], io.shape[0]
    sp = GpuSpace(device=local)
    sp.initialise(pos, idx)
    sp.build()
    stats = sp.stats()
    stream = torch.cuda.ExternalStream(sp.stream, device=f"cuda:{local}")

    dev = f"cuda:{local}"
    rays = {"coherent": (torch.from_numpy(co).to(dev), torch.from_numpy(cd).to(dev)),
            "incoherent": (torch.from_numpy(io).to(dev), torch.from_numpy(idr).to(dev))}
    out = {k: (torch.empty(v[0].shape[0], dtype=torch.int32, device=dev),
               *(torch.empty(v[0].shape[0], dtype=torch.float32, device=dev) for _ in range(3)))
           for k, v in rays.items()}
    torch.cuda.synchronize()

    # one step = one call over the whole batch: the coherent rays, then the
    # incoherent ones, in one pair of arrays
    all_o = torch.cat([rays["coherent"][0], rays["incoherent"][0]])
    all_d = torch.cat([rays["coherent"][1], rays["incoherent"][1]])
    n_all = all_o.shape[0]
    all_out = (torch.empty(n_all, dtype=torch.int32, device=dev),
               *(torch.empty(n_all, dtype=torch.float32, device=dev) for _ in range(3)))

    def step():
        sp.intersects_into(all_o, all_d, *all_out, device_ptrs=True)

    # traversal counts for the algorithmic-bytes figure (untimed stats launch)
    visits = {}
    for k in ("coherent", "incoherent"):
        o, d = rays[k]
        visits[k] = sp.traversal_counts(o, d) if hasattr(sp, "traversal_counts") else None

    for _ in range(args.warmup):
        step()
    sp.sync()
    replicas.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for s in range(args.steps):
                step()
            ev[1].record(stream)
        sp.sync()
        torch.cuda.synchronize()
    clocks = clk.summary()
    total_ms = replicas.max_over_ranks(ev[0].elapsed_time(ev[1]), dev)
    rays_per_step = n_co + n_in
    value = replicas.aggregate_rate(rays_per_step * args.steps, world, total_ms / 1e3) / 1e6

    # each ray set alone, one launch each (untimed by the contract: the
    # coherent / incoherent rates and the incoherent launch's duration for the
    # roofline); its hits must equal the whole batch's
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for s in range(args.steps):
            o, d = rays["coherent"]
            sp.intersects_into(o, d, *out["coherent"], device_ptrs=True)
            ev[2 * s + 1].record(stream)
            o, d = rays["incoherent"]
            sp.intersects_into(o, d, *out["incoherent"], device_ptrs=True)
            ev[2 * s + 2].record(stream)
    sp.sync()
    torch.cuda.synchronize()
    t_co = sum(ev[2 * s].elapsed_time(ev[2 * s + 1]) for s in range(args.steps))
    t_in = sum(ev[2 * s + 1].elapsed_time(ev[2 * s + 2]) for s in range(args.steps))
    for a, b in zip(all_out, out["coherent"]):
        assert torch.equal(a[:n_co], b)
    for a, b in zip(all_out, out["incoherent"]):
        assert torch.equal(a[n_co:], b)

    # the same incoherent batch with the watertight triangle test (ILG_WATERTIGHT)
    o, d = rays["incoherent"]
    wt_out = [torch.empty_like(x) for x in out["incoherent"]]
    sp.intersects_into(o, d, *wt_out, device_ptrs=True, watertight=True)
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record(stream)
    for _ in range(args.steps):
        sp.intersects_into(o, d, *wt_out, device_ptrs=True, watertight=True)
    w1.record(stream)
    sp.sync()
    w1.synchronize()
    wt_mrays = n_in * args.steps / (w0.elapsed_time(w1) / 1e3) / 1e6
    wt_same = float((wt_out[0] == out["incoherent"][0]).float().mean().item())
    del wt_out

    # end to end through the public API: pinned host rays in, hits out
    pin = {k: (torch.from_numpy(v[0].cpu().numpy()).pin_memory(), torch.from_numpy(v[1].cpu().numpy()).pin_memory())
           for k, v in rays.items()}
    pin_all = (torch.cat([pin["coherent"][0], pin["incoherent"][0]]).pin_memory(),
               torch.cat([pin["coherent"][1], pin["incoherent"][1]]).pin_memory())
    hout_all = (torch.empty(n_all, dtype=torch.int32).pin_memory(),
                *(torch.empty(n_all, dtype=torch.float32).pin_memory() for _ in range(3)))
    e2e_steps = max(2, min(args.steps, 5))
    sp.intersects_into(*pin_all, *hout_all, device_ptrs=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    replicas.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        sp.intersects_into(*pin_all, *hout_all, device_ptrs=False)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1), dev)
    e2e_value = replicas.aggregate_rate(rays_per_step * e2e_steps, world, e2e_ms / 1e3) / 1e6
    # the e2e hits must equal the device-resident ones
    assert torch.equal(hout_all[0], all_out[0].cpu())
    # the same from pageable host memory (plain CPU tensors, as a host
    # application's own arrays are): the library stages them through its three
    # page-locked slots
    page = (pin_all[0].clone(), pin_all[1].clone())
    hpage = tuple(torch.empty_like(x, pin_memory=False) for x in hout_all)
    sp.intersects_into(*page, *hpage, device_ptrs=False)
    replicas.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        sp.intersects_into(*page, *hpage, device_ptrs=False)
    e1.record(stream)
    e1.synchronize()
    e2e_page_ms = replicas.max_over_ranks(e0.elapsed_time(e1), dev)
    e2e_page_value = replicas.aggregate_rate(rays_per_step * e2e_steps, world, e2e_page_ms / 1e3) / 1e6
    assert torch.equal(hpage[0], all_out[0].cpu())
    del page, hpage
    # the copy bound of e2e: a step's host->device bytes (rays) and
    # device->host bytes (hits) as plain pinned copies, each alone and both at
    # once on two streams (the link is full duplex; e2e overlaps the two)
    h2d_src = torch.cat([pin["coherent"][0], pin["coherent"][1], pin["incoherent"][0],
                         pin["incoherent"][1]]).pin_memory()
    h2d_dst = torch.empty_like(h2d_src, device=dev)
    d2h_src = torch.empty(rays_per_step * HIT_OUT // 4, dtype=torch.float32, device=dev)
    d2h_dst = torch.empty(d2h_src.shape, dtype=torch.float32, pin_memory=True)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def copies(h2d=True, d2h=True, reps=3):
        ev = []
        torch.cuda.synchronize(dev)
        for st_, on, (dst, src) in ((up, h2d, (h2d_dst, h2d_src)), (down, d2h, (d2h_dst, d2h_src))):
            if not on:
                continue
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(st_):
                dst.copy_(src, non_blocking=True)  # untimed first copy
                a.record(st_)
                for _ in range(reps):
                    dst.copy_(src, non_blocking=True)
                b.record(st_)
            ev.append((a, b))
        torch.cuda.synchronize(dev)
        return max(a.elapsed_time(b) for a, b in ev) / reps  # ms per step's bytes

    h2d_ms, d2h_ms, duplex_ms = copies(d2h=False), copies(h2d=False), copies()
    h2d_gbs = h2d_src.numel() * h2d_src.element_size() / (h2d_ms / 1e3) / 1e9
    d2h_gbs = d2h_src.numel() * d2h_src.element_size() / (d2h_ms / 1e3) / 1e9
    del h2d_src, h2d_dst, d2h_src, d2h_dst

    # the memory level that holds the traversal's working set: L2 when the
    # scene's node and triangle records fit in it, measured here by the
    # library's own streaming read probe (an L2-resident buffer read 64 times)
    l2_size = torch.cuda.get_device_properties(local).L2_cache_size
    scene_bytes = stats["node_bytes"] + stats["tri_bytes"]
    l2_probe = {f"{mb}MB": round(sp.probe_read_gbs(mb << 20, 64), 1) for mb in (32, 64, 96)}
    l2_gbs = max(l2_probe.values())
    hbm_read_gbs = round(sp.probe_read_gbs(2 << 30, 4), 1)

    # the path-tracing, network, batch and cache legs describe one GPU: a
    # multi-GPU run measures the ray query alone (its metric), so that it
    # holds the GPUs for the timed work only
    pt = {} if args.no_path_tracer or world > 1 else bench_path_tracer(
        dev, local, tuple(args.legs.split(",")), tuple(float(b) for b in args.cache_budgets.split(",")))
    hbm, peak_kind = load_peaks()
    # algorithmic bytes of one incoherent launch (the dominant kernel): rays in,
    # hits out, and every node / triangle record the traversal reads
    vin = visits["incoherent"]
    if vin is not None:
        alg_bytes = n_in * (RAY_IN + HIT_OUT) + vin[0] * NODE_BYTES + vin[1] * TRI_BYTES
    else:
        alg_bytes = n_in * (RAY_IN + HIT_OUT)
    launch_s = (t_in / args.steps) / 1e3
    achieved = alg_bytes / launch_s / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):  # DRAM bytes of one incoherent launch from the committed ncu capture
        with open(tp) as f:
            traffic = json.load(f).get("k_trace_dyn_incoherent_dram_bytes")
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rays_per_step": rays_per_step,
                       "calls_per_step": "one ilg_intersect over the whole batch (coherent rays first)",
                       "l2": "ray inputs 268 MB per step exceed the 126 MB L2; the BVH stays resident",
                       "parallelism": f"replicas x{world}",
                       "coherent_mrays_s": round(n_co * args.steps / (t_co / 1e3) / 1e6, 3),
                       "incoherent_mrays_s": round(n_in * args.steps / (t_in / 1e3) / 1e6, 3),
                       "incoherent_watertight_mrays_s": round(wt_mrays, 3),
                       "watertight_same_hit_fraction": round(wt_same, 6),
                       "bvh_nodes": stats["n_nodes"], "bvh_build_ms": round(stats["build_ms"], 3),
                       "scene_bytes": stats["node_bytes"] + stats["tri_bytes"], **pt},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": rays_per_step * RAY_IN,
                    "d2h_bytes_per_step": rays_per_step * HIT_OUT,
                    "pinned_h2d_gbs": round(h2d_gbs, 2),
                    "pinned_d2h_gbs": round(d2h_gbs, 2),
                    "copy_bound_mrays_s": round(rays_per_step / (max(h2d_ms, d2h_ms) / 1e3) / 1e6, 3),
                    "copy_bound": "a step's ray bytes up and hit bytes down as plain pinned copies, each alone, "
                                  "overlapped perfectly: the slower direction's time",
                    "duplex_copies_mrays_s": round(rays_per_step / (duplex_ms / 1e3) / 1e6, 3),
                    "e2e_pageable_mrays_s": round(e2e_page_value, 3),
                    "pipeline": "host-buffer calls run in chunks over three streams: upload, traversal and "
                                "download of neighbouring chunks overlap"},
            "gpu_launches": args.steps,
            "roofline": {"bound": "l2" if scene_bytes <= l2_size else "hbm", "achieved": round(achieved, 2),
                         "peak": l2_gbs if scene_bytes <= l2_size else hbm, "unit": "GB/s",
                         "frac": round(achieved / (l2_gbs if scene_bytes <= l2_size else hbm), 4),
                         "traffic": traffic,
                         "kernel": "k_trace_dyn<closest> (incoherent launch)",
                         "peak_source": (f"measured L2 read bandwidth (ilg_probe_read_gbs, L2-only loads, best of "
                                         f"32/64/96 MB buffers, this run): scene {scene_bytes / 1e6:.1f} MB <= L2 "
                                         f"{l2_size / 1e6:.1f} MB" if scene_bytes <= l2_size else
                                         f"{peak_kind} hbm_gbs (scene exceeds L2)"),
                         "l2_probe_gbs": l2_probe, "hbm_read_probe_gbs": hbm_read_gbs,
                         "hbm_peak": hbm, "hbm_peak_source": f"{peak_kind} hbm_gbs",
                         "frac_of_hbm": round(achieved / hbm, 4),
                         "compulsory_hbm_frac": round(
                             (n_in * (RAY_IN + HIT_OUT) + scene_bytes) / launch_s / 1e9 / hbm, 4),
                         "alg_bytes_per_launch": int(alg_bytes),
                         "node_visits_per_ray": None if vin is None else round(vin[0] / n_in, 3),
                         "tri_tests_per_ray": None if vin is None else round(vin[1] / n_in, 3)},
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline_sample(pos, idx, co, cd, io, idr, gpu_out=out)
        print(json.dumps(line), flush=True)
    sp.close()
    replicas.barrier()
    replicas.finish()


if __name__ == "__main__":
    main()
