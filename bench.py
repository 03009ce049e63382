"""Benchmark: transient path tracing throughput (paths/s) on one B200 per rank.

Workload (the configuration the headline metric is quoted on): the Cornell room with two boxes
plus a displaced icosphere at subdivision 7 (327,714 triangles), 512x512 pixels, 2048 time bins
of 0.0025, 256 samples per pixel, max depth 8 -- 67,108,864 camera paths per frame.  One step
renders one full frame (all 256 samples of every pixel) into the device FP64 streak film.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Multi-GPU (torchrun): every rank renders its own seeded replica
of the frame (weak scaling, no exchange); value = all paths / max-over-ranks device time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Canonical-BVH traffic per query for the icosphere workload, measured by the oracle on its own
# one-sample-per-pixel render rays (python oracle/measure_traffic.py icosphere):
# B = 48 B ray in/out + 64 B per two-child node visit + 48 B per triangle test.
B_CLOSEST = 48 + 64 * 19.397909840536915 + 48 * 8.579641797558255     # 1701.3 B
B_SHADOW = 48 + 64 * 16.98375084460311 + 48 * 6.767252594318216       # 1459.8 B
# DRAM bytes per closest-hit query of k_extend, from one ncu capture of all eight k_extend
# launches of the 2M-path icosphere case (same 2^21-slot batches as this workload):
# (425,001,984 B read + 36,808,704 B written) / 4,550,499 queries -- the BVH stays in L2, DRAM
# carries the ray records.  Scaled to this workload's mean launch for roofline.traffic.
DRAM_BYTES_PER_CLOSEST_QUERY = (425001984 + 36808704) / 4550499
# The same for k_shadow (all eight launches of the same case): (234,519,552 B read + 23,867,904 B
# written) / 3,177,936 any-hit queries.
DRAM_BYTES_PER_SHADOW_QUERY = (234519552 + 23867904) / 3177936

WORKLOAD = "icosphere"
# throughput (value, paths/s) plus the "convergence" object: time to 5% rel-L2, guided vs plain
METRIC = "paths/s; time to 5% rel-L2 streak-film error, guided vs plain, 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp-per-step", type=int, default=None, help="default: the workload's 256")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-convergence", action="store_true",
                    help="skip the time-to-5%%-rel-L2 comparison of guided and plain sampling")
    ap.add_argument("--convergence-ref-spp", type=int, default=131072,
                    help="samples per pixel of each of the two halves of the converged reference")
    ap.add_argument("--no-modes", action="store_true",
                    help="skip the sampling-mode throughputs (time sampling, light subpaths)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the 16-scene batched (CUDA-graph) throughput and accuracy leg")
    # --case: a small render of one workload for ncu captures of single kernels (no JSON line)
    ap.add_argument("--case", default=None, help="render a small case of this workload and exit")
    ap.add_argument("--case-spp", type=int, default=8)
    ap.add_argument("--case-bins", type=int, default=64)
    ap.add_argument("--case-repeat", type=int, default=1)
    ap.add_argument("--case-width", type=int, default=0)
    ap.add_argument("--case-height", type=int, default=0)
    ap.add_argument("--case-guided", action="store_true")
    ap.add_argument("--case-mix", type=float, default=0.7)
    ap.add_argument("--case-train-pool", type=int, default=0)
    return ap.parse_args()


def profile_case(a):
    """Small render for ncu captures: `--case-spp` samples per pixel of a workload's geometry and
    camera at its full resolution but with a short film (`--case-bins` time bins, exposure scaled
    to keep the film's time span), so that the device footprint stays small (the icosphere
    geometry at 512x512, 8 spp, 64 bins: one 2M-path batch, ~0.5 GB on the device) while the
    traversal kernels see the real BVH and the real first-bounce ray distribution.
    `--case-width`/`--case-height` override the resolution (same camera, fewer pixels): 128x64
    pixels at 256 spp and 2048 bins is one 2M-path batch with the benchmark's per-batch shape
    (8192 pixels x 256 paths) and a 0.4 GB film.  `--case-guided` attaches a learned proposal
    (orthonormal shading frames, mixture probability `--case-mix`); with `--case-train-pool 0`
    the network stays at its seeded initialisation, otherwise it trains after every pass."""
    from jarabotransientrendering_b200 import scenes as S
    from jarabotransientrendering_b200.renderer import Context, Guide
    sc = S.WORKLOADS[a.case]()
    sc.exposure = sc.exposure * sc.time_bins / a.case_bins
    sc.time_bins = a.case_bins
    if a.case_width:
        sc.width = a.case_width
    if a.case_height:
        sc.height = a.case_height
    guide = None
    if a.case_guided:
        sc.flags |= S.FLAG_ORTHONORMAL_FRAME
        guide = Guide(seed=1)
    with Context(sc) as ctx:
        if guide is not None:
            ctx.set_guide(guide, mix_prob=a.case_mix, learning_rate=3e-3, train_pool=a.case_train_pool)
        for r in range(a.case_repeat):
            ctx.render(r * a.case_spp, a.case_spp)
        st = ctx.stats()
    print({k: st[k] for k in ("paths", "closest_rays", "shadow_rays", "splats", "render_ms", "bvh_nodes", "bvh_depth",
                              "train_steps", "raygen_ms", "extend_ms", "shade_ms", "shadow_ms", "splat_ms")})
    if guide is not None:
        guide.close()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def _spread_rows(height, procs, per_proc):
    """Scanlines for `procs` processes x `per_proc` scanlines each, spread evenly over the
    image; process p's j-th scanline is sample j * procs + p (so every step's scanlines span the
    whole image).  Rows repeat only when more are asked for than the image has."""
    n = procs * per_proc
    return [[int(((j * procs + p) + 0.5) * height / n) % height for j in range(per_proc)] for p in range(procs)]


def cpu_reference(scene, procs, warmup, steps, binary=None, what="reference integrator and streak film, "
                  "rays cast by its vendored Embree 2.17.4"):
    """Times the reference renderer (oracle/_ref/ref_render: the reference's own World + Embree,
    integrator and streak film, built from its sources) on `procs` host processes at once.
    One step = every process renders one scanline (512 px x 256 spp, streak splat on; the
    scanlines of a step are spread over the image); the first `warmup` steps are untimed.
    Step time = the slowest process's render call for that step's scanline (scene parsing and
    the Embree build happen once per process, before the timed loop, as in the reference's own
    `Total time`).  Without the reference programs, the oracle port on all threads."""
    from oracle import refscene, pyoracle
    binary = binary or refscene.REF_BIN
    if not os.path.exists(binary):
        o = pyoracle.Oracle(scene)
        nthreads = os.cpu_count() or 1
        y0 = scene.height // 2
        t0 = time.perf_counter()
        r = o.render(sample_count=scene.spp, window=(0, y0, scene.width, y0 + steps), nthreads=nthreads,
                     streak=False)
        dt = time.perf_counter() - t0
        return {"value": r["stats"]["paths"] / dt, "unit": "paths/s", "cores": nthreads, "kind": "port",
                "ms_per_step": dt * 1e3 / steps,
                "sample": f"{steps} scanlines x {scene.width} px x {scene.spp} spp, oracle port"}
    wd = tempfile.mkdtemp(prefix="bk_bench_")
    sp = os.path.join(wd, "scene.txt")
    refscene.write_scene(scene, sp)
    rows = _spread_rows(scene.height, procs, warmup + steps)
    ps = []
    for i in range(procs):
        # --timing: each process adds all its scanlines into one film row (T x W x 3 doubles)
        ps.append(subprocess.Popen([binary, sp, os.path.join(wd, f"out{i}.bin"), "--rows", ",".join(map(str, rows[i])),
                                    "--timing"],
                                   stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True))
    per = []
    for p in ps:
        _, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference renderer failed: " + err[-400:])
        per.append(json.loads(err.strip().splitlines()[-1])["row_seconds"])
    for f in os.listdir(wd):
        os.remove(os.path.join(wd, f))
    os.rmdir(wd)
    paths_row = scene.width * scene.spp * scene.incoming_samples
    step_s = [max(r[warmup + k] for r in per) for k in range(steps)]
    secs = sum(step_s)
    paths = procs * paths_row * steps
    return {"value": paths / secs, "unit": "paths/s", "cores": procs, "kind": "reference",
            "ms_per_step": secs * 1e3 / steps,
            "sample": f"per step {procs} processes x 1 scanline x {scene.width} px x {scene.spp} spp "
                      f"({procs * paths_row} paths, scanlines spread over the image), {steps} timed steps after "
                      f"{warmup} untimed; {what}; step time = slowest process's render call"}


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest of a per-rank number over all ranks: the job takes as long as its slowest
    rank (every rank must call it, in the same order)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds):
    """Whole-job throughput: the units every rank processed over the slowest rank's time."""
    return units_per_rank * world / seconds


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


WORKLOAD_CONFIG = "icosphere subdiv 7 in Cornell box, 512x512, 2048 bins x 0.0025, 256 spp, depth 8"


def run_reference(args, rank, world):
    """The reference arm: the reference's own renderer (Embree backend, streak splat on) on all
    host cores; rank 0 alone runs it under torchrun."""
    from jarabotransientrendering_b200 import scenes as S
    if rank != 0:
        return
    sc = S.WORKLOADS[WORKLOAD]()
    procs = max(1, min(host_cores(), sc.height))
    cb = cpu_reference(sc, procs, args.warmup, args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "paths/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD_CONFIG, "triangles": sc.num_triangles,
                       "paths_per_step": sc.paths_per_frame(),
                       "film": "FP64 [512][512][2048][3] in HBM (12.9 GB)",
                       "l2": "film and path state larger than L2; 256 MiB write between steps",
                       "parallelism": f"replicas x{world}"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def convergence(args, device):
    """Time to 5% rel-L2 of the streak film, plain BSDF sampling vs the learned proposal, on the
    guided workload (GGX floor, 0.05 x 0.05 area light hidden behind an occluder slab, 512 x 512,
    2048 bins).  Reference: the plain tracer, two independent halves of ``convergence_ref_spp``
    samples per pixel (its own noise is subtracted from the error).  Both samplers render passes of
    64 samples per pixel from a fresh context and network; the guided run trains online (a pool of
    131,072 samples per pass in batches of 65,536, Adam lr 5e-3, mixture probability 0.7), first
    trains on 32 warm-up passes of 16 samples per pixel that it then drops, and stops training once
    the film holds 8,192 samples per pixel.  Time = host wall clock of the render calls (warm-up and
    training included); the error evaluation between passes is not timed."""
    import torch
    from jarabotransientrendering_b200 import convergence as CV, renderer as R, scenes as S
    sc = S.guided()
    sc.flags = S.FLAG_ORTHONORMAL_FRAME
    t0 = time.perf_counter()
    ref = CV.Reference(sc, args.convergence_ref_spp, device=device)
    ref_s = time.perf_counter() - t0
    plain = CV.time_to_error(sc, ref, target=0.05, pass_spp=64, max_spp=262144, device=device)
    g = R.Guide(device=device, seed=1)
    try:
        guided = CV.time_to_error(sc, ref, target=0.05, pass_spp=64, max_spp=262144, guide=g, mix_prob=0.7,
                                  learning_rate=5e-3, train_pool=131072, device=device, warmup_spp=512,
                                  warmup_pass_spp=16, train_spp=8192)
    finally:
        g.close()
    ref_noise = ref.rel_noise
    del ref
    torch.cuda.empty_cache()

    def leg(r):
        return {"seconds": r["seconds"], "spp": r["spp"], "warmup_spp": r["warmup_spp"],
                "warmup_pass_spp": r["warmup_pass_spp"], "train_spp": r["train_spp"],
                "paths_per_s": r["paths_per_s"], "train_steps": r["train_steps"],
                "rel_l2_at_stop": r["curve"][-1][2] if r["curve"] else None}
    res = {"metric": "seconds to 5% rel-L2 streak-film error (lower is better)", "unit": "s",
           "workload": "guided: Cornell box, GGX floor (alpha 0.2), 0.05x0.05 area light behind an occluder "
                       "slab, 512x512, 2048 bins x 0.0025, depth 8, orthonormal shading frames",
           "reference": {"tracer": "plain", "spp": 2 * args.convergence_ref_spp, "rel_noise": ref_noise,
                         "seconds": ref_s},
           "plain": leg(plain),
           "guided": dict(leg(guided), mix_prob=0.7, learning_rate=5e-3, train_pool=131072, train_batch=65536),
           "passes_spp": 64}
    if plain["seconds"] and guided["seconds"]:
        res["speedup_guided_vs_plain"] = plain["seconds"] / guided["seconds"]
    return res


def modes(args, device, reps=2):
    """Throughput of the sampling modes beside the plain path tracer, from the device time of
    tr_render (one warm-up render, then `reps` timed ones): time sampling in the medium workload
    (256x256, 4096 bins x 0.002, 128 spp x 2 incoming paths, depth 12, homogeneous medium) and,
    on the icosphere workload (327,714 triangles, 512x512, 2048 bins, depth 8, 32 spp), time
    sampling alone and with light subpaths + eye-light vertex connections."""
    import jarabotransientrendering_b200 as T
    from jarabotransientrendering_b200 import scenes as S
    cases = [("medium_plain", S.medium, 0, None),
             ("medium_time_sampling", S.medium, S.FLAG_TIME_SAMPLING, None),
             ("icosphere_plain", S.icosphere, 0, 32),
             ("icosphere_time_sampling", S.icosphere, S.FLAG_TIME_SAMPLING, 32),
             ("icosphere_bidirectional", S.icosphere, S.FLAG_TIME_SAMPLING | S.FLAG_BIDIRECTIONAL, 32)]
    out = {}
    for name, make, flags, spp in cases:
        sc = make()
        sc.flags |= flags
        spp = spp or sc.spp
        paths = sc.width * sc.height * spp * sc.incoming_samples
        with T.Context(sc, device=device) as c:
            T._abi.check(T._abi.lib().tr_set_profiling(c.h, 1))
            c.render(0, spp)
            ms, kern = 0.0, {"extend_ms": 0.0, "shade_ms": 0.0, "shadow_ms": 0.0, "splat_ms": 0.0}
            st0 = c.stats()
            for r in range(reps):
                c.render((r + 1) * spp, spp)
                st = c.stats()
                ms += st["render_ms"]
                for k in kern:
                    kern[k] += st[k] / reps
            st1 = c.stats()
        out[name] = {"paths_per_s": paths * reps / (ms / 1e3), "ms_per_render": ms / reps, "paths_per_render": paths,
                     "closest_rays_per_path": (st1["closest_rays"] - st0["closest_rays"]) / (paths * reps),
                     "shadow_rays_per_path": (st1["shadow_rays"] - st0["shadow_rays"]) / (paths * reps),
                     "kernel_ms_per_render": kern,
                     "scene": f"{sc.name} {sc.width}x{sc.height}, {sc.time_bins} bins, {spp} spp x "
                              f"{sc.incoming_samples}, depth {sc.max_bounces}, flags {sc.flags}"}
    out["note"] = ("shadow_ms includes the connection kernel (one any-hit ray per eye-light vertex pair, "
                   "counted in shadow_rays) in bidirectional mode")
    return out


def batched(args, device, frames=2):
    """16 seeded scenes of uneven size (scenes.batch_scenes) rendered together: every wavefront
    batch holds path slots of several scenes and is one replay of a captured CUDA graph; the
    batch's queue capacity, shade block and film tile width come from the autotuner; one learned
    proposal (scene index among its features) serves all scenes, trained online.  Reports the
    aggregate paths/s of a frame (every scene at its own spp) by host wall clock, training
    included, beside the same batch without the proposal and beside rendering the contexts one
    after another; per scene, the accuracy of the batched guided film against the plain tracer."""
    import torch
    from jarabotransientrendering_b200 import convergence as CV, renderer as R, scenes as S
    scs = S.batch_scenes()
    n = len(scs)
    spp = [sc.spp for sc in scs]
    paths_frame = sum(sc.paths_per_frame() for sc in scs)
    t0 = time.perf_counter()
    ctxs = [R.Context(sc, device) for sc in scs]
    create_s = time.perf_counter() - t0
    g = R.Guide(device=device, seed=1)
    res = {"workload": "16 seeded scenes: displaced icospheres (1,314-327,714 triangles) in Cornell rooms, "
                       "albedo 0.2-0.8, 64^2-512^2, 256-4096 bins, 32-256 spp, 8 with homogeneous media",
           "scenes": [{"triangles": sc.num_triangles, "res": sc.width, "bins": sc.time_bins,
                       "spp": sc.spp * sc.incoming_samples, "medium": sc.medium is not None} for sc in scs],
           "paths_per_frame": paths_frame, "create_s": create_s}
    try:
        B = R.Batch(ctxs)
        B.set_guide(g, mix_prob=0.7, learning_rate=3e-3, train_pool=262144)
        # trials of half a frame: a trial much smaller than the frame favours small queues (its
        # few batches overlap better across the lanes than a full frame's many)
        trial = [max(1, k // 2) for k in spp]
        best, trials = B.autotune(0, trial)
        res["autotune"] = {"best": best, "trials": trials, "trial_spp": trial}
        nxt = [trials * t for t in trial]

        def frame(b):
            nonlocal nxt
            torch.cuda.synchronize(device)
            t = time.perf_counter()
            b.render(nxt, spp)
            dt = time.perf_counter() - t
            nxt = [a + k for a, k in zip(nxt, spp)]
            return dt

        frame(B)                                  # warm-up frame (also trains the proposal)
        for c in ctxs:
            c.clear()
        begin_timed = list(nxt)
        wall = [frame(B) for _ in range(frames)]
        st = B.stats()
        res["guided"] = {"paths_per_s": paths_frame * frames / sum(wall), "ms_per_frame": 1e3 * sum(wall) / frames,
                         "device_ms_last_frame": st["render_ms"], "graph_kernel_launches_per_frame": st["kernel_launches"],
                         "train_steps_last_frame": st["train_steps"]}
        guided_films = []
        for c in ctxs:                            # keep the guided films (frames x spp per pixel)
            guided_films.append(CV.film_device(c).to(torch.float32))
            c.clear()
        B.set_guide(None)
        frame(B)
        wall = [frame(B) for _ in range(frames)]
        st = B.stats()
        res["plain_batched"] = {"paths_per_s": paths_frame * frames / sum(wall), "ms_per_frame": 1e3 * sum(wall) / frames,
                                "graph_kernel_launches_per_frame": st["kernel_launches"]}
        B.close()
        # one context after another (plain), same frame; one untimed render per context first
        # (its first own render allocates its wave buffers)
        for c, k, a in zip(ctxs, spp, nxt):
            c.render(a, k)
        for c in ctxs:
            c.clear()
        torch.cuda.synchronize(device)
        t = time.perf_counter()
        for c, k, a in zip(ctxs, spp, nxt):
            c.render(a, k)
        torch.cuda.synchronize(device)
        seq = time.perf_counter() - t
        nxt = [a + k for a, k in zip(nxt, spp)]
        res["plain_sequential"] = {"paths_per_s": paths_frame / seq, "ms_per_frame": 1e3 * seq}
        # accuracy per scene against the plain tracer: reference = plain, 4 x frames x spp
        # per pixel; beside it an independent plain film with as many samples as the guided one
        acc = []
        for i, c in enumerate(ctxs):
            c.clear()
            c.render(nxt[i], 4 * frames * spp[i])
            ref = CV.film_device(c).to(torch.float32) / (4 * frames * spp[i])
            c.clear()
            c.render(nxt[i] + 4 * frames * spp[i], frames * spp[i])
            pl = CV.film_device(c).to(torch.float32) / (frames * spp[i])
            gd = guided_films[i] / (frames * spp[i])
            nref = float(torch.linalg.vector_norm(ref.double()))
            acc.append({"energy_ratio_guided_vs_plain": float(gd.double().sum() / ref.double().sum()),
                        "rel_l2_guided": float(torch.linalg.vector_norm((gd - ref).double())) / nref,
                        "rel_l2_plain_same_spp": float(torch.linalg.vector_norm((pl - ref).double())) / nref})
            del ref, pl, gd
            guided_films[i] = None
            torch.cuda.empty_cache()
        res["accuracy_vs_plain"] = acc
        res["small_scenes"] = batched_small(device)
        res["speedup_batched_guided_vs_sequential_plain"] = res["guided"]["paths_per_s"] / res["plain_sequential"]["paths_per_s"]
        res["timed_sample_begin"] = begin_timed[:1]
    finally:
        g.close()
        for c in ctxs:
            c.close()
        torch.cuda.empty_cache()
    return res


def batched_small(device, scenes=64, frames=3):
    """Many small scenes (scenes.small_batch_scenes: 64 scenes of 64 x 64 pixels x 32 spp,
    131,072 paths each): plain rendering in shared CUDA-graph batches (autotuned) beside the
    same contexts rendered one after another, both by host wall clock around a frame."""
    import torch
    from jarabotransientrendering_b200 import renderer as R, scenes as S
    scs = S.small_batch_scenes(n=scenes)
    spp = [sc.spp for sc in scs]
    paths_frame = sum(sc.paths_per_frame() for sc in scs)
    ctxs = [R.Context(sc, device) for sc in scs]
    out = {"workload": f"{scenes} scenes of 64x64 pixels, 256 bins, 32 spp (16 x 2), 1,314-327,714 triangles",
           "paths_per_frame": paths_frame}
    try:
        # the batch renders at most 16 scenes: groups of 16 contexts, one batch object each
        groups = [ctxs[i:i + 16] for i in range(0, len(ctxs), 16)]
        batches = [R.Batch(g) for g in groups]
        nxt = 0
        for B, g in zip(batches, groups):
            B.autotune(0, [1] * len(g))
        def frame_batched():
            nonlocal nxt
            torch.cuda.synchronize(device)
            t = time.perf_counter()
            for B, g in zip(batches, groups):
                B.render([nxt] * len(g), [c.scene.spp for c in g])
            torch.cuda.synchronize(device)
            nxt += max(spp)
            return time.perf_counter() - t
        def frame_sequential():
            nonlocal nxt
            torch.cuda.synchronize(device)
            t = time.perf_counter()
            for c, k in zip(ctxs, spp):
                c.render(nxt, k)
            torch.cuda.synchronize(device)
            nxt += max(spp)
            return time.perf_counter() - t
        frame_batched()
        frame_sequential()
        tb = min(frame_batched() for _ in range(frames))
        ts = min(frame_sequential() for _ in range(frames))
        out["plain_batched"] = {"paths_per_s": paths_frame / tb, "ms_per_frame": tb * 1e3}
        out["plain_sequential"] = {"paths_per_s": paths_frame / ts, "ms_per_frame": ts * 1e3}
        out["speedup_batched_vs_sequential"] = ts / tb
        for B in batches:
            B.close()
    finally:
        for c in ctxs:
            c.close()
        torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.case:
        profile_case(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import jarabotransientrendering_b200 as T
    from jarabotransientrendering_b200 import scenes as S

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    sc = S.WORKLOADS[WORKLOAD](seed=1 + rank)
    spp = args.spp_per_step or sc.spp
    paths_per_step = sc.width * sc.height * spp * sc.incoming_samples

    ctx = T.Context(sc, device=local)
    stream = torch.cuda.Stream()
    T._abi.check(T._abi.lib().tr_set_stream(ctx.h, stream.cuda_stream))
    # per-kernel events around every launch of the timed renders, read out once after the timed
    # region (profiling 2: the read-out costs host time, not device time)
    T._abi.check(T._abi.lib().tr_set_profiling(ctx.h, 2))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.zero_()
        ctx.render(0, spp)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kern = {"extend_ms": 0.0, "shade_ms": 0.0, "shadow_ms": 0.0, "splat_ms": 0.0, "raygen_ms": 0.0, "trace_ms": 0.0}
    st0 = ctx.stats()                     # also drops the warm-up renders' pending times
    ev0.record(stream)
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        ctx.render(0, spp)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    st1 = ctx.stats()                     # per-kernel sums over the timed renders
    for k in kern:
        kern[k] = st1[k]
    # launches per render are the same in every step
    launches = st1["kernel_launches"] * args.steps
    ext_launches = st1["extend_launches"] * args.steps
    sh_launches = st1["shadow_launches"] * args.steps
    closest = st1["closest_rays"] - st0["closest_rays"]
    shadow = st1["shadow_rays"] - st0["shadow_rays"]
    ms = max_over_ranks(ms, dist, "cuda")
    value = whole_job_rate(paths_per_step * args.steps, world, ms / 1e3)

    # roofline of the dominant work: the BVH traversal, k_extend (closest hit) and k_shadow (any
    # hit).  The shadow launch of depth d runs on a second stream beside the closest-hit launch
    # of depth d + 1 (and two batches' launches beside each other), so their event times
    # overlap; the pair is timed as the union of their launch intervals (trace_ms) and counted
    # per extend + shadow launch pair.
    peak, peak_kind = peaks()
    algo = closest * B_CLOSEST + shadow * B_SHADOW
    achieved = algo / (kern["trace_ms"] / 1e3) / 1e9 if kern["trace_ms"] > 0 else None
    pairs = max(ext_launches, sh_launches)
    roofline = {"bound": "hbm", "kernel": "k_extend + k_shadow (closest-hit and any-hit BVH traversal, overlapped; "
                                          "timed as the union of their launch intervals)",
                "dominant_by_time": "trace_ms",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "peak_source": peak_kind,
                # the same algorithmic bytes over the whole timed step (shading, splat and gaps
                # included): (N_closest B_closest + N_shadow B_shadow) / wall time
                "achieved_over_step": algo / (ms / 1e3) / 1e9,
                "frac_over_step": algo / (ms / 1e3) / 1e9 / peak,
                "traffic": ((DRAM_BYTES_PER_CLOSEST_QUERY * closest + DRAM_BYTES_PER_SHADOW_QUERY * shadow) / pairs)
                if pairs else None,
                "traffic_unit": "bytes per extend + shadow launch pair (ncu DRAM read + write per query x queries)",
                "algorithmic_bytes_per_launch": (algo / pairs) if pairs else None,
                "algorithmic_bytes_per_query": {"closest": B_CLOSEST, "shadow": B_SHADOW},
                "kernel_ms_per_step": {k: v / args.steps for k, v in kern.items()},
                "queries_per_step": {"closest": closest / args.steps, "shadow": shadow / args.steps}}

    out = {"metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD_CONFIG,
                      "triangles": sc.num_triangles, "paths_per_step": paths_per_step,
                      "film": "FP64 [512][512][2048][3] in HBM (12.9 GB)",
                      "l2": "film and path state larger than L2; 256 MiB write between steps",
                      "parallelism": f"replicas x{world}"},
           "rays_per_s": (closest + shadow) * world / (ms / 1e3),
           "gpu_launches": launches, "clocks": clk, "roofline": roofline}

    if not args.no_e2e:
        # end to end through the C ABI with host buffers: scene upload + BVH build (tr_create),
        # render with the film streamed into pinned host memory as rows complete (tr_render_film:
        # RGBE images as the reference writes them; FP32 and FP64 sums beside), tr_destroy
        ctx.close()
        del flush
        torch.cuda.empty_cache()
        v, t_, m = sc.flatten()
        pv = torch.from_numpy(v).pin_memory().numpy()
        pt = torch.from_numpy(t_).pin_memory().numpy()
        pm = torch.from_numpy(m).pin_memory().numpy()
        H, W, Tb = sc.height, sc.width, sc.time_bins

        def host_film(dt):
            return (torch.empty((H, W, Tb, 3), dtype=dt, pin_memory=True).numpy(),
                    torch.empty((H, W, 3), dtype=dt, pin_memory=True).numpy(),
                    torch.empty((H, W), dtype=dt, pin_memory=True).numpy())

        def host_rgbe():
            return (torch.empty((H, W, Tb, 4), dtype=torch.uint8, pin_memory=True).numpy(),
                    torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True).numpy())

        def e2e_run(arrays, steps):
            """tr_create + tr_render_film (film rows streamed into the pinned arrays while the
            remaining rows render) + tr_destroy; the first iteration warms the allocator."""
            times, phases = [], []
            for i in range(steps + 1):
                t0 = time.perf_counter()
                c = T.Context(sc, device=local, arrays=(pv, pt, pm))
                t1 = time.perf_counter()
                c.render_film(0, spp, *arrays)
                t2 = time.perf_counter()
                bvh_ms = c.stats()["bvh_build_ms"]
                c.close()
                t3 = time.perf_counter()
                times.append(t3 - t0)
                phases.append({"create_ms": (t1 - t0) * 1e3, "bvh_build_ms": bvh_ms,
                               "render_and_film_d2h_ms": (t2 - t1) * 1e3, "destroy_ms": (t3 - t2) * 1e3})
            return sum(times[1:]) / steps, phases[1:]

        e2e_steps = max(1, min(args.steps, 3))
        rg = host_rgbe()
        et, ph = e2e_run(rg, e2e_steps)
        d2h = sum(a.nbytes for a in rg)
        del rg
        f32 = host_film(torch.float32)
        et32, ph32 = e2e_run(f32, 2)
        d2h32 = sum(a.nbytes for a in f32)
        del f32
        f64 = host_film(torch.float64)
        et64, ph64 = e2e_run(f64, 2)
        d2h64 = sum(a.nbytes for a in f64)
        del f64
        et = max_over_ranks(et, dist, "cuda")
        et32 = max_over_ranks(et32, dist, "cuda")
        et64 = max_over_ranks(et64, dist, "cuda")
        out["e2e"] = {"value": whole_job_rate(paths_per_step, world, et), "unit": "paths/s",
                      "h2d_bytes_per_step": int(pv.nbytes + pt.nbytes + pm.nbytes),
                      "d2h_bytes_per_step": int(d2h),
                      "ms_per_step": et * 1e3,
                      "film": "the reference's output images: every averaged film cell RGBE-encoded on the device "
                              "as its .hdr writer encodes it (the pixel data of the 512 per-scanline streak files "
                              "and of the steady image, byte for byte)",
                      "phases_per_step": ph,
                      "fp32_film": {"value": whole_job_rate(paths_per_step, world, et32), "d2h_bytes_per_step": int(d2h32),
                                    "ms_per_step": et32 * 1e3, "film": "FP32 sums and weights", "phases": ph32},
                      "fp64_film": {"value": whole_job_rate(paths_per_step, world, et64), "d2h_bytes_per_step": int(d2h64),
                                    "ms_per_step": et64 * 1e3, "film": "FP64 sums and weights", "phases": ph64},
                      "includes": "tr_create (scene H2D from pinned memory + device BVH build + film alloc), "
                                  "tr_render_film (render with the film streamed into pinned host memory as "
                                  "pixel rows complete), tr_destroy"}
    else:
        ctx.close()

    if rank == 0 and not args.no_cpu_baseline:
        procs = max(1, min(host_cores(), sc.height))
        out["cpu_baseline"] = cpu_reference(sc, procs, 1, 3)
        # the reference's own non-Embree triangle/BVH backend (src/Geometry), for comparison
        from oracle import refscene
        bvh = os.path.join(os.path.dirname(refscene.REF_BIN), "ref_render_bvh")
        if os.path.exists(bvh):
            nb = cpu_reference(sc, procs, 0, 1, binary=bvh, what="reference integrator and streak film, "
                               "rays cast by its own non-Embree BVH (src/Geometry)")
            out["cpu_baseline"]["non_embree_backend"] = {"value": nb["value"], "sample": nb["sample"]}
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            out["batched"] = batched(args, local)
        except Exception as e:            # reported, not fatal: the throughput line stands
            out["batched"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and not args.no_modes:
        try:
            out["modes"] = modes(args, local)
        except Exception as e:            # reported, not fatal: the throughput line stands
            out["modes"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and not args.no_convergence:
        try:
            out["convergence"] = convergence(args, local)
        except Exception as e:            # reported, not fatal: the throughput line stands
            out["convergence"] = {"error": f"{type(e).__name__}: {e}"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
