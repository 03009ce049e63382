"""Generate the golden fixtures of tests/golden/ from the reference renderer itself.

Runs oracle/_ref/ref_render (the reference's own integrator, sampler, camera, lights, media
and streak film, compiled from the reference sources by oracle/Makefile) on small seeded
scenes with K independent seeds and stores per-bin mean and standard error of the streak
film, plus per-seed total energy.  Needs the reference sources (only in the build
container); the committed .npz files are what the tests read.

    python tests/golden/make_golden.py [names]    # writes tests/golden/ref_*.npz

`unwarp`, `bounces` and `components` exercise the film options: the camera unwarp of
StreakCameraFilm, three per-bounce films of MultibounceStreakFilm (their per-bounce streaks are
stored as one film of 3H rows, their weights and the base steady image beside them) and the
depth / position / normal components of Film (per-pixel sums beside the streak).

`timesampling` (time sampling in a medium: the time-angular direction sampler) has a heavy-tailed
per-run energy, so its fixture holds per-run statistics of KR runs instead of per-bin moments:
the total energy and the energy in each window of 8 time bins.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jarabotransientrendering_b200 import scenes as S  # noqa: E402
from oracle import refscene  # noqa: E402

K = 96
KR = 512              # runs of the per-run (robust) fixtures
ROBUST = ("timesampling",)


def window_sums(streak, width=8):
    """Energy of a streak film [H][W][T][3] in consecutive windows of `width` time bins."""
    prof = streak.sum(axis=(0, 1, 3))
    return prof.reshape(-1, width).sum(1)


def _robust_run(args):
    name, seed = args
    r = refscene.render(golden_scenes()[name], seed=seed)
    return r["streak"].sum(), window_sums(r["streak"])


def golden_scenes():
    """Small variants of the benchmark workloads (light 0.2 below the ceiling so that the
    per-bin variance has no near-singular ceiling hot spot)."""
    c = S.cornell(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6)
    c.lights[0].position = (0.5, 0.8, 0.5)
    m = S.medium(width=12, height=12, time_bins=48, exposure=0.15, sqrt_spp=8, incoming_samples=1,
                 max_bounces=12)
    m.lights[0].position = (0.5, 0.8, 0.5)
    a = S.guided(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6,
                 lambertian_floor=True)
    a.lights = [S.rect_light((0.6, 0.8, 0.6), (0.6, 0.0, 0.6), (0.2, 0.2), 4.0)]
    u = S.cornell(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6)
    u.lights[0].position = (0.5, 0.8, 0.5)
    u.camera_unwarp = 1
    b = S.cornell(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6)
    b.lights[0].position = (0.5, 0.8, 0.5)
    b.bounce_films = 3
    k = S.medium(width=12, height=12, time_bins=48, exposure=0.15, sqrt_spp=8, incoming_samples=1,
                 max_bounces=12)
    k.lights[0].position = (0.5, 0.8, 0.5)
    k.components = S.COMP_DEPTH | S.COMP_POSITIONS | S.COMP_NORMALS
    ts = S.medium(width=12, height=12, time_bins=48, exposure=0.15, sqrt_spp=8, incoming_samples=1,
                  max_bounces=12)
    ts.lights[0].position = (0.5, 0.8, 0.5)
    ts.flags = S.FLAG_TIME_SAMPLING
    tc = S.cornell(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6)
    tc.lights[0].position = (0.5, 0.8, 0.5)
    tc.flags = S.FLAG_TIME_SAMPLING
    bd = S.cornell(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=6)
    bd.lights[0].position = (0.5, 0.8, 0.5)
    bd.flags = S.FLAG_TIME_SAMPLING | S.FLAG_BIDIRECTIONAL
    br = S.guided(width=12, height=12, time_bins=48, exposure=0.1, sqrt_spp=8, max_bounces=5,
                  lambertian_floor=True)
    br.lights = [S.rect_light((0.6, 0.8, 0.6), (0.6, 0.0, 0.6), (0.2, 0.2), 4.0)]
    br.flags = S.FLAG_TIME_SAMPLING | S.FLAG_BIDIRECTIONAL
    return {"cornell": c, "medium": m, "arealight": a, "unwarp": u, "bounces": b, "components": k,
            "timesampling": ts, "timesampling_surface": tc, "bidir": bd, "bidir_rect": br}


def main(names=None):
    if not refscene.build_ref():
        raise SystemExit("reference sources not available: cannot build oracle/_ref/ref_render")
    for name, sc in golden_scenes().items():
        if names and name not in names:
            continue
        if name in ROBUST:
            from multiprocessing import get_context
            with get_context("spawn").Pool(os.cpu_count() or 4) as pool:
                res = pool.map(_robust_run, [(name, s) for s in range(1, KR + 1)])
            energy = np.array([e for e, _ in res])
            windows = np.array([w for _, w in res])
            out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}.npz")
            np.savez_compressed(out, energy=energy, windows=windows, k=KR)
            print(name, out, "energy median %.4f mean %.4f" % (np.median(energy), energy.mean()))
            continue
        runs = [refscene.render(sc, seed=s) for s in range(1, K + 1)]
        films = np.array([r["streak"] for r in runs])
        if sc.bounce_films:
            nb, H = sc.bounce_films, sc.height
            films = np.array([r["bstreak"].reshape(nb * H, *r["bstreak"].shape[2:]) for r in runs])
        mean = films.mean(0)
        se = films.std(0, ddof=1) / np.sqrt(K)
        energy = films.sum(axis=(1, 2, 3, 4))
        extra = {}
        if sc.bounce_films:
            bw = np.array([r["bweight"] for r in runs])
            sd = np.array([r["steady"] for r in runs])
            extra = dict(bweight_mean=bw.mean(0), bweight_se=bw.std(0, ddof=1) / np.sqrt(K),
                         steady_mean=sd.mean(0), steady_se=sd.std(0, ddof=1) / np.sqrt(K))
        if sc.components:
            for key in ("depth", "positions", "normals"):
                arr = np.array([r[key] for r in runs])
                extra[key + "_mean"] = arr.mean(0)
                extra[key + "_se"] = arr.std(0, ddof=1) / np.sqrt(K)
        out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}.npz")
        np.savez_compressed(out, mean=mean.astype(np.float32), se=se.astype(np.float32), energy=energy, k=K, **extra)
        print(name, out, "energy %.4f +- %.4f" % (energy.mean(), energy.std(ddof=1) / np.sqrt(K)))


if __name__ == "__main__":
    main(sys.argv[1:])
