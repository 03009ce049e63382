"""Small, self-contained render used for ncu captures of single kernels.

Renders `--spp` samples per pixel of a benchmark workload's geometry and camera at its full
resolution but with a short film (`--bins` time bins), so that the device footprint stays small
(the icosphere geometry at 512x512, 8 spp, 64 bins: one 2M-path batch, ~0.5 GB on the device)
while the traversal kernels see the real BVH and the real first-bounce ray distribution.

    python -m jarabotransientrendering_b200.profile_case --workload icosphere --spp 8 --bins 64

`--width`/`--height` override the film resolution (same camera, fewer pixels), so that a
film with the benchmark's full time-bin count and samples per pixel still fits a small
capture: 128x64 pixels at 256 spp and 2048 bins is one 2M-path batch with the benchmark's
per-batch shape (8192 pixels x 256 paths) and a 0.4 GB film.

`--guided` attaches a learned proposal (orthonormal shading frames, mixture probability
`--mix`); with `--train-pool 0` the network stays at its seeded initialisation, otherwise it is
trained after every pass.
"""
import argparse

from . import scenes as S
from .renderer import Context, Guide


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="icosphere", choices=sorted(S.WORKLOADS))
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--bins", type=int, default=64)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--guided", action="store_true")
    ap.add_argument("--mix", type=float, default=0.7)
    ap.add_argument("--train-pool", type=int, default=0)
    a = ap.parse_args()
    sc = S.WORKLOADS[a.workload]()
    sc.exposure = sc.exposure * sc.time_bins / a.bins
    sc.time_bins = a.bins
    if a.width:
        sc.width = a.width
    if a.height:
        sc.height = a.height
    guide = None
    if a.guided:
        sc.flags |= S.FLAG_ORTHONORMAL_FRAME
        guide = Guide(seed=1)
    with Context(sc) as ctx:
        if guide is not None:
            ctx.set_guide(guide, mix_prob=a.mix, learning_rate=3e-3, train_pool=a.train_pool)
        for r in range(a.repeat):
            ctx.render(r * a.spp, a.spp)
        st = ctx.stats()
    print({k: st[k] for k in ("paths", "closest_rays", "shadow_rays", "splats", "render_ms", "bvh_nodes", "bvh_depth",
                              "train_steps", "raygen_ms", "extend_ms", "shade_ms", "shadow_ms", "splat_ms")})
    if guide is not None:
        guide.close()


if __name__ == "__main__":
    main()
