"""Small, self-contained render used for ncu captures of single kernels.

Renders `--spp` samples per pixel of a benchmark workload's geometry and camera at its full
resolution but with a short film (`--bins` time bins), so that the device footprint stays small
(the icosphere geometry at 512x512, 8 spp, 64 bins: one 2M-path batch, ~0.5 GB on the device)
while the traversal kernels see the real BVH and the real first-bounce ray distribution.

    python -m jarabotransientrendering_b200.profile_case --workload icosphere --spp 8 --bins 64
"""
import argparse

from . import scenes as S
from .renderer import Context


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="icosphere", choices=sorted(S.WORKLOADS))
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--bins", type=int, default=64)
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    sc = S.WORKLOADS[a.workload]()
    sc.exposure = sc.exposure * sc.time_bins / a.bins
    sc.time_bins = a.bins
    with Context(sc) as ctx:
        for r in range(a.repeat):
            ctx.render(r * a.spp, a.spp)
        st = ctx.stats()
    print({k: st[k] for k in ("paths", "closest_rays", "shadow_rays", "splats", "render_ms", "bvh_nodes", "bvh_depth")})


if __name__ == "__main__":
    main()
