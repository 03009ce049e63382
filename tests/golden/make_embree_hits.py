"""Generate the hit-record fixtures tests/golden/embree_hits_*.npz from the reference itself.

Casts the seeded correctness batches (origins uniform in the room, directions uniform on the
sphere, tnear 1e-5, tfar inf: scenes.random_rays) through the reference's World and its
vendored Embree 2.17.4 (oracle/_ref/ref_hits, built by `make -C oracle ref` from the reference
sources) and stores the records compactly relative to the CPU oracle's deterministic hits:
the ulp offset of each distance where the triangle ids agree, the full record where they do
not, and the sha256 of the reference's arrays (oracle/refhits.py encode/decode).  Needs the
reference sources (only in the build container); the committed .npz files are what the tests
read.

    python tests/golden/make_embree_hits.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jarabotransientrendering_b200 import scenes as S  # noqa: E402
from oracle import pyoracle, refhits, refscene  # noqa: E402

RAY_SEED = 2


def batches():
    """name -> (scene, number of rays): the icosphere workload's 1,048,576-ray batch over the
    subdivision-7 displaced sphere in the Cornell box, and a Cornell-box batch."""
    return {"icosphere7": (S.icosphere(), 1 << 20), "cornell": (S.cornell(), 1 << 18)}


def main():
    if not refscene.build_ref():
        raise SystemExit("reference sources not available: cannot build oracle/_ref/ref_hits")
    for name, (sc, n) in batches().items():
        rays = S.random_rays(n, seed=RAY_SEED)
        gid, t = refhits.run(sc, rays)
        o = pyoracle.Oracle(sc)
        ours = o.trace(rays)
        fx = refhits.encode(gid, t, ours)
        rep = refhits.classify(o, sc.flatten()[1], rays, ours, gid, t)
        out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"embree_hits_{name}.npz")
        np.savez_compressed(out, rays=n, ray_seed=RAY_SEED, **fx)
        print(name, out, rep)


if __name__ == "__main__":
    main()
