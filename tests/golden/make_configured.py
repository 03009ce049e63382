"""Generate tests/golden/ref_config_*.npz: reference statistics of the configured workloads.

Renders the workloads exactly as configured with the reference's own renderer
(oracle/_ref/ref_render: its integrator, sampler, camera, light, medium and streak film, rays
cast by its vendored Embree) over K independent seeds and stores, per workload, the per-run
total energy, and the mean and standard error of the image-summed time curve [T][3] and of
coarse sums (8 x 8-pixel tiles x 16-bin windows, channels summed).  Full-resolution per-bin
statistics are too large to commit; the GPU test recomputes those live from oracle/_ref where
it is built (tests/test_gpu_configured_parity.py).

  cornell: 128 x 128 pixels, 1024 bins x 0.005, point light 0.01 below the ceiling, depth 6,
           64 spp, all Lambertian, no medium (the full film);
  medium:  the same room filled with a homogeneous medium (sigma_a 0.05, sigma_s 0.5, HG g 0.3),
           256 x 256 pixels, 4096 bins x 0.002, depth 12, 8 x 8 camera samples x 2 incoming
           paths = 128 spp; scanlines 112-143 (32 rows through the middle of the image).

Needs the reference sources (only in the build container).

    python tests/golden/make_configured.py [names]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from jarabotransientrendering_b200 import scenes as S  # noqa: E402
from oracle import refscene, refstats  # noqa: E402

# name -> (scene factory, scanline rows or None, reference runs)
CONFIGS = {"cornell": (S.cornell, None, 512), "medium": (S.medium, (112, 144), 256),
           "icosphere": (S.icosphere, (252, 260), 1024)}


def main(names=None):
    if not refscene.build_ref():
        raise SystemExit("reference sources not available: cannot build oracle/_ref/ref_render")
    for name, (make, rows, K) in CONFIGS.items():
        if names and name not in names:
            continue
        sc = make()
        st = refstats.Stats(full=False)
        for f in refstats.reference_runs(sc, range(1, K + 1), rows=rows):
            st.add(f)
        cm, cs = refstats.run_moments(st.curve)
        gm, gs = refstats.run_moments(st.coarse)
        out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_config_{name}.npz")
        np.savez_compressed(out, k=K, energy=np.array(st.energy), curve_mean=cm.astype(np.float32),
                            curve_se=cs.astype(np.float32), coarse_mean=gm.astype(np.float32),
                            coarse_se=gs.astype(np.float32), tile=st.tile, window=st.window,
                            rows=np.array(rows if rows else (0, sc.height)))
        e = np.array(st.energy)
        print(name, out, "energy %.2f +- %.2f (rel se %.5f)" % (e.mean(), e.std(ddof=1) / np.sqrt(K),
                                                                e.std(ddof=1) / np.sqrt(K) / e.mean()))


if __name__ == "__main__":
    main(sys.argv[1:])
