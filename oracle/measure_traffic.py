"""Algorithmic traffic model of the traversal kernels, measured on the canonical BVH.

TEST / MEASUREMENT INFRASTRUCTURE.  Renders one sample per pixel of a workload with the CPU
oracle and reports the mean interior-node visits (N_node) and triangle tests (N_tri) per
closest-hit and per shadow query on the canonical binary SAH BVH (16 bins, <= 4 triangles
per leaf).  Bytes per query: B = 48 (ray in 32 + hit out 16) + 64 * N_node + 48 * N_tri.

    python oracle/measure_traffic.py icosphere
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from jarabotransientrendering_b200 import scenes as S  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402


def measure(name, nthreads=8):
    sc = S.WORKLOADS[name]()
    o = Oracle(sc)
    r = o.render(sample_count=1, nthreads=nthreads, streak=False)["stats"]
    out = {"workload": name, "paths": r["paths"], "closest_rays": r["closest_rays"], "shadow_rays": r["shadow_rays"],
           "N_node_closest": r["closest_nodes"] / r["closest_rays"], "N_tri_closest": r["closest_tris"] / r["closest_rays"],
           "N_node_shadow": r["shadow_nodes"] / max(1, r["shadow_rays"]),
           "N_tri_shadow": r["shadow_tris"] / max(1, r["shadow_rays"])}
    out["B_closest"] = 48 + 64 * out["N_node_closest"] + 48 * out["N_tri_closest"]
    out["B_shadow"] = 48 + 64 * out["N_node_shadow"] + 48 * out["N_tri_shadow"]
    out["bvh"] = o.bvh_info()
    return out


if __name__ == "__main__":
    for n in sys.argv[1:] or ["cornell", "icosphere", "medium"]:
        print(json.dumps(measure(n)))
