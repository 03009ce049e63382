"""Hit records against the reference's own ray caster (World + vendored Embree 2.17.4).

The fixtures tests/golden/embree_hits_*.npz hold the reference's (triangle id, distance) for
every ray of the seeded correctness batches (tests/golden/make_embree_hits.py), encoded against
the CPU oracle's deterministic hits and sealed with a sha256 of the reference's arrays.  The
oracle's closest hits equal the GPU's bit for bit (tests/test_gpu_parity.py), so these tests pin
the GPU traversal to the reference over every ray:

* triangle ids: identical except ties - the ray meets both triangles within 2 ulp of distance
  (coplanar overlaps, shared edges); no other disagreement (`other` == 0) and no hit/miss
  disagreement;
* distances where the ids agree: within 2 ulp, except where the reference's Newton-refined
  reciprocal is itself up to 3 ulp from the exactly rounded quotient that this project computes
  (`rcp_rounding`; checked ray by ray against that reciprocal's error bound, `t_other` == 0).
"""
import os

import numpy as np
import pytest

from jarabotransientrendering_b200 import scenes as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BATCHES = {"icosphere7": lambda: S.icosphere(), "cornell": lambda: S.cornell()}


def load(name):
    fx = np.load(os.path.join(GOLDEN, f"embree_hits_{name}.npz"))
    return BATCHES[name](), S.random_rays(int(fx["rays"]), seed=int(fx["ray_seed"])), fx


def check_report(rep):
    assert rep["other"] == 0, rep
    assert rep["t_other"] == 0, rep
    assert rep.get("tie_t_ulp_max", 0) <= 2, rep
    assert len(rep["t_ulp_hist"]) <= 4, rep              # no same-id distance gap above 3 ulp
    gaps = np.array(rep["t_ulp_hist"])
    n_same_hit = gaps.sum()
    assert gaps[:3].sum() / n_same_hit > 0.9999, rep     # <= 2 ulp for all but the rcp cases
    assert rep["same_id"] / rep["rays"] > 0.99, rep


@pytest.mark.parametrize("name", list(BATCHES))
def test_oracle_hits_match_reference_embree(oracle_lib, name):
    from oracle import refhits
    sc, rays, fx = load(name)
    o = oracle_lib.Oracle(sc)
    ours = o.trace(rays)
    gid, t = refhits.decode(fx, ours)          # raises unless the records decode exactly
    rep = refhits.classify(o, sc.flatten()[1], rays, ours, gid, t)
    check_report(rep)
    # every tie is a genuine one: both triangles met within 2 ulp (checked in classify); the
    # icosphere batch's origins inside the boxes see box bottoms lying on the floor
    assert rep["ties_coplanar"] + rep["ties_edge"] == rep["rays"] - rep["same_id"]


@pytest.mark.parametrize("name", list(BATCHES))
def test_live_reference_reproduces_fixture(oracle_lib, name):
    """Where the reference's hit harness is built (oracle/_ref/ref_hits), rerun it and require
    the committed records bit for bit."""
    from oracle import refhits
    if not refhits.available():
        pytest.skip("oracle/_ref/ref_hits not built on this machine")
    sc, rays, fx = load(name)
    gid, t = refhits.run(sc, rays)
    assert refhits.digest(gid, t) == str(fx["sha256"])


def test_restated_moeller_is_embree_on_this_host(oracle_lib):
    """The oracle's restatement of Embree's Moeller test (orc_trace_moller, same operations and
    this host's reciprocal estimate) reproduces the live reference's distances bit for bit
    wherever both report the same triangle."""
    from oracle import refhits
    if not refhits.available():
        pytest.skip("oracle/_ref/ref_hits not built on this machine")
    sc = S.icosphere(subdiv=5)
    rays = S.random_rays(100000, seed=5)
    gid, t = refhits.run(sc, rays)
    hm = oracle_lib.Oracle(sc).trace_moller(rays)
    same = (hm["prim_id"] == gid) & (gid != refhits.MISS)
    assert same.mean() > 0.85
    assert (hm["t"][same].view(np.uint32) == t[same].view(np.uint32)).all()
