"""Closest-hit records of the reference's own ray caster (vendored Embree 2.17.4 behind
World::add_triangle_mesh / first_intersection) and their comparison with this project's hits.

TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_embree_hits.py.

The reference casts every ray with rtcIntersect (src/RayTracing/World.h:570-585), whose
triangle test is Embree's non-watertight Moeller-Trumbore intersector
(src/External/Embree/kernels/geometry/triangle_intersector_moeller.h:66-104) with the distance
t = T * rcp(|den|), rcp = Newton-refined hardware reciprocal estimate
(common/simd/vfloat8_avx.h:242-254).  This project's traversal is watertight (Woop et al. 2013)
and divides exactly: t = RN(T / |den|) with Embree's own T and |den|.  So two kinds of
difference are expected and classified here:

* ties: the ray meets two triangles at distances within 2 ulp of each other (coplanar overlaps
  such as a box's bottom face lying on the floor, or a shared edge that one test counts and the
  other does not); Embree keeps whichever its BVH visits last among equals, this project the
  lower triangle id;
* reciprocal rounding: where both report the same triangle, Embree's t differs from the exactly
  rounded quotient by its own reciprocal error, at most (e0^2 + 3 * 2^-24) relative with
  e0 = 1.5 * 2^-12 (the estimate's documented accuracy) - up to 3 ulp.

Everything else counts as `other`, which the tests require to be zero.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import tempfile

import numpy as np

from .pyoracle import HERE

HITS_BIN = os.path.join(HERE, "_ref", "ref_hits")
MISS = 0xFFFFFFFF
RCP_REL_BOUND = (1.5 * 2.0 ** -12) ** 2 + 3 * 2.0 ** -24   # Embree's t vs the exact quotient
REC_DTYPE = np.dtype([("geom", "<u4"), ("prim", "<u4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])


def available():
    return os.path.exists(HITS_BIN)


def run(scene, rays):
    """Casts `rays` (float32 [N][8]) through the reference's World + Embree; returns
    (global triangle id uint32 with 0xFFFFFFFF for a miss, t float32)."""
    from .refscene import write_scene
    rays = np.ascontiguousarray(rays, np.float32)
    with tempfile.TemporaryDirectory(prefix="tr_hits_") as wd:
        sp, rp, op = (os.path.join(wd, f) for f in ("scene.txt", "rays.bin", "hits.bin"))
        write_scene(scene, sp)
        rays.tofile(rp)
        subprocess.run([HITS_BIN, sp, rp, op], check=True)
        rec = np.fromfile(op, REC_DTYPE)
    sizes = np.array([len(m.triangles) for m in scene.meshes], np.int64)
    first = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    hit = rec["geom"] != MISS
    gid = np.full(len(rec), MISS, np.uint32)
    gid[hit] = (first[rec["geom"][hit]] + rec["prim"][hit]).astype(np.uint32)
    return gid, rec["t"].copy()


def digest(gid, t):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(gid, "<u4").tobytes())
    h.update(np.ascontiguousarray(t, "<f4").tobytes())
    return h.hexdigest()


def encode(gid, t, ours):
    """Compact fixture of the reference's records relative to a deterministic hit array `ours`
    (oracle hits): the ulp offset of t where the ids agree, the full record where they do not,
    and the sha256 of the reference's arrays, so a decode against changed `ours` is detected."""
    same = gid == ours["prim_id"]
    d = t.view(np.int32).astype(np.int64) - ours["t"].view(np.int32).astype(np.int64)
    d[~same] = 0
    assert np.abs(d).max() < 127
    idx = np.nonzero(~same)[0].astype(np.int64)
    return dict(dulp=d.astype(np.int8), mis_idx=idx, mis_id=gid[idx], mis_t=t[idx], sha256=digest(gid, t))


def decode(fx, ours):
    """Rebuilds the reference's (gid, t) from a fixture and the same deterministic `ours`;
    raises if the rebuilt arrays do not hash to the recorded digest."""
    gid = ours["prim_id"].copy()
    t = (ours["t"].view(np.int32).astype(np.int64) + fx["dulp"].astype(np.int64)).astype(np.int32).view(np.float32)
    idx = fx["mis_idx"]
    gid[idx] = fx["mis_id"]
    t[idx] = fx["mis_t"]
    if digest(gid, t) != str(fx["sha256"]):
        raise ValueError("hit fixture does not decode to the recorded reference records")
    return gid, t


def _ulp_gap(a, b):
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))


def classify(oracle, triangles, rays, ours, gid, t, edge_ulps=64):
    """Compares this project's hits `ours` (dict-like with prim_id, t) with the reference's
    (gid, t) over every ray.  `triangles` is the scene's flattened [nt][3] vertex indices.

    An id disagreement is a tie when neither side misses, the two distances are within 2 ulp and
    either Embree's own test also accepts this project's triangle (coplanar overlap), or the two
    triangles share a vertex and this project's triangle fails Embree's test only by a
    barycentric within `edge_ulps` ulp(1) of the boundary (shared edge or vertex: the watertight
    test closes the crack that the Moeller test leaves).  Returns counts: same_id,
    ties_coplanar, ties_edge, other, the ulp histogram of t where the ids agree, and how many of
    those gaps exceed 2 ulp but lie within the reference's reciprocal bound (`rcp_rounding`) or
    outside it (`t_other`)."""
    rays = np.ascontiguousarray(rays, np.float32)
    a, ta = ours["prim_id"], ours["t"]
    same = a == gid
    out = {"rays": int(len(rays)), "same_id": int(same.sum()), "ties_coplanar": 0, "ties_edge": 0, "other": 0}
    # ---- id disagreements: both triangles met within 2 ulp of each other?
    dm = np.nonzero(~same)[0]
    if len(dm):
        one_miss = (a[dm] == MISS) | (gid[dm] == MISS)
        ours_terms = oracle.moller_terms(rays[dm], np.where(a[dm] == MISS, 0, a[dm]))
        tgap = _ulp_gap(ta[dm], t[dm])
        U, V, den = ours_terms["u"], ours_terms["v"], ours_terms["absden"]
        W = den - U - V
        inside = (U >= 0) & (V >= 0) & (W >= 0) & (den > 0)
        margin = np.minimum(np.minimum(U, V), W) / np.where(den > 0, den, 1)
        tri = np.asarray(triangles)
        ta_i, tb_i = tri[np.where(a[dm] == MISS, 0, a[dm])], tri[np.where(gid[dm] == MISS, 0, gid[dm])]
        shared = (ta_i[:, :, None] == tb_i[:, None, :]).any(axis=(1, 2))
        near_edge = shared & (den > 0) & (margin < 0) & (-margin <= edge_ulps * 2.0 ** -23)
        ok = ~one_miss & (tgap <= 2)
        out["ties_coplanar"] = int((ok & inside).sum())
        out["ties_edge"] = int((ok & ~inside & near_edge).sum())
        out["other"] = int((~(ok & (inside | near_edge))).sum())
        out["tie_t_ulp_max"] = int(tgap[ok].max()) if ok.any() else 0
    # ---- same triangle: distance gap
    both = same & (gid != MISS)
    gap = _ulp_gap(ta[both], t[both])
    out["t_ulp_hist"] = np.bincount(np.minimum(gap, 8)).tolist()
    big = np.nonzero(both)[0][gap > 2]
    out["rcp_rounding"] = out["t_other"] = 0
    if len(big):
        terms = oracle.moller_terms(rays[big], gid[big])
        q = terms["T"].astype(np.float64) / terms["absden"].astype(np.float64)
        emb_ok = np.abs(t[big].astype(np.float64) - q) <= RCP_REL_BOUND * q * (1 + 1e-9)
        ours_ok = np.abs(ta[big].astype(np.float64) - q) <= 0.5 * np.spacing(ta[big]).astype(np.float64)
        out["rcp_rounding"] = int((emb_ok & ours_ok).sum())
        out["t_other"] = int((~(emb_ok & ours_ok)).sum())
    return out
