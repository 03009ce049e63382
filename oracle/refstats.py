"""Statistics of many independent streak films, for parity at the configured film sizes.

TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_configured.py.

A film of the configured workloads is large (the Cornell workload: 128 x 128 pixels x 1024 bins
x RGB = 50 M bins), so K runs are never held at once: `Stats` accumulates per-bin sums and sums
of squares (the full-resolution mean and standard error) and, per run, the total energy, the
image-summed time curve and coarse (tile x time-window) sums, which are small enough to commit
as fixtures.  `reference_runs` renders K seeds with the reference's own renderer
(oracle/_ref/ref_render: its integrator, Embree ray casting and streak film), several processes
at once, and yields each film as it completes.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

from .pyoracle import REF_BIN


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class Stats:
    """Per-bin moments of K films [H][W][T][3] plus per-run energy, time curve [T][3] and
    coarse sums [H/tile][W/tile][T/window] (channels summed)."""

    def __init__(self, tile=8, window=16, full=True):
        self.tile, self.window, self.full = tile, window, full
        self.k = 0
        self.s1 = self.s2 = None
        self.energy, self.curve, self.coarse = [], [], []

    def coarse_of(self, f):
        H, W, T, _ = f.shape
        t, w = self.tile, self.window
        c = f.sum(axis=3)
        return c.reshape(H // t, t, W // t, t, T // w, w).sum(axis=(1, 3, 5))

    def add(self, film):
        f = np.asarray(film, np.float64)
        if self.full:
            if self.s1 is None:
                self.s1 = np.zeros_like(f)
                self.s2 = np.zeros_like(f)
            self.s1 += f
            self.s2 += f * f
        self.k += 1
        self.energy.append(f.sum())
        self.curve.append(f.sum(axis=(0, 1)))
        self.coarse.append(self.coarse_of(f))

    def mean_se(self):
        """Full-resolution per-bin mean and standard error of the mean."""
        k = self.k
        m = self.s1 / k
        var = np.maximum(self.s2 / k - m * m, 0.0) * k / (k - 1)
        return m, np.sqrt(var / k)

    def summary(self):
        """The committable part: per-run energy, curve and coarse sums."""
        return {"energy": np.array(self.energy), "curve": np.array(self.curve, np.float32),
                "coarse": np.array(self.coarse, np.float32), "k": self.k,
                "tile": self.tile, "window": self.window}


def reference_runs(scene, seeds, rows=None, procs=None):
    """Yields the reference renderer's streak film for each seed (scanlines rows = (y0, y1) only,
    when given), running up to `procs` processes at once."""
    from .refscene import write_scene
    procs = procs or host_cores()
    H = scene.height if rows is None else rows[1] - rows[0]
    shape = (H, scene.width, scene.time_bins, 3)
    n = int(np.prod(shape))
    with tempfile.TemporaryDirectory(prefix="tr_refstats_") as wd:
        pending = list(seeds)
        running = []
        while pending or running:
            while pending and len(running) < procs:
                s = pending.pop(0)
                sp = os.path.join(wd, f"scene{s}.txt")
                op = os.path.join(wd, f"film{s}.bin")
                write_scene(scene, sp, seed=s)
                cmd = [REF_BIN, sp, op] + ([str(rows[0]), str(rows[1])] if rows else [])
                running.append((s, sp, op, subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                                                            text=True)))
            s, sp, op, p = running.pop(0)
            _, err = p.communicate()
            if p.returncode != 0:
                raise RuntimeError(f"reference renderer failed (seed {s}): {err[-300:]}")
            json.loads(err.strip().splitlines()[-1])
            film = np.fromfile(op, np.float64, count=n).reshape(shape)
            os.remove(op)
            os.remove(sp)
            yield film


def zscores(m1, se1, m2, se2):
    """z of the difference of two independent means, over the cells with a nonzero error."""
    tot = np.sqrt(np.asarray(se1, np.float64) ** 2 + np.asarray(se2, np.float64) ** 2)
    ok = tot > 0
    z = (np.asarray(m1, np.float64) - np.asarray(m2, np.float64))[ok] / tot[ok]
    one_sided = int(((~ok) & ((np.asarray(m1) != 0) | (np.asarray(m2) != 0))).sum())
    return z, one_sided


def run_moments(a):
    """Mean and standard error over the first axis (the runs)."""
    a = np.asarray(a, np.float64)
    return a.mean(0), a.std(0, ddof=1) / np.sqrt(len(a))
