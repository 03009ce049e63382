"""Convergence of a progressive streak-film render towards a converged reference.

rel-L2 = ||F - F_ref||_2 / ||F_ref||_2 over every (y, x, t, rgb) bin, with both films
normalised by their samples per pixel. F_ref is a high-spp render of the plain tracer made of two
independent halves A and B, so its own noise can be taken out of the error:
E||F - F_ref||^2 = ||F - F_true||^2 + ||F_ref - F_true||^2, and ||F_ref - F_true||^2 is
estimated by ||A - B||^2 / 4. Films stay in device memory; the error of a pass costs one device
copy of the FP64 film and one reduction, which lie outside the timed render calls.

The comparison of samplers (``time_to_error``) times each ``Context.render`` call with the host
clock: that call returns after the pass is on the film and, with a learned proposal attached,
after the network has been trained on the previous pass's samples (that training runs beside
the pass's rendering, within the call), so training counts as render time.
"""
from __future__ import annotations

import math
import time
from typing import Optional

from . import renderer as R
from . import scenes as S


def _torch():
    import torch
    return torch


def film_device(ctx: R.Context, out=None):
    """The context's FP64 streak film [H, W, T, 3] copied into a torch CUDA tensor."""
    torch = _torch()
    sc = ctx.scene
    if out is None:
        out = torch.empty((sc.height, sc.width, sc.time_bins, 3), dtype=torch.float64,
                          device=f"cuda:{ctx.device}")
    # the library writes `out` on its own stream: torch's pending work on that memory first
    torch.cuda.current_stream(ctx.device).synchronize()
    R._abi.check(R._abi.lib().tr_get_film_device(ctx.h, R.C.c_void_p(out.data_ptr()), None, None))
    return out


class Reference:
    """Converged plain-tracer film: mean of two independent halves of ``spp`` samples each
    (sample indices [0, spp) and [spp, 2 spp) of every pixel), kept as float32 on the device."""

    def __init__(self, scene: S.Scene, spp: int, device: int = 0, chunk_spp: int = 256):
        torch = _torch()
        self.spp = 2 * spp
        halves = []
        buf = None
        with R.Context(scene, device) as ctx:
            for h in range(2):
                ctx.clear()
                done = 0
                while done < spp:
                    n = min(chunk_spp, spp - done)
                    ctx.render(h * spp + done, n)
                    done += n
                buf = film_device(ctx, buf)
                halves.append((buf / spp).to(torch.float32))
            del buf
        a, b = halves
        self.film = (a + b) * 0.5
        self.noise_sq = float(torch.sum(((a - b).double()) ** 2)) / 4.0
        self.norm_sq = float(torch.sum(self.film.double() ** 2))
        # relative error of the reference itself
        self.rel_noise = math.sqrt(self.noise_sq / self.norm_sq) if self.norm_sq > 0 else float("nan")
        del halves, a, b

    def rel_l2(self, film_fp64, spp: int, chunk: int = 1 << 26) -> float:
        """Bias-corrected rel-L2 of film_fp64 / spp (the FP64 device film of ``spp`` samples per
        pixel). Reduced in chunks so no full-size temporary is made."""
        torch = _torch()
        f = film_fp64.view(-1)
        r = self.film.view(-1)
        acc = torch.zeros((), dtype=torch.float64, device=f.device)
        inv = 1.0 / spp
        for i in range(0, f.numel(), chunk):
            d = f[i:i + chunk] * inv - r[i:i + chunk].double()
            acc += torch.dot(d, d)
        e2 = float(acc) - self.noise_sq
        return math.sqrt(max(e2, 0.0) / self.norm_sq)


def time_to_error(scene: S.Scene, ref: Reference, target: float = 0.05, pass_spp: int = 4,
                  max_spp: int = 4096, guide: Optional[R.Guide] = None, mix_prob: float = 0.5,
                  learning_rate: float = 1e-3, train_pool: int = 262144, device: int = 0,
                  sample_offset: int = 1 << 20, warmup_spp: int = 0, train_spp: Optional[int] = None,
                  warmup_pass_spp: Optional[int] = None):
    """Renders ``scene`` progressively, ``pass_spp`` samples per pixel per pass, until the film's
    rel-L2 against ``ref`` is at most ``target`` (or ``max_spp`` is reached). Sample indices start
    at ``sample_offset``, so the passes are independent of the reference's samples.

    With a learned proposal, the first ``warmup_spp`` samples per pixel train the network and are
    then dropped from the film (the film is cleared once), as in the iterative schemes of path
    guiding; their render and training time counts like every other pass.  They are rendered in
    passes of ``warmup_pass_spp`` (default ``pass_spp``): every pass fills the same training pool,
    so smaller warm-up passes give the network as many training steps for fewer rendered paths.  ``train_spp`` (when
    given) is the training budget: once the film holds that many samples per pixel the network is
    frozen and the remaining passes render with it without training.

    Returns {"seconds": render wall time to the target (None if not reached), "spp": samples per
    pixel in the film then, "warmup_spp", "paths_per_s", "curve": [(spp in film, seconds, rel_l2),
    ...], "train_steps", "train_loss"}."""
    torch = _torch()
    curve = []
    buf = None
    spent = 0.0
    reached = None
    train_steps = 0
    rendered = 0
    with R.Context(scene, device) as ctx:
        if guide is not None:
            ctx.set_guide(guide, mix_prob=mix_prob, learning_rate=learning_rate, train_pool=train_pool)
        else:
            warmup_spp = 0
        wpass = warmup_pass_spp or pass_spp
        while rendered < warmup_spp:
            n = min(wpass, warmup_spp - rendered)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            ctx.render(sample_offset + rendered, n)
            spent += time.perf_counter() - t0
            rendered += n
            train_steps += ctx.stats()["train_steps"]
        if warmup_spp:
            ctx.clear()
        spp = 0
        frozen = guide is None or train_spp is None
        while spp < max_spp:
            if not frozen and spp >= train_spp:
                ctx.set_guide(guide, mix_prob=mix_prob, learning_rate=learning_rate, train_pool=0)
                frozen = True
            n = min(pass_spp, max_spp - spp)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            ctx.render(sample_offset + rendered, n)
            spent += time.perf_counter() - t0
            spp += n
            rendered += n
            st = ctx.stats()
            train_steps += st["train_steps"]
            buf = film_device(ctx, buf)
            err = ref.rel_l2(buf, spp)
            curve.append((spp, spent, err))
            if err <= target:
                reached = (spent, spp)
                break
        train_loss = ctx.stats()["train_loss"]
    paths = rendered * scene.width * scene.height * scene.incoming_samples
    return {"seconds": reached[0] if reached else None, "spp": reached[1] if reached else None,
            "warmup_spp": warmup_spp, "warmup_pass_spp": (warmup_pass_spp or pass_spp) if warmup_spp else None,
            "train_spp": train_spp, "paths_per_s": paths / spent if spent > 0 else 0.0, "curve": curve,
            "train_steps": train_steps, "train_loss": train_loss}
