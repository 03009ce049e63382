"""Context counters and per-kernel timing (tr_stats_get, tr_set_profiling)."""
import ctypes as C

import pytest

from jarabotransientrendering_b200 import _abi, scenes as S

pytestmark = pytest.mark.gpu


def test_profiled_sums_cover_every_render_past_the_event_limit(gpu):
    """tr_set_profiling(ctx, 2) reads its launch events out once 2^16 are pending; the kernel
    times of the renders before such a read-out must stay in the sums that tr_stats_get hands
    out, so the per-render mean over a long series equals that over a short one."""
    sc = S.cornell(width=16, height=16, time_bins=64, exposure=0.08, sqrt_spp=1, max_bounces=6)
    with gpu.Context(sc) as ctx:
        _abi.check(_abi.lib().tr_set_profiling(ctx.h, 2))
        ctx.render(0, 1)
        ctx.stats()                                    # drops the warm-up render's times
        n1 = 64
        for i in range(n1):
            ctx.render(1 + i, 1)
        a = ctx.stats()
        events_per_render = 2 * a["kernel_launches"]
        n2 = (1 << 16) // events_per_render * 2 + 17  # crosses the read-out limit at least once
        for i in range(n2):
            ctx.render(1 + n1 + i, 1)
        b = ctx.stats()
    for k in ("extend_ms", "shade_ms", "trace_ms"):
        per1, per2 = a[k] / n1, b[k] / n2
        assert per1 > 0 and 0.5 < per2 / per1 < 2.0, (k, per1, per2)
