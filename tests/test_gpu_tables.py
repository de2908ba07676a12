"""GPU: sources and probes added between steps.

Adding a source or a probe marks the handle's source and probe descriptor
arrays stale; the library uploads them once, before the next step, and
drops the captured step graphs that held the old arrays.  A grid that gets
its second source and second probe after 40 steps (32-step graphs captured
before and after the additions) must equal, bit for bit, a grid that had
both from the start: the source's values zero before step 40, the probe
accumulating from step 40 (Probe::accumulate's start test,
src/probe.rs:127).  Fields, every probe's sums and counts are compared.
"""
import numpy as np
import pytest

from wavefront_b200 import configs
from wavefront_b200.probe import FieldComponent as PC
from wavefront_b200.probe import Probe
from wavefront_b200.source import FieldComponent, Source, default_waveform

pytestmark = pytest.mark.gpu

FIRST, REST = 40, 40


def _eq(got, want, what):
    bad = got != want  # +0 == -0
    assert not bad.any(), f"{what}: {int(bad.sum())} values differ"


@pytest.mark.parametrize("kernel", ["fused", "split"])
def test_sources_and_probes_added_between_steps(kernel):
    steps = FIRST + REST
    sc = configs.plain_cube_64(steps=steps)
    f0 = sc.meta["f0"]
    s2 = Source(20, 40, 28, FieldComponent.Ey, 0.5, default_waveform("gaussian", f0))
    p2 = Probe(44, 24, 36, PC.Hz, [f0, 0.5 * f0], 0.0)
    v2 = s2.values(sc.dt, steps)
    v2_late = v2.copy()
    v2_late[:FIRST] = 0.0
    c2, si2 = p2.tables(sc.dt, steps)

    def base(g):
        for s in sc.sources:
            g.add_source_values(s.x, s.y, s.z, s.component, s.values(sc.dt, steps), s.mode)
        for p in sc.probes:
            c, si = p.tables(sc.dt, steps)
            g.add_probe_tables(p.x, p.y, p.z, p.component, c, si, p.first_step(sc.dt))

    early = configs.device_grid(sc, kernel=kernel)
    late = configs.device_grid(sc, kernel=kernel)
    try:
        base(early)
        early.add_source_values(s2.x, s2.y, s2.z, s2.component, v2_late)
        early.add_probe_tables(p2.x, p2.y, p2.z, p2.component, c2, si2, FIRST)
        early.step(steps)

        base(late)
        late.step(FIRST)
        late.add_source_values(s2.x, s2.y, s2.z, s2.component, v2)
        late.add_probe_tables(p2.x, p2.y, p2.z, p2.component, c2, si2, FIRST)
        late.step(REST)

        early.sync()
        late.sync()
        want, got = early.fields(), late.fields()
        assert np.any(want != 0)
        _eq(got, want, "fields")
        for i, nf in ((0, len(sc.probes[0].frequencies_hz)), (1, 2)):
            wc, ws, wn = early.probe_sums(i, nf)
            gc, gs, gn = late.probe_sums(i, nf)
            assert gn == wn and (i == 0 or wn == REST), (i, gn, wn)
            _eq(gc, wc, f"probe {i} cos sums")
            _eq(gs, ws, f"probe {i} sin sums")
        assert np.any(wc != 0)
    finally:
        early.close()
        late.close()
