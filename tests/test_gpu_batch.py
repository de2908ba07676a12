"""GPU: batched stepping (wf_batch_*) of many independent grids of uneven
size by one persistent kernel per step.  Every grid must equal the oracle
bit for bit (fields, every psi array, probe sums), through runs long enough
to replay the captured 32-step graphs; the autotuner must leave the state
as it found it; lockstep violations are reported, not run."""
import os

import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import configs

pytestmark = pytest.mark.gpu
NT = min(os.cpu_count() or 1, 32)


def _eq(got, want, what):
    bad = got != want  # +0 == -0
    if bad.any():
        raise AssertionError(f"{what}: {bad.sum()} values differ, first {np.argwhere(bad)[:3].tolist()}")


def _check_against_oracle(oracle, b, scenes, steps):
    for i, sc in enumerate(scenes):
        sim = oracle.sim_from_scenario(sc, steps=steps)
        sim.step(steps, NT)
        g = b.grid(i)
        _eq(g.fields(), sim.fields(), f"scene {i} ({sc.dims.nx}^3) fields")
        for w in range(12):
            _eq(g.psi(w), sim.psi(w), f"scene {i} {wf.PSI_NAMES[w]}")
        gc, gs, gn = g.probe_sums(0, 1)
        oc, os_, on = sim.probe_sums(0, 1)
        assert gn == on and np.array_equal(gc, oc) and np.array_equal(gs, os_), i
        assert g.steps_done == steps
        sim.close()


def test_batch_matches_oracle_through_graph_replays(oracle):
    """9 scenes of 32..96 cells, 70 steps: two 32-step graph replays plus 6
    directly launched steps."""
    scenes = configs.batched_sweep(9, steps=70, seed=7, sizes=(32, 48, 64, 96))
    b = configs.device_batch(scenes)
    try:
        b.step(70)
        b.sync()
        # per step: one persistent launch per non-empty CPML class, then the tail
        per_step, rest = divmod(b.kernel_launches, 70)
        assert rest == 0 and 2 <= per_step <= 9, b.kernel_launches
        _check_against_oracle(oracle, b, scenes, 70)
    finally:
        b.close()


def test_narrow_batch_is_one_launch_per_step_and_matches_oracle(oracle):
    """The narrow tiling (tile_rows 32: every grid in 16-wide, 32-row tiles,
    all items in one persistent launch of the all-axes body): one step
    kernel plus the tail per step, bit for bit against the oracle, on grids
    whose x extent is not a multiple of the 16-cell tile (40, 56, 120)."""
    scenes = configs.batched_sweep(7, steps=70, seed=13, sizes=(32, 40, 56, 120))
    b = configs.device_batch(scenes)
    try:
        b.set_tiling(32, 16, 3)
        b.step(70)
        b.sync()
        assert b.kernel_launches == 2 * 70, b.kernel_launches
        _check_against_oracle(oracle, b, scenes, 70)
    finally:
        b.close()


@pytest.mark.parametrize("tiling", [(8, 16, 4), (4, 1000, 3), (16, 8, 3), (32, 1000, 3), (32, 7, 3)])
def test_batch_tilings_match_oracle(oracle, tiling):
    scenes = configs.batched_sweep(5, steps=40, seed=11, sizes=(32, 48, 64))
    b = configs.device_batch(scenes)
    try:
        b.set_tiling(*tiling)
        b.step(40)
        b.sync()
        _check_against_oracle(oracle, b, scenes, 40)
    finally:
        b.close()


def test_batch_autotune_restores_state(oracle):
    scenes = configs.batched_sweep(4, steps=35, seed=3, sizes=(32, 64))
    b = configs.device_batch(scenes)
    try:
        best, ms = b.autotune(2)
        assert best in [(ty, zc, s) for ty in (4, 8, 16) for s in (3, 4)
                        for zc in (8, 12, 16, 24, 32, 64, 128)] + [
                            (32, zc, 3) for zc in (8, 12, 16, 24, 32, 64, 128)]
        assert ms > 0
        b.step(35)
        b.sync()
        _check_against_oracle(oracle, b, scenes, 35)
    finally:
        b.close()


def test_batch_requires_lockstep():
    scenes = configs.batched_sweep(2, steps=10, seed=5, sizes=(32,))
    b = configs.device_batch(scenes)
    try:
        b.grid(0).step(1)  # one grid alone: the batch is out of lockstep
        with pytest.raises(wf.WfError, match="same steps"):
            b.step(1)
    finally:
        b.close()
