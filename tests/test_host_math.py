"""Host-side setup math: the reference's own unit tests (src/layout.rs:793-897,
src/source.rs:103-156, src/probe.rs:188-260, src/scene.rs:238-286) run
against the library's C++ host code, plus bit-for-bit agreement of that host
code with the oracle's independent restatement."""
import math
import os

import numpy as np
import pytest

import wavefront_b200 as wf
from wavefront_b200 import configs

DT, DX = 1.5e-12, 1.0e-3


# ---- src/layout.rs tests ----------------------------------------------------

def test_fixed_point_round_trips():
    for v in [0.0, 1.0, -1.0, 0.5, -0.5, 123.456, -999.999, 3.0e-4]:
        q = wf.FixedQ16_16.from_f32(v)
        assert abs(wf.FixedQ16_16.to_f32(q) - np.float32(v)) < 2.0e-4 * max(abs(v), 1.0)


def test_vacuum_material_coeffs_match_closed_form():
    t = wf.MaterialTable.vacuum_filled(DT, DX)
    ca, cb, da, db = (wf.FixedQ16_16.to_f32(q) for q in t.get(0))
    assert abs(ca - 1.0) < 1e-4 and abs(da - 1.0) < 1e-4
    eps0, mu0 = np.float32(8.854188e-12), np.float32(1.2566371e-6)
    exp_cb = np.float32(DT) / (eps0 * np.float32(DX))
    exp_db = np.float32(DT) / (mu0 * np.float32(DX))
    assert abs(cb - exp_cb) < exp_cb * 5e-2
    assert abs(db - exp_db) < exp_db * 5e-2


def test_lossy_material_ca_is_between_zero_and_one():
    t = wf.MaterialTable.vacuum_filled(DT, DX)
    t.set_material(5, 2.0, 1.0, 0.02, DT, DX)
    ca = wf.FixedQ16_16.to_f32(t.get(5)[0])
    assert 0.0 < ca < 1.0


def test_pml_disabled_gives_identity_everywhere():
    p = wf.PmlProfile1D.build(64, wf.PmlConfig(), DT, DX, 0)
    assert np.all(p.b == 1.0) and np.all(p.a == 0.0) and np.all(p.inv_kappa == 1.0)


def test_pml_interior_is_identity_and_edges_are_graded():
    p = wf.PmlProfile1D.build(64, wf.PmlConfig(), DT, DX, 8)
    assert p.get(32) == (1.0, 0.0, 1.0)
    b, a, ik = p.get(0)
    assert ik < 1.0 and a != 0.0 and 0.0 < b < 1.0
    assert p.get(63) == p.get(0)


def test_effective_pml_thickness_clamps_to_grid_size():
    d = wf.GridDims(16, 16, 16)
    assert wf.effective_pml_thickness_blocks(d, 1000) == 1
    assert wf.effective_pml_thickness_blocks(d, 0) == 0
    assert wf.effective_pml_thickness_blocks(wf.GridDims(64, 64, 64), 10) == 2


def test_grid_dims_block_accounting():
    d = wf.GridDims(32, 16, 8)
    assert d.voxel_count() == 32 * 16 * 8
    assert d.block_dims() == (4, 2, 1)
    assert d.block_count() == 8
    with pytest.raises(ValueError):
        wf.GridDims(12, 16, 8)


# ---- src/source.rs tests ----------------------------------------------------

def test_ricker_wavelet_is_dc_free_over_a_full_period():
    w = wf.Waveform.ricker_wavelet(1.0, 2.0)
    n, span = 4000, 4.0
    dt = np.float32(span) / np.float32(n)
    total = np.float32(0.0)
    for i in range(n):
        total = np.float32(total + w.evaluate(float(np.float32(i) * dt)))
    assert abs(total * dt) < 0.05


def test_sinusoid_matches_a_sine_wave():
    w = wf.Waveform.sinusoid(1.0)
    assert abs(w.evaluate(0.0)) < 1e-6
    assert abs(w.evaluate(0.25) - 1.0) < 1e-5


def test_source_values_are_amplitude_times_waveform_at_step_times():
    s = wf.Source(8, 8, 8, wf.FieldComponent.Ez, 2.0, wf.Waveform.sinusoid(1.0e9))
    v = s.values(1e-12, 10)
    for i in range(10):
        t = np.float32(np.float32(i) + np.float32(1.0)) * np.float32(1e-12)
        assert v[i] == np.float32(2.0) * s.waveform.evaluate(float(t))


# ---- src/probe.rs tests (accumulation restated in f64 numpy) -----------------

def _accumulate(tables, values, first):
    c, s = tables
    sc = np.zeros(c.shape[1])
    ss = np.zeros(c.shape[1])
    n = 0
    for i, v in enumerate(values):
        if i >= first:
            sc += float(v) * c[i]
            ss += float(v) * s[i]
            n += 1
    return sc, ss, n


def test_dft_recovers_amplitude_and_phase_of_a_known_sinusoid():
    f, amp, ph, dt, steps = 1.0e9, 3.5, 0.7, 1.0e-12, 4000
    p = wf.Probe(8, 8, 8, wf.ProbeComponent.Ez, [f, 3 * f], 0.0)
    om = np.float32(2.0) * np.float32(np.pi) * np.float32(f)
    vals = [np.float32(amp) * np.float32(math.sin(float(om * np.float32((np.float32(i) + 1) * np.float32(dt))) + ph))
            for i in range(steps)]
    p.sum_cos, p.sum_sin, p.samples_recorded = _accumulate(p.tables(dt, steps), vals, p.first_step(dt))
    sp = p.spectrum()
    assert abs(sp[0].amplitude - amp) < 0.05 * amp
    err = (sp[0].phase_rad - ph + math.pi) % (2 * math.pi) - math.pi
    assert abs(err) < 0.05
    assert sp[1].amplitude < 0.05 * amp


def test_samples_before_start_recording_at_are_ignored():
    p = wf.Probe(0, 0, 0, wf.ProbeComponent.Ex, [1.0e9], 5.0e-9)
    # t = (s+1)*dt with dt = 1 ns: steps 0..3 (t <= 4 ns) are before the window
    assert p.first_step(1.0e-9) == 4
    p.sum_cos, p.sum_sin, p.samples_recorded = _accumulate(p.tables(1.0e-9, 4), [1e6] * 4, 4)
    assert p.spectrum()[0].amplitude == 0.0


# ---- src/scene.rs tests ------------------------------------------------------

def test_parses_comments_blank_lines_and_both_primitives():
    wf.Scene.parse("# a comment\n\nsphere 4.0 1.0 0.0 16 16 16 5\nbox 2.0 1.0 0.01 0 0 0 8 8 8\n")


def test_rejects_unknown_primitive():
    with pytest.raises(wf.SceneError, match="unknown primitive"):
        wf.Scene.parse("cone 1.0 1.0 0.0 0 0 0 1")


def test_rejects_wrong_argument_count():
    with pytest.raises(wf.SceneError, match="expected 'sphere"):
        wf.Scene.parse("sphere 1.0 2.0 3.0")


def test_deduplicates_identical_materials_into_one_id():
    d = wf.GridDims(32, 32, 32)
    g = wf.MaterialGrid(d)
    t = wf.MaterialTable.vacuum_filled(DT, DX)
    n = wf.Scene.parse("sphere 4.0 1.0 0.0 8 8 8 3\nsphere 4.0 1.0 0.0 24 24 24 3\n").voxelize(g, t, DT, DX)
    assert n == 1


# ---- product host code == oracle host code, bit for bit ---------------------

def test_material_coeffs_bit_identical_to_oracle(oracle):
    rng = np.random.default_rng(1)
    for _ in range(300):
        eps, mu = rng.uniform(1, 12), rng.uniform(1, 3)
        sig = rng.choice([0.0, rng.uniform(0, 0.1)])
        dt = float(np.float32(rng.uniform(0.5e-12, 2e-12)))
        assert np.array_equal(wf.material_coeffs(eps, mu, sig, dt, DX),
                              oracle.material_coeffs(eps, mu, sig, dt, DX))


@pytest.mark.parametrize("n,t", [(64, 16), (64, 8), (512, 16), (8, 8), (24, 8), (40, 10), (1080, 64)])
def test_pml_profile_bit_identical_to_oracle(oracle, n, t):
    p = wf.PmlProfile1D.build(n, wf.PmlConfig(), 1.9e-12, DX, t)
    b, a, k = oracle.pml_profile(n, 1.9e-12, DX, t)
    assert np.array_equal(p.b, b) and np.array_equal(p.a, a) and np.array_equal(p.inv_kappa, k)


def test_waveforms_and_tables_bit_identical_to_oracle(oracle):
    dt = configs.courant_dt(1e-3)
    f = float(np.float32(299792458.0 / 0.02))
    for w in [wf.default_waveform("ricker", f), wf.default_waveform("gaussian", f),
              wf.default_waveform("sinusoid", f)]:
        s = wf.Source(1, 1, 1, wf.FieldComponent.Ez, 1.0, w)
        assert np.array_equal(s.values(dt, 1000), oracle.source_values(w.kind, w.p0, w.p1, 1.0, dt, 1000))
    p = wf.Probe(0, 0, 0, wf.ProbeComponent.Ez, [f, 2 * f, 0.5 * f], 3e-11)
    c, s = p.tables(dt, 700)
    oc, os_ = oracle.probe_tables([f, 2 * f, 0.5 * f], dt, 700)
    assert np.array_equal(c, oc) and np.array_equal(s, os_)
    assert p.first_step(dt) == oracle.probe_first_step(3e-11, dt)
    for start in [0.0, 1e-12, 1.9e-12, 5e-9, 2.5e-10]:
        assert wf.Probe(0, 0, 0, 0, [1.0], start).first_step(dt) == oracle.probe_first_step(start, dt)


def test_scene_voxelizer_bit_identical_to_oracle(oracle):
    fixture = os.path.join(os.path.dirname(__file__), "golden", "two_spheres.scene")
    texts = [open(fixture).read(), configs.two_spheres_text(64),
             "box 2 1 0 -3.5 2.2 7.9 30.1 17 9\nsphere 3 1 0.01 10.5 11 12 6.3\nbox 2 1 0 4 4 4 4 9 9\n"]
    for text in texts:
        d = wf.GridDims(32, 32, 32) if "26" in text or "-3.5" in text else wf.GridDims(64, 64, 64)
        g = wf.MaterialGrid(d)
        t = wf.MaterialTable.vacuum_filled(DT, DX)
        n = wf.Scene.parse(text).voxelize(g, t, DT, DX)
        og, ot, on = oracle.scene_voxelize(text, d.nx, d.ny, d.nz, DT, DX)
        assert n == on and np.array_equal(g.ids, og) and np.array_equal(t.q16, ot)
    g = wf.MaterialGrid(wf.GridDims(64, 64, 64))
    wf.demo_sphere(g)
    assert np.array_equal(g.ids, oracle.demo_sphere(64, 64, 64))
