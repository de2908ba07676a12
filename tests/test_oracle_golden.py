"""Pins the CPU oracle to the reference's own golden outputs.

The reference commits the results of its two validation studies
(validation/convergence_data.csv from examples/convergence_study.rs and
validation/pml_reflection_data.csv from examples/pml_reflection_study.rs).
Both studies are deterministic f32 arithmetic, so the oracle's restatement
must reproduce every printed value exactly: f32 columns are compared after
parsing the CSV text to f32, f64 columns to the last printed digit.
"""
import csv
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _rows(name):
    with open(os.path.join(GOLD, name)) as f:
        return list(csv.DictReader(f))


def test_convergence_study_matches_reference_csv_bit_for_bit(oracle):
    rows, mslope, tslope, maxd = oracle.convergence_study()
    gold = _rows("convergence_data.csv")
    cols = ["dx_m", "points_per_wavelength", "measured_phase_velocity",
            "theoretical_phase_velocity", "measured_relative_error",
            "theoretical_relative_error"]
    for r, g in zip(rows, gold):
        for c, name in enumerate(cols):
            assert np.float32(g[name]) == r[c], (name, g[name], r[c])
    # the study's own gates, examples/convergence_study.rs:340-349
    assert 1.5 <= mslope < 2.6
    assert maxd < 0.01
    # VALIDATION.md:110-115 quotes 2.16 / 2.03 / 3.05e-3
    assert abs(mslope - 2.162) < 5e-4 and abs(tslope - 2.025) < 5e-4
    assert abs(maxd - 3.05e-3) < 5e-6


def test_pml_reflection_study_matches_reference_csv(oracle):
    refl = oracle.pml_reflection_study()
    gold = _rows("pml_reflection_data.csv")
    for r, g in zip(refl, gold):
        # Rust prints the shortest repr that round-trips an f64, so parsing
        # it back must give the identical double.
        assert float(g["reflection_coeff"]) == r, (g, r)
    # gates, examples/pml_reflection_study.rs:351-374
    assert all(refl[i + 1] < refl[i] for i in range(3))
    assert refl[-1] < 1e-2
