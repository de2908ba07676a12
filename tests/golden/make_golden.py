"""Copies the reference's own golden validation outputs into tests/golden/.

The reference (AndrejRumenovski/wavefront) commits the outputs of its two
validation studies as CSV files:
  validation/convergence_data.csv    <- examples/convergence_study.rs
  validation/pml_reflection_data.csv <- examples/pml_reflection_study.rs
The reference's example scene scenes/two_spheres.scene is copied too, as a
scene-format fixture.  They are data, not code, and they pin the oracle (oracle/wf_oracle.c) to the
reference's arithmetic: the oracle's restated studies must reproduce them.

Usage: python tests/golden/make_golden.py REF_ROOT
(or REF_ROOT in the environment), where REF_ROOT is a checkout of the
reference; there is no default location.
"""
import os
import shutil
import sys

REF_ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
if not REF_ROOT:
    sys.exit("usage: make_golden.py REF_ROOT (a checkout of the reference)")
HERE = os.path.dirname(os.path.abspath(__file__))

for sub, name in (("validation", "convergence_data.csv"),
                  ("validation", "pml_reflection_data.csv"),
                  ("scenes", "two_spheres.scene")):
    src = os.path.join(REF_ROOT, sub, name)
    if not os.path.exists(src):
        sys.exit(f"missing {src}")
    shutil.copyfile(src, os.path.join(HERE, name))
    print("copied", name)
