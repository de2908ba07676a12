"""CPU: the oracle's storage emulations against its FP64 run.

The field error of a 16-bit store grows with the store's unit roundoff
(every step rounds every stored value).  The oracle's "f16r8" emulation
(binary16 plus a residual byte per value: the byte cost of a compensated
store, which has no device form) must cut binary16's relative L2 error by
about the 2^8 its 8 extra significant bits give, on random spheres at 32^3
over 300 steps; bfloat16 (3 fewer bits than binary16) must be worse than
binary16.  These are emulations of storage formats, test infrastructure for
the error statement of the 16-bit forms.
"""
import numpy as np
import pytest

from oracle import oracle as O
from wavefront_b200 import configs


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def errors():
    sc = configs.random_spheres(32, steps=300)
    ref = O.sim_from_scenario(sc, dtype="f64")
    ref.step(sc.steps, 4)
    fr = ref.fields()
    ref.close()
    out = {}
    for st in ("f16", "bf16", "f16r8"):
        sim = O.sim_from_scenario(sc, storage=st)
        sim.step(sc.steps, 4)
        f = sim.fields().astype(np.float64)
        assert sim.storage_overflows == 0
        sim.close()
        out[st] = max(_rel(f[c], fr[c]) for c in range(6))
    return out


def test_residual_byte_cuts_the_binary16_error(errors):
    assert errors["f16r8"] < errors["f16"] / 64, errors
    assert errors["f16r8"] < 1e-3, errors


def test_bfloat16_is_coarser_than_binary16(errors):
    assert errors["bf16"] > 2 * errors["f16"], errors
