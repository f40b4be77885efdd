"""The GPU path against the committed golden fixtures (tests/golden/, made
by make_golden.py from the oracle): the same inputs stepped on the GPU give
the stored outputs bit for bit, without the oracle running."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


# fixture, shape (nx, ny, nz), form, svisc, steps, les_cs, fp16 scale, output key
CASES = [
    ("tgv_f64_5x7x9", (5, 7, 9), "fp64", 0.01, 10, 0.0, 0.0, "pops10"),
    ("hit_f16_8", (8, 8, 8), "fp16", 0.005, 5, 0.0, 2.0 ** 16, "pops5"),
    ("les_tgv_f64_6x5x4", (6, 5, 4), "fp64", 0.001, 6, 0.3, 0.0, "pops6"),
    ("les_f16_8", (8, 8, 8), "fp16", 1e-4, 5, 0.17, 2.0 ** 16, "pops5"),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("scheme", ["two_lattice", "aa"])
def test_gpu_reproduces_golden_fixture(bgk, case, scheme):
    name, shape, form, svisc, steps, les, scale, key = case
    ref = np.load(os.path.join(GOLDEN, name + ".npz"))
    box = bgk.BGK3D(*shape, svisc=svisc, precision=form, scheme=scheme, fp16_scale=scale, les_cs=les)
    box.set_populations(ref["pops0"])
    box.run(steps)
    assert _same(box.populations(), ref[key])
    box.close()
