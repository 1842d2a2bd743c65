"""The oracle (CPU) and the CUDA library (GPU) against the committed golden fixtures."""
import os

import numpy as np
import pytest

from tests.golden import make_golden

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["dam_break_64", "coupled_64"]


def _check(out, name):
    want = np.load(os.path.join(HERE, f"{name}.npz"))
    assert set(want.files) == set(out)
    for k in want.files:
        assert np.array_equal(out[k], want[k]), f"{name}: {k} differs from the fixture"


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(oracle_api, name):
    _check(make_golden.run(oracle_api, name), name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_matches_golden(gpu_api, name):
    _check(make_golden.run(gpu_api, name), name)
