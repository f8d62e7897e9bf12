"""Size-independent properties at the benchmark's full size (65,536 histories
of the 50 MeV Si scene, 16 tiles, 238 reflections, 2048 bins).

Histories are keyed by index (Philox), so the same histories split into two
batches must give the same tallies exactly and the same spectra to the float
rounding of per-pass partial sums; every history ends in exactly one fate;
and the tile-summed mixed-precision spectrum agrees with FP64 statistically.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 65536


def _run(spec, precision, splits, cuda_device):
    from pyrite_b200.pipeline import ScoringCase

    case = ScoringCase(spec, precision=precision, batch_histories=H // splits, device=cuda_device)
    for k in range(splits):
        case.run_batch(k * (H // splits), H // splits)
    assert case.device_status() == 0
    return case.results()


def test_batch_split_invariance_and_fates(cuda_device):
    from pyrite_b200 import configs

    spec = configs.c2_si_50mev(seed=99)
    one = _run(spec, "mixed", 1, cuda_device)
    two = _run(spec, "mixed", 2, cuda_device)
    assert int(one["fates"].sum()) == H
    for k in ("fates", "exit_E", "exit_theta"):
        np.testing.assert_array_equal(one[k], two[k])
    for k in ("cxr", "brem"):
        peak = np.max(np.abs(one[k]))
        assert peak > 0
        assert np.max(np.abs(one[k] - two[k])) <= 2e-6 * peak
    np.testing.assert_allclose(one["deposit_keV"], two["deposit_keV"], rtol=1e-9)
