"""The TVD limiters of kcfd.interpolation (core/interpolation.py:17-52) on numpy arrays
equal the oracle's restatement (pinned to the reference through the MUSCL fixtures),
bit for bit, including r <= 0, r = -1 and large r; get_limiter rejects unknown names."""
import numpy as np
import pytest

from kcfd.interpolation import LIMITER_REGISTRY, get_limiter
from oracle.fvm import limiter


@pytest.mark.filterwarnings("ignore::RuntimeWarning")  # r = 1e300 overflows in both, as in the reference
def test_limiters_match_oracle():
    r = np.concatenate([np.linspace(-3.0, 5.0, 801), [-1.0, 0.0, 1e-300, 1e300, -1e300]])
    for name in ("minmod", "superbee", "van_albada", "van_leer"):
        np.testing.assert_array_equal(get_limiter(name)(r), limiter(name, r))
    assert set(LIMITER_REGISTRY) == {"minmod", "superbee", "van_albada", "van_leer"}
    with pytest.raises(ValueError):
        get_limiter("koren")
