"""Float32 against Float64 on the GPU (moist2d_b200.precision): the warm bubble (200 x 100 cells,
dt = 1 s) after 300 large steps, per field. The bounds are a few times the errors measured on a
B200 and guard against a regression of the Float32 path (e.g. losing the FP64 elimination)."""
import numpy as np
import pytest

from moist2d_b200 import precision
from moist2d_b200.init import warm_bubble

pytestmark = pytest.mark.gpu

# measured: theta 8.0e-7, u 5.1e-5, w 5.8e-5, qv 6.6e-5, qc 1.0e-4, qr 1.1e-4, rain 3.9e-4
BOUNDS = {"theta": 1e-5, "u": 5e-4, "w": 5e-4, "qv": 5e-4, "qc": 1e-3, "qr": 1e-3, "rain": 4e-3}


def test_fp32_error_against_fp64():
    res = precision.run(warm_bubble, 300)
    for k, v in res.items():
        print("%-5s rel_l2 %.3e  max_abs %.3e  max_ref %.3e" % (k, v["rel_l2"], v["max_abs"], v["max_ref"]))
        assert np.isfinite(v["rel_l2"]) and v["rel_l2"] < BOUNDS[k], k
