"""The kernels replace IEEE division by a fixed divisor (the box sizes 9 and
25 of the guided filter and the USM blur) with Markstein's two-FMA method;
this checks it against the GPU's IEEE division on every binary32 value in its
range, bit for bit (filmic's log(109) as a third divisor the method holds for)."""
import ctypes as C

import numpy as np
import pytest
from cpipe_b200 import _abi as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("divisor", [9.0, 25.0, float(np.float32(np.log(109.0)))])
def test_const_division_equals_ieee_everywhere(cuda_device, divisor):
    bad, seen = C.c_uint64(), C.c_uint64()
    assert A.lib().cpipe_cuda_selftest_const_division(C.c_float(divisor), C.byref(bad), C.byref(seen)) == 0
    assert seen.value > 3_000_000_000  # every finite float with |x| in [2^-90, 2^126], both signs
    assert bad.value == 0, f"{bad.value} quotients differ from IEEE division by {divisor}"
