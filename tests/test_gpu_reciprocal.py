"""The rational tanh's reciprocal 1/den (cnnpp_cplusplus.cpp:662-666) is computed by the kernels
with a packed Newton-Raphson reciprocal; it must equal the IEEE reciprocal for every float."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from compactcnncascade_b200 import _capi  # noqa: E402


def test_packed_reciprocal_is_ieee_for_every_float_from_one():
    bad, n = ctypes.c_longlong(-1), ctypes.c_longlong(0)
    assert _capi.lib().ccnn_check_reciprocal(ctypes.byref(bad), ctypes.byref(n)) == 0, _capi.last_error()
    assert n.value > 1_000_000_000
    assert bad.value == 0
