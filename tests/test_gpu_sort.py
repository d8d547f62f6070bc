"""The replay kernel's block-wide sort (partition rounds and leaf insertion sorts in parallel) gives
libstdc++ std::sort's permutation (the reference's unstable sort of detections by scale) on
tie-heavy sequences, the detector's own case of descending runs, sizes across the block form's range
and beyond it (where one thread sorts), and the golden permutations recorded from the reference."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from compactcnncascade_b200 import _capi  # noqa: E402
from oracle import oracle as orc  # noqa: E402
from tests.goldens import golden  # noqa: E402


def _perm_device(keys):
    keys = np.ascontiguousarray(keys, np.float32)
    perm = np.empty(len(keys), np.int32)
    st = _capi.lib().ccnn_sort_permutation_device(keys.ctypes.data_as(ctypes.c_void_p), len(keys), perm.ctypes.data_as(ctypes.c_void_p))
    assert st == 0, _capi.last_error()
    return perm


def test_block_sort_golden():
    for rec in golden()["sort"]:
        keys = np.array([np.frombuffer(bytes.fromhex(k), "<f4")[0] for k in rec["keys"]], np.float32)
        assert _perm_device(keys).tolist() == rec["perm"]


def test_block_sort_random():
    rng = np.random.default_rng(11)
    for trial in range(400):
        n = int(rng.integers(0, 2000)) if trial % 10 else int(rng.integers(2000, 13000))
        kind = trial % 5
        if kind == 0:
            keys = rng.integers(0, 3, n).astype(np.float32)
        elif kind == 1:
            keys = np.sort(rng.integers(0, 13, n))[::-1].astype(np.float32)  # the detector's case: descending runs
        elif kind == 2:
            keys = rng.random(n).astype(np.float32)
        elif kind == 3:
            keys = np.repeat(rng.random(max(1, n // 20)).astype(np.float32), 20)[:n]
        else:
            keys = (np.arange(n) % 5).astype(np.float32)
        assert _perm_device(keys).tolist() == orc.sort_perm(keys).tolist(), (trial, n)
