"""The device renderer of the seeded frames writes the same bytes as the host generator."""
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import numpy as np  # noqa: E402

import compactcnncascade_b200 as ccnn  # noqa: E402

CASES = [(640, 480, 1, 5, 40, 200, 3), (1920, 1080, 7, 20, 30, 300, 3), (333, 211, 3, 4, 20, 90, 1), (320, 240, 9, 3, 30, 100, 4),
         (1280, 720, 77, 0, 30, 300, 3), (800, 600, 400, 300, 20, 120, 3), (97, 61, 5, 2, 20, 90, 3)]


@pytest.mark.parametrize("w,h,seed,nf,lo,hi,ch", CASES)
def test_device_frame_equals_host_frame(w, h, seed, nf, lo, hi, ch):
    want, wf = ccnn.synth_frame(w, h, seed, nf, lo, hi, ch)
    step = (w * ch + 63) // 64 * 64  # a padded pitch as well
    buf = torch.full((h, step), 7, dtype=torch.uint8, device="cuda")
    gf = ccnn.synth_frame_device(buf.data_ptr(), w, h, seed, nf, lo, hi, channels=ch, step=step)
    got = buf.cpu().numpy()
    assert gf == wf
    assert np.array_equal(got[:, :w * ch].reshape(want.shape), want)
    assert np.all(got[:, w * ch:] == 7)  # nothing written past the row


def test_invalid_arguments_are_rejected():
    buf = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(ccnn.CCNNError):
        ccnn.synth_frame_device(buf.data_ptr(), 4, 4, 1, 1, 40, 20)  # max face below min face
    with pytest.raises(ccnn.CCNNError):
        ccnn.synth_frame_device(buf.data_ptr(), 4, 4, 1, 1, 4, 8, channels=2)
