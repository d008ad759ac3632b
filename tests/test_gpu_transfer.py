"""Reference-layout state transfers through the C ABI (cfd_upload_field / cfd_download_field)
with pinned host buffers, issued as a user's time loop issues them: upload u, v, w, p, step,
download them into the same host buffers, with no host synchronisation until the end.  The
library orders each field's upload after its previous download (own staging buffers and copy
streams), so the result must equal the same steps run on the device alone, bit for bit."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FID = {"u1": 0, "u2": 1, "u3": 2, "p": 3}


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.float64).copy()).pin_memory()


@pytest.mark.parametrize("prec,grid", [("fp64", (64, 96, 17)), ("mixed", (64, 96, 17)), ("fp64", (24, 18, 17))])
def test_unsynchronised_round_trips_equal_device_steps(torch_cuda, prec, grid):
    """(24, 18, 17) has 108 columns: transfer chunks of 14 and a last one of 10."""
    from cfd_b200.channel import Channel, build_channel
    from cfd_b200.config import tiny
    s = build_channel(tiny(*grid, cyl_diameter=0.3, cyl_spacing=1.5, seed=21))
    ref = Channel(s, device=0, precision=prec)
    ref.upload_state()
    ref.step(4)
    want = ref.download_state()
    ref.close()

    ch = Channel(s, device=0, precision=prec)
    host = {k: pinned(torch_cuda, v) for k, v in s.state().items()}
    ptr = {k: C.cast(h.data_ptr(), C.POINTER(C.c_double)) for k, h in host.items()}
    for _ in range(4):
        for k in FID:
            assert ch.lib.cfd_upload_field(ch.ctx, FID[k], ptr[k], 0) == 0
        ch.step(1)
        for k in FID:
            assert ch.lib.cfd_download_field(ch.ctx, FID[k], ptr[k], 0) == 0
    ch.synchronize()
    for k in FID:
        got = host[k].numpy().view(np.complex128).reshape(want[k].shape)
        assert np.array_equal(got, want[k]), k
    # a later synchronous download of the same state gives the same fields
    st = ch.download_state()
    for k in FID:
        assert np.array_equal(st[k], want[k]), k
    ch.close()
