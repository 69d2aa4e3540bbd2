"""Device-resident corpus I/O: code files streamed into HBM (turboquant.io)
and DLPack inputs (CUDA producers exposing only __dlpack__)."""
import numpy as np
import pytest

import turboquant as tq

pytestmark = pytest.mark.gpu


class _DLPackOnly:
    """A CUDA array that exposes DLPack but not __cuda_array_interface__."""

    def __init__(self, t):
        self._t = t

    def __dlpack__(self, stream=None):
        return self._t.__dlpack__(stream=stream)

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


def _codes(dim=256, bits=4, n=5003):
    s = tq.TurboQuantSpace(dim, bits)
    X = np.random.default_rng(n).standard_normal((n, dim)).astype(np.float32)
    return s, s.encode_batch(X)


def test_load_codes_npy_raw_and_array(cuda_ok, tmp_path):
    s, codes = _codes()
    np.save(tmp_path / "c.npy", codes)
    codes.tofile(tmp_path / "c.bin")
    for src in (tmp_path / "c.npy", str(tmp_path / "c.bin"), codes):
        d = tq.load_codes(src, s, chunk_bytes=64 * 1024)  # many chunks, ragged last
        assert d.is_cuda and tuple(d.shape) == codes.shape
        np.testing.assert_array_equal(d.cpu().numpy(), codes)
    with pytest.raises(ValueError, match="codes size not a multiple of code_size_bytes"):
        tq.load_codes(codes.reshape(-1)[:-1], s)


def test_dlpack_inputs_match_host_path(cuda_ok):
    import torch
    s, codes = _codes(768, 8, 2001)
    q = np.random.default_rng(1).standard_normal(768).astype(np.float32)
    cd = _DLPackOnly(torch.from_numpy(codes).cuda())
    qd = _DLPackOnly(torch.from_numpy(q).cuda())
    got = s.distance_1_to_n(qd, cd)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), s.distance_1_to_n(q, codes))
    sym = s.distance_m_to_n_symmetric(_DLPackOnly(torch.from_numpy(codes[:5]).cuda()), cd)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(sym.cpu().numpy(), s.distance_m_to_n_symmetric(codes[:5], codes))
