"""The staged 1->N scan against the oracle: byte units (bits >= 5, D 128 ..
1024) and nibble units (bits <= 4, D 128 .. 2048).

distance_1_to_n on a 16-byte aligned device corpus runs the staged kernel:
groups of 4 codes are bulk-copied into per-warp shared-memory rings and the
last n mod 4 codes are read with plain loads.  A corpus at a 4-byte (not
16-byte) offset runs the register-fed kernels instead.  Both must agree with
the oracle within DIST_RTOL for every count, ragged tails and ring wrap-around
included; for byte units the two kernels share their arithmetic and agree bit
for bit.
"""
import numpy as np
import pytest

import oracle as O
import turboquant as tq
from conftest import asym_term_scale, dist_close

pytestmark = pytest.mark.gpu

# (dim, bits): D = 128, 256, 512, 1024 with byte units (bits >= 5) and
# D = 128 (a half-warp per code), 256, 512, 1024, 2048 with nibble units
STAGED = [(128, 8), (200, 5), (500, 9), (768, 8), (1024, 6),
          (128, 4), (100, 3), (256, 4), (300, 3), (768, 4), (1536, 2), (2048, 4)]
COUNTS = [1, 2, 3, 4, 5, 7, 63, 1001, 4099]


def _corpus(dim, bits, n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, dim)).astype(np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    q = rng.standard_normal(dim).astype(np.float32)
    s = tq.TurboQuantSpace(dim, bits)
    return s, s.encode_batch(X), q


def _device_scan(s, q, codes, offset):
    """distance_1_to_n on device buffers; the corpus starts `offset` bytes
    into a fresh (256-byte aligned) allocation."""
    import torch
    flat = codes.reshape(-1)
    buf = torch.empty(flat.size + 16, dtype=torch.uint8, device="cuda")
    dev = buf[offset:offset + flat.size]
    dev.copy_(torch.from_numpy(flat))
    assert dev.data_ptr() % 16 == (offset % 16)
    d = s.distance_1_to_n(torch.from_numpy(q).cuda(), dev.view(-1, s.code_size_bytes()))
    torch.cuda.synchronize()
    return d.cpu().numpy()


@pytest.mark.parametrize("dim,bits", STAGED)
def test_staged_scan_counts_vs_oracle(cuda_ok, dim, bits):
    s, codes_all, q = _corpus(dim, bits, max(COUNTS), seed=dim + bits)
    cs = s.code_size_bytes()
    pb = cs - 12
    for n in COUNTS:
        codes = codes_all[:n]
        ref = O.OracleSpace(dim, bits).distance_1_to_n(q, codes)
        got = _device_scan(s, q, codes, 0)
        ts = asym_term_scale(q, codes, cs, pb)[0]
        err, ok = dist_close(got, ref, ts)
        assert ok, f"n={n}: max rel err {err.max():.3e}"
        # the unaligned corpus takes the register-fed kernel
        other = _device_scan(s, q, codes, 4)
        if bits >= 5:
            np.testing.assert_array_equal(other, got)
        else:
            err, ok = dist_close(other, ref, ts)
            assert ok, f"n={n}, unaligned: max rel err {err.max():.3e}"


@pytest.mark.parametrize("dim,bits,n", [(128, 8, 100003), (768, 8, 50001), (384, 4, 200003),
                                        (1536, 4, 30001), (128, 4, 300001)])
def test_staged_scan_many_groups_per_warp(cuda_ok, dim, bits, n):
    """Enough codes that every warp wraps its ring several times and runs
    several 16-code batches, with a ragged tail."""
    s, codes, q = _corpus(dim, bits, n, seed=7)
    cs = s.code_size_bytes()
    ref = O.OracleSpace(dim, bits).distance_1_to_n(q, codes)
    got = _device_scan(s, q, codes, 0)
    ts = asym_term_scale(q, codes, cs, cs - 12)[0]
    err, ok = dist_close(got, ref, ts)
    assert ok, f"max rel err {err.max():.3e}"
    other = _device_scan(s, q, codes, 4)
    if bits >= 5:
        np.testing.assert_array_equal(other, got)
    else:
        assert dist_close(other, ref, ts)[1]


def test_staged_scan_host_path_equals_device(cuda_ok):
    """The host-pointer entry point (chunked H2D, staged kernel per chunk)
    gives the device path's numbers."""
    s, codes, q = _corpus(768, 8, 20001, seed=3)
    np.testing.assert_array_equal(s.distance_1_to_n(q, codes), _device_scan(s, q, codes, 0))


def test_device_status_word_clean_after_scans(cuda_ok):
    """No bounded wait gave up in the scans above: the status word reads 0."""
    import ctypes
    from turboquant import _capi
    s, codes, q = _corpus(768, 8, 4099, seed=11)
    _device_scan(s, q, codes, 0)
    code = ctypes.c_int(-1)
    assert _capi.lib().tq_space_take_device_status(s._h, ctypes.byref(code)) == 0
    assert code.value == 0
