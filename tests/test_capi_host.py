"""Host-side checks of the product library that need no GPU: the C ABI loads
and exports what include/turboquant_b200.h declares, the space's geometry and
tables equal the reference's, the quantizer's bucket table is exact, and the
Python mirror raises the reference binding's errors (bindings.cpp:14-49,
159-209) before any device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import turboquant as tq
from turboquant import _capi
from conftest import GOLDEN_CASES, ROOT, load_case


def _declared_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(tq_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_capi.EXPORTS) == declared


def test_version():
    assert b"sm_100a" in _capi.lib().tq_version()


@pytest.mark.parametrize("dim,bits", GOLDEN_CASES)
def test_geometry_and_tables_equal_reference(dim, bits):
    g = load_case(dim, bits)
    s = tq.TurboQuantSpace(dim, bits)
    assert s.dim() == dim and s.bits_per_coord() == bits
    D = 1
    while D < max(dim, 4):
        D *= 2
    assert s.padded_dim() == D and s.padded() == (D != dim)
    assert s.code_size_bytes() == g["codes"].shape[1]
    c, b, rs, qs = s.tables()
    np.testing.assert_array_equal(c, g["centroids"])
    np.testing.assert_array_equal(b, g["boundaries"])
    np.testing.assert_array_equal(rs, g["rot_signs"])
    np.testing.assert_array_equal(qs, g["qjl_signs"])
    assert np.float32(s.scale()) == g["scale"]


@pytest.mark.parametrize("bits", [2, 3, 4, 5, 6, 7, 8, 9])
def test_quantizer_table_is_exact(bits):
    s = tq.TurboQuantSpace(64, bits)
    _, b, _, _ = s.tables()
    rng = np.random.default_rng(bits)
    z = [rng.standard_normal(200_000).astype(np.float32) * 1.5,
         np.array([0.0, -0.0, np.inf, -np.inf, 1e30, -1e30, 1e-40, -1e-40], np.float32)]
    for bb in b:   # every boundary and its float neighbours
        z.append(np.array([bb, np.nextafter(bb, np.float32(np.inf)),
                           np.nextafter(bb, np.float32(-np.inf))], np.float32))
    z = np.concatenate(z).astype(np.float32)
    want = (z[:, None] > b[None, :]).sum(axis=1).astype(np.uint8)
    np.testing.assert_array_equal(s.quantize(z), want)


def test_padding_warning(capfd):
    tq.TurboQuantSpace(100, 4)
    assert "padding to 128" in capfd.readouterr().err


def test_constructor_rejects_bad_bits():
    with pytest.raises(ValueError, match="need at least 2 bits"):
        tq.TurboQuantSpace(64, 1)
    with pytest.raises(ValueError, match="max 9 bits"):
        tq.TurboQuantSpace(64, 10)
    with pytest.raises(ValueError, match="dim must be >= 1"):
        tq.TurboQuantSpace(0, 4)


def test_defaults_match_reference():
    s = tq.TurboQuantSpace(32)
    assert s.bits_per_coord() == 4
    c, _, rs, qs = s.tables()
    np.testing.assert_array_equal(rs, O.OracleSpace(32, 4, 42, 137).tables()[2])
    np.testing.assert_array_equal(qs, O.OracleSpace(32, 4, 42, 137).tables()[3])


@pytest.mark.parametrize("call,args,msg", [
    ("encode_batch", (np.zeros((3, 64), np.float64),), "input: expected float32"),
    ("encode_batch", (np.zeros(64, np.float32),), "input: wrong ndim"),
    ("encode_batch", (np.zeros((3, 63), np.float32),), "input: wrong dim"),
    ("encode_batch", (np.zeros((3, 128), np.float32)[:, ::2],), "input: must be C-contiguous float32"),
    ("encode", (np.zeros(63, np.float32),), "input: wrong length"),
    ("distance_1_to_n", (np.zeros(64, np.float32), np.zeros(45, np.uint8)),
     "codes size not a multiple of code_size_bytes"),
    ("distance_1_to_n", (np.zeros(64, np.float32), np.zeros(44, np.int32)), "codes must be uint8"),
    ("distance_1_to_n", (np.zeros(65, np.float32), np.zeros(44, np.uint8)), "query: wrong length"),
    ("distance_m_to_n", (np.zeros((2, 64), np.float32), np.zeros(45, np.uint8)),
     "codes size not a multiple of code_size_bytes"),
    ("distance_m_to_n", (np.zeros(64, np.float32), np.zeros(44, np.uint8)), "queries: wrong ndim"),
    ("distance_m_to_n_symmetric", (np.zeros(44, np.uint8), np.zeros(45, np.uint8)),
     "codes size not a multiple of code_size_bytes"),
    ("distance_m_to_n_symmetric", (np.zeros(44, np.float32), np.zeros(44, np.uint8)),
     "codes must be uint8"),
    ("distance", (np.zeros(64, np.float32), np.zeros(43, np.uint8)), "code: wrong byte size"),
    ("distance_symmetric", (np.zeros(44, np.uint8), np.zeros(43, np.uint8)), "code_b: wrong byte size"),
])
def test_validation_errors_match_reference(call, args, msg):
    s = tq.TurboQuantSpace(64, 4)   # cs = 44
    assert s.code_size_bytes() == 44
    with pytest.raises(ValueError, match=re.escape(msg)):
        getattr(s, call)(*args)


def test_encode_into_rejects_readonly_and_wrong_size():
    s = tq.TurboQuantSpace(64, 4)
    with pytest.raises(ValueError, match="codes: wrong byte size"):
        s.encode_batch_into(np.zeros((2, 64), np.float32), np.zeros(87, np.uint8))
    ro = np.zeros(88, np.uint8)
    ro.flags.writeable = False
    with pytest.raises(BufferError):
        s.encode_batch_into(np.zeros((2, 64), np.float32), ro)


def test_compute_without_gpu_fails_loudly():
    """No silent CPU path: without a device every compute call raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = tq.TurboQuantSpace(64, 4)
    with pytest.raises(tq.TQError, match="no CUDA device"):
        s.encode_batch(np.zeros((2, 64), np.float32))
    with pytest.raises(tq.TQError, match="no CUDA device"):
        s.distance_1_to_n(np.zeros(64, np.float32), np.zeros(44, np.uint8))
    for prec in _capi.PRECISION:
        with pytest.raises(tq.TQError, match="no CUDA device"):
            s.distance_m_to_n(np.zeros((2, 64), np.float32), np.zeros((3, 44), np.uint8), precision=prec)
    code = ctypes.c_int(-1)
    st = _capi.lib().tq_space_take_device_status(s._h, ctypes.byref(code))
    assert st != 0 and code.value == 0


def test_precision_names_match_the_header():
    """The Python mirror's precision keywords are the header's tq_precision
    values: "split_bf16_decoded" is TQ_PRECISION_SPLIT_BF16_DECODED, and so on."""
    text = open(os.path.join(ROOT, "include", "turboquant_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    enum = {m.group(1).lower(): int(m.group(2))
            for m in re.finditer(r"\bTQ_PRECISION_([A-Z0-9_]+)\s*=\s*(\d+)", text)}
    assert enum == _capi.PRECISION, (enum, _capi.PRECISION)
