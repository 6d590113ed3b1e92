"""The C-ABI library loads and exports every entry point the header declares (no GPU needed)."""

import ctypes
import re
from pathlib import Path

import pytest

from pystarc_b200 import _lib
from pystarc_b200 import build as b

HEADER = Path(__file__).resolve().parents[1] / "include" / "pystarc_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(bd_\w+)\s*\(", text, flags=re.M)))


def test_header_and_binding_agree():
    names = declared()
    assert len(names) >= 20
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_library_exports_all_symbols():
    b.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in declared():
        assert hasattr(lib, n), n
    assert _lib.load().bd_version().startswith(b"pystarc_b200")


def test_errors_are_codes_not_crashes():
    lib = _lib.load()
    buf = ctypes.create_string_buffer(256)
    assert lib.bd_create(0, None) == _lib.BD_ERR_ARG
    assert lib.bd_last_error(None, buf, 256) == 0 and b"NULL" in buf.value
    assert lib.bd_destroy(None) == 0
    assert lib.bd_set_ligand(None, 1, None, None) == _lib.BD_ERR_ARG
    assert lib.bd_set_contact(None, 0, None, 0, None, 0.17, -1.0) == _lib.BD_ERR_ARG
    assert lib.bd_set_reaction_states(None, 0, None, None, 0, None) == _lib.BD_ERR_ARG
    assert lib.bd_sim_reaction_fires(None, None, None, 0) == _lib.BD_ERR_ARG
    assert lib.bd_sim_get_states(None, None) == _lib.BD_ERR_ARG
    assert lib.bd_sim_set_states(None, None) == _lib.BD_ERR_ARG


_NO_HANDLE = {"bd_version", "bd_create", "bd_destroy", "bd_last_error", "bd_mlp_last_error", "bd_mlp_destroy",
              "bd_multi_destroy"}


def test_every_entry_point_rejects_a_null_handle():
    """Each entry point that takes a handle returns BD_ERR_ARG for NULL (zero sizes, NULL arrays)
    before it touches the GPU; destroying NULL is a no-op."""
    lib = _lib.load()
    ints = (ctypes.c_int, ctypes.c_int8, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_uint64,
            ctypes.c_long, ctypes.c_longlong, ctypes.c_size_t)
    for name, (_, args) in _lib.SIGNATURES.items():
        if name in _NO_HANDLE:
            continue
        vals = [0 if a in ints else 0.0 if a in (ctypes.c_double, ctypes.c_float) else None for a in args]
        assert getattr(lib, name)(*vals) == _lib.BD_ERR_ARG, name
    assert lib.bd_multi_destroy(None) == 0


def test_create_without_gpu_reports_cuda_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = _lib.P()
    rc = lib.bd_create(0, ctypes.byref(h))
    assert rc == _lib.BD_ERR_CUDA
    buf = ctypes.create_string_buffer(256)
    lib.bd_last_error(None, buf, 256)
    assert buf.value
