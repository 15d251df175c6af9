"""The C-ABI library loads and exports every function include/prt.h declares
(no GPU needed: nothing here launches work)."""

import re
from pathlib import Path

import pytest

from pyrticle_b200 import _lib

HEADER = Path(__file__).resolve().parent.parent / "include" / "prt.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(prt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_bound_functions():
    decl = declared_functions()
    assert set(decl) == set(_lib.SIGNATURES), set(decl) ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    if not _lib.LIB_PATH.exists():
        pytest.skip("libprt.so not built")
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.prt_version()


def test_struct_layouts_match_header():
    import ctypes as C
    # offsets the C side relies on
    assert C.sizeof(_lib.ShapeFunctionDesc) == 24
    assert C.sizeof(_lib.Brick) == 3 * 8 + 3 * 8 + 4 * 4 + 8
    assert C.sizeof(_lib.FindCounters) == 32
    assert C.sizeof(_lib.DepositStats) == 13 * 8


def test_product_path_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pyrticle_b200 import cloud
    with pytest.raises(RuntimeError, match="CUDA device"):
        cloud.device()
