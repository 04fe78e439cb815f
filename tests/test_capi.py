"""The C-ABI library loads without a GPU and exports every function that
include/bv.h declares (and nothing is left out of the Python binding)."""
import ctypes
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "bv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bv_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(bvlib):
    from blockvecchia_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 17
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header(bvlib):
    from blockvecchia_b200 import _lib
    assert set(_declared()) <= set(_lib.EXPORTS), set(_declared()) - set(_lib.EXPORTS)


def test_no_oracle_in_product():
    """The product package never imports or links the oracle."""
    pkg = os.path.join(ROOT, "blockvecchia_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.replace("oracle/gen_rgamma_coeffs.py", ""), f


def test_errors_without_device(bvlib):
    """Host-only entry points validate their arguments and report errors."""
    import numpy as np
    bn = np.array([3, 2], dtype=np.int32)
    mask = np.zeros(2, dtype=np.uint8)
    rc = bvlib.lib().bv_shard_blocks(bn.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 2, 1, 2, 5,
                                     mask.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
    assert rc == -1
    assert b"invalid" in bvlib.lib().bv_last_error()


def test_server_without_device(bvlib):
    """bv_server_create reports a CUDA error (it does not crash) where no
    device is usable."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(bvlib.BvError):
        bvlib.Server()


def test_ctypes_structs_match_the_header(bvlib):
    """The Python binding's restated structs have the C ABI's sizes."""
    import ctypes as C
    from blockvecchia_b200 import _lib
    out = (C.c_size_t * 6)()
    assert _lib.lib().bv_abi_sizes(out, 6) == 6
    mine = [C.sizeof(t) for t in (_lib.BvLayout, _lib.BvOpts, _lib.BvStatus, _lib.BvServerOpts,
                                  _lib.BvServerStats, _lib.BvJobOpts)]
    assert list(out) == mine
