"""The C ABI library loads without a GPU and exports every entry point that
include/dfft.h declares; host-only queries work through it."""
import os
import re

import dfft
from dfft import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "dfft.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dfft_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(_lib.lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_version_and_errors_without_gpu():
    assert dfft.__version__.startswith("dfft-b200")
    try:
        dfft.Plan((8, 8, 8), (8, 8, 8), (0, 1, 2), (2, 1, 1), (1, 1, 4), analyze_only=True)
    except dfft.DistributedFFTError as e:
        assert e.status == dfft.Status.INVALID_TOPOLOGY
        assert "same size" in str(e)
    else:
        raise AssertionError("expected an error")


def test_local_extents_and_offsets():
    # (10, 7) on topology (3, 1): extents 4,3,3 and starts 0,4,7 (compute_local_extents_and_starts example)
    p = dfft.Plan((10, 7, 4), (10, 7, 4), (1, 2), (3, 1, 1), (3, 1, 1), analyze_only=True)
    assert [p.local_extents(r)[0][0] for r in range(3)] == [4, 3, 3]
    assert [p.local_extents(r)[1][0] for r in range(3)] == [0, 4, 7]
    assert [p.local_offset(r) for r in range(3)] == [0, 4 * 28, 7 * 28]
    assert p.buffer_elements("in") == 280
