"""The C-ABI library builds, loads without a GPU and exports every function the header declares."""

from __future__ import annotations

import ctypes
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, "include", "aldvc_b200.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(aldvc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from pyaldvc_b200 import _lib
    from pyaldvc_b200.build import build

    path = build()
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.PROTOTYPES), "ctypes prototypes and header disagree"


def test_abi_version_and_error_string_without_gpu():
    from pyaldvc_b200 import _lib

    L = _lib.load()
    assert L.aldvc_abi_version() == 1
    # argument validation runs on the host: a null descriptor is rejected with a message
    rc = L.aldvc_precompute(None, None, None, 0, 0.5, 1e12, None, None, None, None, None, None, None)
    assert rc == -1
    assert b"null" in L.aldvc_last_error()


def test_workspace_queries_are_host_only():
    from pyaldvc_b200 import _lib

    L = _lib.load()
    sub = _lib.Subset(12, 12, 12, 1, 1, 0, None, None, 0)
    batched = _lib.IcgnParams(1e-2, 1e-3, 100, 5, 0.0, 1, 0, 0, 0, 0.0, 0.0)
    plain = _lib.IcgnParams(1e-2, 1e-3, 100, 5, 0.0, 1, 1, 0, 0, 0.0, 0.0)
    n = 4096
    wb = L.aldvc_icgn_workspace_size(ctypes.byref(sub), n, ctypes.byref(batched))
    wp = L.aldvc_icgn_workspace_size(ctypes.byref(sub), n, ctypes.byref(plain))
    assert wb >= 4 and wp >= n * 25 ** 3 * 4  # the plain form keeps a sample row per node in flight
    assert L.aldvc_ncc_search_workspace_size(128, 128, 128, n, 8, 8, 8, 8, 8, 8, 1) >= 17 ** 3 * 4
