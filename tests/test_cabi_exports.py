"""The C-ABI library loads on a CPU-only host and exports every symbol that
include/openjij_b200.h declares."""
import ctypes
import os
import re

from openjij_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "openjij_b200.h")).read()
    decl = re.findall(r"^(?:const\s+)?[a-z_0-9]+\s*\*?\s*(oj_[a-z0-9_]+)\s*\(", hdr, re.M)
    return sorted(set(decl))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(N.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(N.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_status_strings_and_version():
    L = N.lib()
    assert b"sm_100a" in L.oj_version()
    assert L.oj_status_string(N.OJ_ERR_ARG) == b"invalid argument"
    assert L.oj_status_string(N.OJ_ERR_UNSUPPORTED).startswith(b"unsupported")


def test_null_arguments_are_rejected_without_a_device():
    L = N.lib()
    assert L.oj_ctx_create(0, None) == N.OJ_ERR_ARG
    assert L.oj_graph_destroy(None) == N.OJ_OK
    assert L.oj_ctx_destroy(None) == N.OJ_OK


def test_host_blocks_are_ordinary_memory_without_a_device():
    """oj_host_alloc on a host without a GPU: usable ordinary memory, not
    reported as page-locked, freed by oj_host_free."""
    import torch

    if torch.cuda.is_available():
        return  # with a device the block is page-locked (GPU test)
    L = N.lib()
    p = L.oj_host_alloc(100003)
    assert p
    assert L.oj_host_is_pinned(p) == 0
    ctypes.memset(p, 0x5A, 100003)
    assert ctypes.string_at(p + 100002, 1) == b"\x5a"
    L.oj_host_free(p)
    L.oj_host_free(None)
