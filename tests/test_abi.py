"""The C-ABI library loads and exports every entry point include/ragdoll_cuda.h declares, and the
host-side argument checks reject bad input without touching a device (CPU test)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "ragdoll_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("rg_create", "rg_destroy", "rg_analyse_frame", "rg_analyse_batch", "rg_get_recon",
              "rg_quality_frame", "rg_ssim_plane", "rg_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from ragdoll_b200.engine import EXPORTS, lib
    L = lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, f"not exported: {missing}"
    assert set(declared_symbols()) == set(EXPORTS)


def test_create_rejects_bad_config_without_a_device():
    from ragdoll_b200.engine import RgConfig, lib
    L = lib()
    for cfg in (RgConfig(0, 1080, 2, 26, 1, 0), RgConfig(1920, 1080, 2, 0, 1, 0),
                RgConfig(1920, 1080, 7, 26, 1, 0), RgConfig(1920, 1080, 2, 26, 0, 0)):
        assert not L.rg_create(ctypes.byref(cfg))
        assert L.rg_last_error()


def test_version_string():
    from ragdoll_b200.engine import lib
    assert b"sm_100a" in lib().rg_version()


def test_group_and_compaction_calls_reject_bad_arguments_without_a_device():
    """The group calls, the compact-record calls and the encoder's group submit check their
    arguments before touching a device: null pointers, context counts outside 1..8 and null
    contexts are RG_ERR_INVALID."""
    from ragdoll_b200.engine import lib
    L = lib()
    P = ctypes.c_void_p
    one = (P * 1)(None)
    sz = (ctypes.c_size_t * 1)(64)
    for n in (0, 9, 1):
        assert L.rg_analyse_gops_group(one, n, one, sz, sz, one, 1) < 0
        assert L.rg_analyse_gops_group_async(one, n, one, sz, sz, one, 1, one) < 0
        assert L.rg_analyse_gops_group_stream(one, n, one, sz, sz, one, 1, one) < 0
        assert L.rg_encoder_submit_group(one, n, one, sz, sz, 1) < 0
    assert L.rg_analyse_gops_group_async(None, 1, None, None, None, None, 1, None) < 0
    assert L.rg_set_record_compaction(None, 96) < 0
    data, nbytes = P(), ctypes.c_size_t()
    assert L.rg_analyse_gops_fetch_compact(None, None, 0, ctypes.byref(data), ctypes.byref(nbytes)) < 0
    assert L.rg_encoder_record_bytes(None) < 0
    cap, lau = ctypes.c_int64(), ctypes.c_int64()
    assert L.rg_group_graph_counts(None, ctypes.byref(cap), ctypes.byref(lau)) < 0
    assert L.rg_last_error()
