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
