"""The C-ABI library loads and exports every function include/hitomi_gpu.h declares
(no compute call: runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "hitomi_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hg_[a-z_]+)\s*\(", src)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for n in ("hg_create", "hg_destroy", "hg_last_error", "hg_set_particles", "hg_pk_box", "hg_bk_box"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from hitomi_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.SYMBOLS) == set(declared_functions())


def test_create_without_gpu_fails_with_message():
    import torch
    if torch.cuda.is_available():
        return
    from hitomi_b200.api import Binning, Context, HitomiError
    try:
        Context(32, 1000.0, Binning(0.01, 0.1, 5))
    except HitomiError as e:
        assert "cuda" in str(e).lower()
    else:
        raise AssertionError("context creation must fail loudly without a GPU")
