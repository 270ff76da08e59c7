"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "hyperprec_gpu.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "hp_f128_gemm" in syms and "hp_last_error" in syms


def test_library_exports_every_declared_symbol(hp):
    import quadprec_b200.build as b

    b.build()
    L = hp.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_table_matches_header(hp):
    assert sorted(hp.SIGNATURES) == declared_symbols()


def test_no_device_means_error_not_fallback(hp):
    """Without a GPU every compute entry point returns HP_ERR_CUDA."""
    import numpy as np

    if hp.device_ok():
        pytest.skip("a CUDA device is present")
    a = np.zeros((2, 2, 2))
    with pytest.raises(hp.HPError) as ei:
        hp.f128_gemm(a, a, 2, 2, 2)
    assert ei.value.code == hp.HP_ERR_CUDA
