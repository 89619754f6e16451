"""CPU checks of the drop-in boundary: the sm_100a library loads and
exports every entry point that include/bn_b200.h declares."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "bn_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bn_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_boundary():
    syms = declared_symbols()
    for must in ("bn_flat_build", "bn_flat_compute_products", "bn_flat_decode_dense_terms", "bn_flat_verify",
                 "bn_flat_query", "bn_ivf_build", "bn_ivf_compute_products", "bn_ivf_query", "bn_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from bn_b200 import capi

    missing = [s for s in declared_symbols() if not hasattr(capi.lib, s)]
    assert not missing, missing


def test_build_info_and_device_count_without_gpu():
    from bn_b200 import capi

    assert "sm_100a" in capi.build_info()
    assert capi.device_count() >= 0


def test_no_device_is_a_clean_error():
    from bn_b200 import capi

    if capi.device_count() > 0:
        pytest.skip("a device is visible")
    with pytest.raises(capi.BnError) as e:
        capi.Context(0)
    assert e.value.code == capi.BN_ENODEV
