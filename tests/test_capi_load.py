"""CPU checks of the drop-in boundary: the sm_100a library loads and
exports every entry point that include/*.h declares (the device ABI
bn_b200.h and the host-side bn_host.h)."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(headers=("bn_b200.h", "bn_host.h")):
    syms = set()
    for h in headers:
        with open(os.path.join(ROOT, "include", h)) as f:
            text = f.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(bn_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_header_declares_boundary():
    syms = declared_symbols()
    for must in ("bn_flat_build", "bn_flat_compute_products", "bn_flat_decode_dense_terms", "bn_flat_verify",
                 "bn_flat_query", "bn_ivf_build", "bn_ivf_compute_products", "bn_ivf_query", "bn_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from bn_b200 import capi

    syms = declared_symbols()
    assert "bn_host_encode_query" in syms and "bn_host_ivf_cache_open" in syms and "bn_ivf_route" in syms
    missing = [s for s in syms if not hasattr(capi.lib, s)]
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
