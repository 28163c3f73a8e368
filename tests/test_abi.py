"""The C-ABI library loads and exports every symbol include/*.h declares."""
import re
from pathlib import Path

import pytest

from conftest import ROOT, has_cuda


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(imp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_exported_list(pkg):
    assert declared_functions() == sorted(pkg.EXPORTED)


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings(pkg):
    L = pkg.lib()
    assert L.imp_abi_version() == 100
    for s in range(9):
        assert L.imp_status_string(s)
    assert L.imp_status_string(0) == b"ok"


@pytest.mark.skipif(has_cuda(), reason="checks the no-GPU error path")
def test_context_create_without_gpu_fails_cleanly(pkg):
    with pytest.raises(pkg.ImpError) as e:
        pkg.Context(0)
    assert e.value.status in (1, 2)


@pytest.mark.skipif(has_cuda(), reason="checks the no-GPU error path")
def test_mgpu_without_gpu_fails_cleanly(pkg):
    """-mgpu with no visible GPU: an error status and message, no worker runs."""
    import numpy as np
    a = np.zeros(16, np.float32)
    with pytest.raises(pkg.ImpError) as e:
        pkg.bruteForceMgpu(pkg.bf_options(cg_num=2), a, a, a, a, a, a, a, a, a, a, a, a, a, a,
                           16, 16, 1, 1)
    assert e.value.status == 2 and "device" in str(e.value)


def test_invalid_device_is_rejected(pkg):
    with pytest.raises(pkg.ImpError):
        pkg.Context(9999)


def test_no_cpu_fallback_symbols(pkg):
    """The product library must not carry the oracle's entry points."""
    L = pkg.lib()
    for n in ("orc_ft", "orc_bf_cg", "ref_bf_cg", "bruteForceCpu"):
        assert not hasattr(L, n)
