"""CPU-only checks of the C ABI: the library loads without a GPU and exports
every entry point include/par2gpu.h declares, with the ctypes signatures the
Python front end uses."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(prefix="p2g"):
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(%s_[a-z0-9_]+)\s*\(" % prefix, text))
    return names


def test_format_library_exports_every_declared_symbol():
    from par2gpu import format as fmt

    L = ctypes.CDLL(fmt.LIB_PATH)
    names = declared_symbols("p2f")
    assert {"p2f_create", "p2f_create_ex", "p2f_repair", "p2f_repair_ex",
            "p2f_last_error"} <= names
    for n in sorted(names):
        assert hasattr(L, n), f"missing export {n}"
    assert names == {s[0] for s in fmt.SIGNATURES}


def test_library_exports_every_declared_symbol():
    import par2gpu

    L = ctypes.CDLL(par2gpu.LIB_PATH)
    names = declared_symbols()
    assert "p2g_encode" in names and "p2g_muladd_region" in names
    for n in sorted(names):
        assert hasattr(L, n), f"missing export {n}"
    bound = {s[0] for s in par2gpu.SIGNATURES}
    assert names == bound, f"header vs binding mismatch: {names ^ bound}"


def test_strategy_info_without_gpu():
    import par2gpu

    name, prio, avail = par2gpu.strategy_info()
    assert name == "CUDA-sm100a"
    assert prio == par2gpu.PRIORITY_OPTIMAL


def test_constants_match_oracle():
    import par2gpu
    from oracle import oracle

    assert (par2gpu.par2_constants(5000) == oracle.par2_constants(5000)).all()


def test_create_fails_loudly_without_device():
    import torch

    import par2gpu

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        par2gpu.Context(0)
    assert ei.value.code == par2gpu.ENODEV
