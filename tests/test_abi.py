"""The C-ABI library loads and exports every entry point its headers declare;
without a GPU every call that needs the device fails loudly."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\**\s*(fb_[a-z0-9_]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from fargo3d_b200 import _abi
    lib = _abi.lib()
    names = declared_symbols()
    assert "fb_disk_step" in names and len(names) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fargo3d_b200 import Disk, FargoError, config_fargo2d
    with pytest.raises(FargoError) as e:
        Disk(config_fargo2d(32, 16))
    assert "FB_ERR_CUDA" in str(e.value)
    from fargo3d_b200 import Server
    with pytest.raises(FargoError) as e:
        Server("fp32")
    assert "FB_ERR_CUDA" in str(e.value)


def test_params_bytes_bound():
    """fb_params_bytes (host arithmetic only): the fields dominate and the
    bound scales with cells and element size."""
    from fargo3d_b200 import config_fargo2d, config_p3disof
    from fargo3d_b200._abi import params_bytes
    c = config_fargo2d(384, 128)
    b64, b32 = params_bytes(c, "fp64"), params_bytes(c, "fp32")
    cells = 384 * (128 + 6)
    assert 11 * cells * 8 <= b64 <= 11 * cells * 8 * 1.2
    assert 11 * cells * 4 <= b32 < b64
    c3 = config_p3disof(64, 32, 16)
    assert params_bytes(c3, "fp64") >= 22 * 64 * 38 * 22 * 8


def test_params_layout_matches_oracle():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fargo3d_b200 import _abi
    a = [(n, getattr(_abi.FbParams, n).offset) for n, _ in _abi.FbParams._fields_]
    b = [(n, getattr(pyoracle.FoParams, n).offset) for n, _ in pyoracle.FoParams._fields_]
    assert a == b
    assert C.sizeof(_abi.FbParams) == C.sizeof(pyoracle.FoParams)
