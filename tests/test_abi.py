"""The C-ABI library builds, loads without a GPU and exports every entry
point include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(pmc_coag_gpu_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from partmc_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from partmc_b200 import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_status_strings_without_device():
    from partmc_b200 import _lib
    L = _lib.lib()
    for code in range(0, 9):
        assert L.pmc_coag_gpu_status_string(code)


def test_init_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import numpy as np
    from partmc_b200 import _lib
    L = _lib.lib()
    ctx = ctypes.c_void_p()
    d = np.array([1000.0])
    t = np.array([1], dtype=np.int32)
    m = np.array([1.0])
    e = np.array([0.0])
    rc = L.pmc_coag_gpu_init(1, _lib.dp(d), 0, 1, 1, _lib.ip(t), _lib.dp(m), _lib.dp(e), 1, ctypes.byref(ctx))
    assert rc == 8  # PMC_ERR_NO_DEVICE


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from partmc_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()
