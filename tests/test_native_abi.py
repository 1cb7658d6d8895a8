"""The C-ABI library loads and exports every entry point include/*.h declares (CPU only)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(zs_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "zs_m31_circle_fft" in names and "zs_m31_commit_plan_create" in names and "zs_free" in names


def test_library_exports_every_declared_symbol():
    from zs_b200 import native
    lib = native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert "sm_100a" in native.version()


def test_library_is_in_tree():
    from zs_b200 import native
    assert os.path.dirname(native.LIB_PATH).startswith(os.path.join(ROOT, "zig-stark_b200"))


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from zs_b200 import native
    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        native.lib()


def test_context_without_device_is_a_device_error():
    """On a host without a CUDA device, zs_m31_ctx_create returns -5 (no device work)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from zs_b200 import native
    with pytest.raises(native.ZsError) as e:
        native.Context(0)
    assert e.value.code == -5


def test_context_entry_points_check_arguments_first():
    """zs_m31_prove_ctx rejects a null context with -2 before touching a device,
    zs_m31_ctx_destroy(NULL) is a no-op and zs_m31_ctx_device(NULL) is -2."""
    import ctypes
    from zs_b200 import native
    L = native._bind_prove()
    L.zs_m31_prove_ctx.argtypes = [ctypes.c_void_p] + L.zs_m31_prove.argtypes
    L.zs_m31_ctx_destroy.argtypes = [ctypes.c_void_p]
    L.zs_m31_ctx_destroy.restype = None
    L.zs_m31_ctx_device.argtypes = [ctypes.c_void_p]
    out, n = ctypes.c_void_p(), ctypes.c_size_t()
    args = [native.HOST, 1] + [b"", 0] * 5
    assert L.zs_m31_prove_ctx(None, *args, ctypes.byref(out), ctypes.byref(n)) == -2
    L.zs_m31_ctx_destroy(None)
    assert L.zs_m31_ctx_device(None) == -2


def test_binius_entry_points_reject_malformed_arguments_first():
    """The sum-check entry points check their arguments before any device work and
    return -2 (so this runs without a GPU)."""
    from zs_b200 import native
    cur = bytes(16)
    bad_calls = [
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01", [0, 2], [0, 2], 2, 4),      # index >= m
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01", [0, 1], [0, 2], 2, 5),      # 2 half > len
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01", [0, 1], [0, 2], 256, 4),    # 257 points
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01\x01", [0, 1], [0, 2, 1], 2, 4),  # offsets decrease
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01", [0] * 1025, [0, 1025], 1025, 4),  # > 1024 factors
        lambda: native.binius_gf256_values(cur, 8, 2, b"\x01" * 257, [], [0] * 258, 0, 4),  # > 256 terms
        lambda: native.binius_prove_combination(8, cur, 3, 2, [([0] * 64, 1)]),             # 65 points
        lambda: native.binius_prove_combination(16, cur, 3, 2, [([0], 1)]),                 # field_bits
        lambda: native.binius_fold_device(128, 0, 8, 2, 3, 0),                               # null buffers
    ]
    for call in bad_calls:
        with pytest.raises(native.ZsError) as e:
            call()
        assert e.value.code == -2
