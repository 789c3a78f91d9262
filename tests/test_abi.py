"""The C-ABI library loads and exports every entry point include/*.h declares (CPU:
no compute calls)."""
import ctypes
import glob
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "minilake_b200", "_lib", "libminilake_gpu.so")


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^(?:int|const char\*)\s+(ml_gpu_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(LIB)
    names = declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT " + n + r"$", out, re.M), n


def test_python_binding_loads_the_library():
    from minilake_b200 import gpu
    assert gpu.LIB._name == LIB


def test_build_targets_sm_100a():
    mk = open(os.path.join(ROOT, "minilake_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_context_rejects_unknown_flags():
    """Flag bits the library does not implement are refused before any device is touched."""
    from minilake_b200 import abi
    lib = ctypes.CDLL(LIB)
    out = ctypes.c_void_p()
    rc = lib.ml_gpu_ctx_create(0, ctypes.c_uint64(0), ctypes.c_uint32(1), ctypes.byref(out))
    assert rc == abi.ERR_INVALID and not out.value
    lib.ml_gpu_last_error.restype = ctypes.c_char_p
    assert b"unknown context flags" in lib.ml_gpu_last_error()


def test_rust_binding_declares_every_entry_point():
    """INTEGRATION.md's Rust `ffi.rs` block declares each function include/*.h declares."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    rust = set(re.findall(r"pub fn (ml_gpu_\w+)\(", text))
    missing = [n for n in declared() if n not in rust]
    assert not missing, missing
