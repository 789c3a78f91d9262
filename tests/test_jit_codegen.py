"""The runtime-specialized kernels compile for sm_100a (CPU: no GPU is needed to compile).

tests/jit_codegen_probe.cpp asks the library for the sources it generates for the filter,
cardinality-scan and aggregate kernels (strided and consecutive-row tiles, per-thread
accumulators, direct group slots and speculative loads, a semi-join probe, GROUP BY the dense
join key); each is compiled here with NVRTC, with the device headers the library embeds, the
way ml_jit.cpp does.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "minilake_b200", "csrc")
LIBDIR = os.path.join(ROOT, "minilake_b200", "_lib")
HEADERS = ["ml_internal.hpp", "ml_args.hpp", "ml_device.cuh", "ml_agg.cuh"]


def _nvrtc():
    try:
        from cuda.bindings import nvrtc
    except ImportError:
        pytest.skip("cuda-python (NVRTC bindings) not installed")
    return nvrtc


def _header_set():
    """(names, texts) of the headers a generated source includes, as the library embeds them."""
    names, texts = [], []
    for h in HEADERS:
        names.append(h.encode())
        texts.append(open(os.path.join(CSRC, h)).read().encode())
    pub = open(os.path.join(ROOT, "include", "minilake_gpu.h")).read()  # enums only
    names.append(b"../../include/minilake_gpu.h")
    texts.append(("#pragma once\n" + "\n".join(re.findall(r"enum\s*\{.*?\};", pub, re.S)) + "\n").encode())
    jit = open(os.path.join(CSRC, "ml_jit.cpp")).read()
    for var, name in (("kStdint", b"stdint.h"), ("kStddef", b"stddef.h")):
        m = re.search(r"const char " + var + r"\[\] =(.*?);\n", jit, re.S)
        names.append(name)
        texts.append(eval("(" + m.group(1) + ")").encode())  # the C string literal(s) of the source
    return names, texts


def _generated_sources(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    lib = os.path.join(LIBDIR, "libminilake_gpu.so")
    assert os.path.exists(lib), "build the library first (__graft_entry__.build())"
    exe = str(tmp_path / "jit_codegen_probe")
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["g++", "-std=c++17", "-O0", "-I", CSRC, "-I", cuda_inc,
                    os.path.join(ROOT, "tests", "jit_codegen_probe.cpp"), "-L", LIBDIR, "-lminilake_gpu",
                    "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    parts = re.split(r"^//@@ (\S+)\n", out, flags=re.M)
    return dict(zip(parts[1::2], parts[2::2]))


def test_specialized_kernels_compile_for_sm_100a(tmp_path):
    nvrtc = _nvrtc()
    sources = _generated_sources(tmp_path)
    assert len(sources) == 10, sorted(sources)
    names, texts = _header_set()
    opts = [b"--gpu-architecture=sm_100a", b"-std=c++17", b"--fmad=false"]
    failed = {}
    for name, src in sources.items():
        err, prog = nvrtc.nvrtcCreateProgram(src.encode(), name.encode() + b".cu", len(names), texts, names)
        assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
        (res,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        if res != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            _, n = nvrtc.nvrtcGetProgramLogSize(prog)
            log = b" " * n
            nvrtc.nvrtcGetProgramLog(prog, log)
            failed[name] = log.decode()[:2000]
        nvrtc.nvrtcDestroyProgram(prog)
    assert not failed, failed
    # the layouts differ where they should
    assert "ld_stream_v4_u32" in sources["select_contig"] and "__ballot_sync" in sources["select_strided"]
    assert "dense_member" in sources["aggregate_semi_join_contig"]
    assert "dense_slot" in sources["aggregate_dense_groups_contig"]
    assert "dsl[dsg]" in sources["aggregate_groups_contig"]
    # per-thread accumulators after a filter: speculative loads in the consecutive-row form only
    assert "specd" in sources["aggregate_groups_contig"] and "specd" not in sources["aggregate_groups_strided"]
    assert "specd" not in sources["aggregate_dense_groups_contig"]
