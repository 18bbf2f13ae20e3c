"""CPU-side checks of the C ABI boundary: the product library builds, loads,
and exports every function include/zoda_b200.h declares (no GPU calls)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "zoda_b200.h")
PKG = os.path.join(ROOT, "zoda-cu_b200")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


def test_header_declares_reference_ffi():
    fns = header_functions()
    # src/ntt/cuda.rs:15-22 binds these four from the CUDA library
    for name in ("cuda_ntt", "cuda_intt", "cuda_host_alloc", "cuda_host_free"):
        assert name in fns


def test_library_exports_every_header_function():
    import zoda_b200
    lib = zoda_b200.load()
    out = subprocess.run(["nm", "-D", "--defined-only", zoda_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    for name in header_functions():
        assert name in exported, f"{name} declared in zoda_b200.h but not exported"
        assert hasattr(lib, name)
    assert set(zoda_b200.EXPORTS) <= set(header_functions())


def test_static_archive_has_reference_symbols():
    # the reference's build.rs links `static=ntt_cuda`; the archive must carry its symbols
    path = os.path.join(PKG, "libntt_cuda.a")
    out = subprocess.run(["nm", "--defined-only", path], capture_output=True, text=True).stdout
    for name in ("cuda_ntt", "cuda_intt", "cuda_host_alloc", "cuda_host_free"):
        assert re.search(rf"\bT {name}$", out, flags=re.M), name


def test_status_strings_without_gpu():
    import zoda_b200
    lib = zoda_b200.load()
    assert lib.zoda_status_string(0) == b"ok"
    assert lib.zoda_status_string(4) == b"unsupported shape"
    assert lib.zoda_max_side() == 1 << 26  # sides above 4096 run the three-pass long-column path
