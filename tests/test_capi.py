"""CPU tests of the C ABI: the library builds, loads without a GPU, and
exports every function that include/*.h declares; the Python bindings cover
the same set.  No compute calls are made here."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(dage_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"dage_op3d_create", "dage_op3d_apply", "dage_integrate", "dage_last_error"} <= names


def test_library_exports_every_declared_symbol():
    from dage_b200 import build

    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_bindings_cover_header():
    from dage_b200 import _capi

    assert declared_functions() == set(_capi.SIGNATURES)


def test_abi_version_and_error_string_without_gpu():
    import dage_b200

    lib = dage_b200.load()
    assert lib.dage_abi_version() == 1
    # invalid-argument path: no CUDA call is reached before the check
    assert lib.dage_op3d_create(None, None, None, 0, None) == -1
    assert b"null" in lib.dage_last_error()
    assert lib.dage_set_wait_limit(0) == -1


def test_fortran_interface_block_binds_every_entry_point():
    """The Fortran module in INTEGRATION.md binds each C symbol the header
    declares (bind(C, name="...")), and nothing else."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = doc[doc.index("```fortran\nmodule dage_gpu_m"):]
    block = block[:block.index("end module")]
    bound = set(re.findall(r'bind\(C, name="(dage_[a-z0-9_]+)"\)', block))
    assert bound == declared_functions(), (sorted(declared_functions() - bound),
                                           sorted(bound - declared_functions()))


def test_tune_cache_path_host_only(dage_host, tmp_path):
    """dage_set_tune_cache is host logic: it creates the cache file, loads
    what is in it and refuses a path it cannot write (no GPU call)."""
    lib = dage_host.load()
    path = tmp_path / "tune.txt"
    path.write_text("dev/op3d_fp64/5x5,5x5,5x5,P2 32 64 128\n")
    assert lib.dage_set_tune_cache(str(path).encode()) == 0
    assert lib.dage_set_tune_cache(str(tmp_path).encode()) == -1  # a directory
    assert b"tune cache" in lib.dage_last_error()
    assert lib.dage_set_tune_cache(None) == 0
