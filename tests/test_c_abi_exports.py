"""The shared library loads on a machine without a GPU or a CUDA driver and
exports every function include/*.h declares: each C function (the reference's
extern "C" Launch* kernels and this library's gpufhe_* C ABI) resolves by
name, and each C++ API function of namespace gpufhe appears in the dynamic
symbol table. No compute call is made."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "gpu-resident-library_b200", "gpufhe_b200", "libgpufhe_b200.so")
HEADERS = sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))

DECL = re.compile(r"^\s*(?:extern\s+\"C\"\s+)?(?:const\s+)?[A-Za-z_][\w:<>]*\s*[*&]*\s+\**\s*(\w+)\s*\(", re.M)
KEYWORDS = {"return", "if", "while", "for", "switch", "sizeof"}


def declared():
    c_names, cpp_names = set(), set()
    for h in HEADERS:
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        cpp = "namespace gpufhe" in src
        for m in DECL.finditer(src):
            name = m.group(1)
            if name in KEYWORDS:
                continue
            # skip functions defined inline in the header (body follows before any ';')
            semi, brace = src.find(";", m.end()), src.find("{", m.end())
            if brace != -1 and (semi == -1 or brace < semi):
                continue
            line = src[m.start():m.end()]
            if name.startswith(("gpufhe_", "Launch")) or 'extern "C"' in line:
                c_names.add(name)
            elif cpp:
                cpp_names.add(name)
    return sorted(c_names), sorted(cpp_names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        pytest.fail("libgpufhe_b200.so is not built (python -m gpufhe_b200.build)")
    return ctypes.CDLL(LIB)   # must load without libcuda.so.1


def test_headers_declare_the_boundary():
    c_names, cpp_names = declared()
    assert len([n for n in c_names if n.startswith("Launch")]) >= 14
    assert {"gpufhe_ctx_create", "gpufhe_plan_launch", "gpufhe_server_submit", "gpufhe_rescale_noalloc",
            "gpufhe_keygen", "gpufhe_encode_batch"} <= set(c_names)
    assert {"keyswitch_resident", "rescale_resident_raw", "ks_context_create", "keygen_host"} <= set(cpp_names)
    # the reference's headerless helpers its tests declare in place
    assert {"automorphism_eval_host", "rotate_ct_host", "pt_to_eval_host", "ct_add_ct_host",
            "ct_mul_pt_host"} <= set(cpp_names)


def test_every_c_function_resolves(lib):
    missing = []
    for name in declared()[0]:
        try:
            getattr(lib, name)
        except AttributeError:
            missing.append(name)
    assert not missing, missing


def test_every_cpp_function_exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    have = set(re.findall(r"gpufhe::(?:\w+::)*(\w+)\(", out))
    missing = [n for n in declared()[1] if n not in have]
    assert not missing, missing


def test_no_link_time_driver_dependency():
    """The library reaches the driver API only through the runtime's entry
    points, so it loads (and the CPU tests run) where no driver is installed."""
    out = subprocess.run(["readelf", "-d", LIB], capture_output=True, text=True, check=True).stdout
    assert "libcuda.so" not in out


def test_reference_globals_exported():
    """Variables the reference's test programs declare and write
    (gpufhe::g_ks_batched in tests/test_rot_resident.cpp:17) are data symbols
    of the library, so those programs link unchanged."""
    out = subprocess.run(["nm", "-DC", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    assert re.search(r"\s[BD]\s+gpufhe::g_ks_batched$", out, re.M), "gpufhe::g_ks_batched not exported"
