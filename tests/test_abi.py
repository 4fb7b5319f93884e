"""The C ABI library loads and exports every symbol include/cupythia_b200.h declares (no compute
without a GPU), and the product fails loudly without one."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(cp_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_exports_every_declared_symbol():
    from cupythia_b200 import build
    lib_path = build.build()
    lib = C.CDLL(lib_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(declared()) >= 20


def test_python_binding_covers_the_header():
    from cupythia_b200 import _lib
    names = set(_lib.SIGNATURES) | set(_lib.OPTIONAL) | {"cp_last_error"}
    assert not [n for n in declared() if n not in names]


def test_abi_version_and_defaults_without_gpu():
    from cupythia_b200 import _lib
    lib = _lib.load()
    assert lib.cp_abi_version() == 1
    cfg = _lib.cp_config()
    assert lib.cp_config_default(C.byref(cfg)) == 0
    assert cfg.sqrt_s == 13000.0 and cfg.pt_hat_min == 20.0 and cfg.n_bins == 50 and cfg.seed == 42


def test_no_silent_cpu_path_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import cupythia_b200 as cp
    with pytest.raises(cp.CpError):
        cp.Integrator()


def test_device_event_struct_layout_matches_ctypes(tmp_path):
    """cp_device_events as a C compiler lays it out (the reference's DeviceEvents member order)
    equals the ctypes mirror the Python layer passes."""
    import ctypes as C
    import subprocess

    from cupythia_b200 import _lib
    fields = [f for f, _ in _lib.cp_device_events._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "cupythia_b200.h"\nint main(void) {\n'
                   '  printf("%zu", sizeof(cp_device_events));\n' +
                   "".join(f'  printf(" %zu", offsetof(cp_device_events, {f}));\n' for f in fields) +
                   "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_lib.cp_device_events)] + [getattr(_lib.cp_device_events, f).offset for f in fields]
    assert got == want
