"""The C ABI without a GPU: the library loads, exports every function include/gral_prog.h
declares, and the ctypes mirrors in gral_b200.abi have the header's struct layout (sizes and field
offsets, checked against a C probe compiled with gcc from the header)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from gral_b200 import abi
from gral_b200 import build as B
from gral_b200.prognostic import EXPORTS, lib

HEADER = os.path.join(B.ROOT, "include", "gral_prog.h")
STRUCTS = {"gral_params": abi.GralParams, "gral_static": abi.GralStatic, "gral_fields": abi.GralFields,
           "gral_stats": abi.GralStats}


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gral_prog_\w+)\s*\(", text)))


def test_header_declares_the_python_export_list():
    assert declared_functions() == sorted(EXPORTS)


def test_library_exports_every_declared_function():
    L = lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", B.LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gral_prog_\w+)", out))
    assert set(declared_functions()) <= exported


def test_version():
    assert lib().gral_prog_version() == abi.ABI_VERSION


def test_status_codes_match_header():
    text = open(HEADER).read()
    for name, value in re.findall(r"#define (GRAL_E\w+|GRAL_OK)\s+\(?(-?\d+)\)?", text):
        assert getattr(abi, name) == int(value), name
    assert int(re.search(r"#define GRAL_NOALLOC_MAX_ROWS (\d+)", text).group(1)) == abi.GRAL_NOALLOC_MAX_ROWS
    assert int(re.search(r"#define GRAL_MAX_HISTORY (\d+)", text).group(1)) == abi.MAX_HISTORY


def test_struct_layout_matches_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gral_prog.h"', "int main(void) {"]
    for sname, cls in STRUCTS.items():
        lines.append(f'printf("{sname} size %zu\\n", sizeof({sname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{sname} {fname} %zu\\n", offsetof({sname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for sname, cls in STRUCTS.items():
        assert got[(sname, "size")] == C.sizeof(cls), sname
        for fname, _ in cls._fields_:
            assert got[(sname, fname)] == getattr(cls, fname).offset, (sname, fname)


def test_noalloc_entry_rejects_before_touching_a_device():
    """Argument checks of the allocation-free entry point run before any CUDA call."""
    L = lib()
    counts = (C.c_int32 * 4)()
    n = abi.GRAL_NOALLOC_MAX_ROWS + 1
    assert L.gral_prog_check_speeds_noalloc(n, 8, 8, 4, 1.0, 1, 1, 1, 1, 1, counts, None) == abi.GRAL_ETOOLARGE
    assert L.gral_prog_check_speeds_noalloc(8, 8, 8, 4, 1.0, 1, 1, 1, 1, 1, None, None) == abi.GRAL_EINVAL
    assert L.gral_prog_check_speeds_noalloc(8, 8, 8, 4, 1.0, None, 1, 1, 1, 1, counts, None) == abi.GRAL_EINVAL


def test_create_without_gpu_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    L = lib()
    ctx = C.c_void_p()
    rc = L.gral_prog_create(16, 14, 63, 20, 1, C.byref(ctx))
    assert rc == abi.GRAL_ENODEV
    assert not ctx.value


def test_params_mirror_rejects_missing_keys():
    with pytest.raises(KeyError):
        abi.params_to_c({"nii": 4})


def test_phase_names_match_header():
    from gral_b200.prognostic import PHASES
    text = open(HEADER).read()
    n = int(re.search(r"#define GRAL_NUM_PHASES (\d+)", text).group(1))
    assert len(PHASES) == n
    ids = {int(v): k for k, v in re.findall(r"#define GRAL_PHASE_(\w+) (\d+)", text)}
    assert sorted(ids) == list(range(n))


def test_batch_devices_argument_checks_need_no_gpu():
    """gral_prog_solve_batch_devices rejects an empty device list and fewer situations than
    devices before touching a device."""
    L = lib()
    dv = (C.c_int32 * 2)(0, 0)
    p = (abi.GralParams * 1)()
    s = abi.GralStatic()
    f = (abi.GralFields * 1)()
    assert L.gral_prog_solve_batch_devices(0, dv, 1, p, C.byref(s), f, None) == abi.GRAL_EINVAL
    assert L.gral_prog_solve_batch_devices(2, dv, 1, p, C.byref(s), f, None) == abi.GRAL_EINVAL
    assert L.gral_prog_solve_batch_devices(1, None, 1, p, C.byref(s), f, None) == abi.GRAL_EINVAL

