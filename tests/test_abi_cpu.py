"""The C-ABI library loads and exports every symbol include/bbkde.h declares.
No compute calls: this runs without a GPU."""
from __future__ import annotations

import ctypes as C
import glob
import os
import re
import subprocess

import pytest

import bbrcit_kde_b200 as bk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", "bbkde.h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        names |= set(re.findall(r"BBKDE_API\s+[\w\s\*]*?\b(bbkde_\w+)\s*\(", text))
    return names


def test_header_declares_what_bindings_expect():
    assert declared_symbols() == set(bk.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = bk.load_library()
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", bk.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(bbkde_\w+)", out))
    assert declared_symbols() <= exported
    # Nothing but the ABI leaks out of the library.
    assert all(s.startswith("bbkde_") for s in re.findall(r"\sT\s+(\w+)", out)), out


def test_abi_version_and_status_strings():
    lib = bk.load_library()
    assert lib.bbkde_abi_version() == 2
    assert lib.bbkde_status_string(bk.OUT_OF_RANGE) == b"out of range"
    assert lib.bbkde_status_string(bk.INVALID_ARGUMENT) == b"invalid argument"
    assert lib.bbkde_status_string(99) == b"unknown status"


def test_null_context_is_rejected():
    lib = bk.load_library()
    assert lib.bbkde_size(None, bk.REFERENCE) == -1
    assert lib.bbkde_last_launch_stats(None, None, None, None) == bk.INVALID_ARGUMENT
    assert lib.bbkde_ctx_destroy(None) == bk.OK
    assert lib.bbkde_ctx_create(0, None) == bk.INVALID_ARGUMENT


def test_kernel_desc_layout_matches_header():
    # int32 kind, int32 dim, double h[2], int32 flags, int32 reserved
    assert C.sizeof(bk.KernelDesc) == 32
    assert bk.KernelDesc.h.offset == 8


@pytest.mark.skipif(bool(glob.glob("/dev/nvidia[0-9]*")), reason="a GPU is present")
def test_ctx_create_without_device_reports_no_device():
    lib = bk.load_library()
    h = C.c_void_p()
    assert lib.bbkde_ctx_create(0, C.byref(h)) == bk.NO_DEVICE
    assert not h.value


# Every ctypes mirror of a C struct of the header, by C name.
MIRRORS = {"bbkde_kernel_desc": bk.KernelDesc, "bbkde_dataset": bk.Dataset,
           "bbkde_train_config": bk.TrainConfig, "bbkde_cull_stats": bk.CullStats,
           "bbkde_grid": bk.Grid, "bbkde_grid_config": bk.GridConfig,
           "bbkde_grid_stats": bk.GridStats}


def test_struct_layouts_match_header(tmp_path):
    """The Python mirrors have the C structs' sizes and field offsets, as gcc lays
    them out from include/bbkde.h (a field added on one side only shifts the
    others and silently corrupts every call that passes the struct)."""
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "bbkde.h"',
             'int main(void) {']
    for cname, py in MIRRORS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src),
                           "-o", str(exe)])
    got = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        cname, key, value = line.split()
        got[(cname, key)] = int(value)
    for cname, py in MIRRORS.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
