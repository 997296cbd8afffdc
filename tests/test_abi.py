"""The C-ABI library loads, exports every declared symbol, and its structs match ctypes (CPU only)."""

from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from torchls_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "torchls_b200.h")

STRUCTS = {
    "tls_var_group": L.VarGroup,
    "tls_factor_group": L.FactorGroup,
    "tls_segments": L.Segments,
    "tls_linearize_args": L.LinearizeArgs,
    "tls_normal_tiles": L.NormalTiles,
    "tls_normal_args": L.NormalArgs,
    "tls_block_group": L.BlockGroup,
    "tls_pcg_control": L.PcgControl,
    "tls_schur_args": L.SchurArgs,
    "tls_pcg_args": L.PcgArgs,
    "tls_schur_general_args": L.SchurGeneralArgs,
    "tls_fixed_system": L.FixedSystem,
    "tls_retained_matrix": L.RetainedMatrix,
}


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^TLS_API\s+(?:int|int64_t|const char\*)\s+(tls_\w+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(L._SIGNATURES), set(names) ^ set(L._SIGNATURES)
    assert lib.tls_version() == 1


def test_struct_layouts_match_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof(struct {cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof(struct {cname}, {fname}));')
    lines.append("  return 0; }")
    with tempfile.TemporaryDirectory() as tmp:
        src, exe = os.path.join(tmp, "layout.c"), os.path.join(tmp, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            cname, field, value = line.split()
            got[(cname, field)] = int(value)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_pcg_state_fits_control_struct():
    assert L.lib().tls_pcg_state_bytes() >= ctypes.sizeof(L.PcgControl)


def test_errors_map_to_python_exceptions():
    lib = L.lib()
    seg = L.Segments(4, 3, 3, 0, None, None)  # lanes must be a power of two or 256
    status = lib.tls_segment_reduce(ctypes.byref(seg), None, L.F64, 0, 3, None, L.F64, None)
    assert status == L.TLS_ERR_INVALID
    with pytest.raises(ValueError, match="lanes"):
        L.check(status)
