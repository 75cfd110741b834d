"""C ABI checks that need no GPU: the library loads, exports every function declared in
include/imcb200.h, the ctypes mirrors match the header, and host-only entry points work."""
import ctypes
import re
import pathlib

import numpy as np

from radtranbook_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parents[1]


def header_functions():
    txt = (ROOT / "include" / "imcb200.h").read_text()
    return re.findall(r"IMC_API\s+[\w\s\*]+?\b(imc_\w+)\s*\(", txt)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_status_strings_and_workspace_size_without_gpu():
    lib = _lib.load()
    assert lib.imc_status_str(0) == b"ok"
    assert b"capacity" in lib.imc_status_str(1)
    e = np.linspace(0, 1, 11)
    v = np.ones(10)
    m = _lib.ImcMesh(0, 10, 1, 1, e.ctypes.data, e.ctypes.data, v.ctypes.data, None)
    small = lib.imc_workspace_bytes(ctypes.byref(m), 1000)
    big = lib.imc_workspace_bytes(ctypes.byref(m), 1_000_000)
    assert small > 0 and big > small and big % 256 == 0


def test_struct_layout_matches_header(tmp_path):
    """Compile a C probe of include/imcb200.h and compare every field offset with ctypes."""
    import shutil
    import subprocess

    import pytest

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"imc_mesh": _lib.ImcMesh, "imc_bank": _lib.ImcBank, "imc_material": _lib.ImcMaterial,
               "imc_step_params": _lib.ImcStepParams, "imc_tallies": _lib.ImcTallies,
               "imc_step_report": _lib.ImcStepReport, "imc_comb_report": _lib.ImcCombReport,
               "imc_step_summary": _lib.ImcStepSummary, "imc_batch": _lib.ImcBatch,
               "imc_batch_state": _lib.ImcBatchState, "imc_batch_launch": _lib.ImcBatchLaunch,
               "imc_material_law": _lib.ImcMaterialLaw}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT}/include/imcb200.h"', "int main(){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} __sizeof__ %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "__sizeof__")] == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)
