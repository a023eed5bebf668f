"""C-ABI checks that need no GPU: exported symbols, struct layouts, host helpers."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ermod_b200.h")
HEADERS = sorted(os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))
                 if h.endswith(".h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(ermod_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_and_ctypes_agree():
    assert set(declared_functions()) == set(A.SIGNATURES)


def test_library_exports_every_declared_symbol(engine_lib):
    for name in declared_functions():
        assert hasattr(engine_lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", A.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (ermod_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    structs = {"ermod_params": A.ErmodParams, "ermod_topology": A.ErmodTopology, "ermod_mesh": A.ErmodMesh,
               "ermod_hist": A.ErmodHist, "ermod_accum": A.ErmodAccum, "ermod_store_info": A.ErmodStoreInfo}
    io_header = os.path.join(ROOT, "include", "ermod_io.h")
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', f'#include "{io_header}"',
             "int main(void){"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, f"{cname}.{fname}"


@pytest.mark.parametrize("hist", [{}, dict(ecdmin=-80.0), dict(pecore=0), dict(ecdmin=-200.0, ecfmns=-0.5)])
def test_library_mesh_matches_oracle(engine_lib, oracle_mod, hist):
    from ermod_openacc_b200 import enginit_mesh
    for numslv in (1, 2):
        a = enginit_mesh(hist, numslv)
        b = oracle_mod.enginit_mesh(S.hist_struct(hist), numslv)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_mesh_rejects_bad_hist(engine_lib):
    from ermod_openacc_b200 import ErmodError, enginit_mesh
    with pytest.raises(ErmodError):
        enginit_mesh(dict(ecfmns=-20.0, ecdmin=-0.1), 1)   # region narrower than its bin: eng_ecd
