"""A plain C host over the C-ABI, with no Python in the engine's call path.

tests/c_host/erdst_host.c replays trjmain's division (erdst/enganal.F90:54-106):
enginit's mesh, create, engclear, engconst for each frame, engstore.  It is
compiled and linked against libermod_b200.so here; on a GPU its normalised
distribution and avediv must equal the ctypes host's on the same frames bit for
bit (the engine is deterministic).
"""
import os
import subprocess

import numpy as np
import pytest

from ermod_openacc_b200 import Engine
from ermod_openacc_b200 import _capi as A
from ermod_openacc_b200 import systems as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_host", "erdst_host.c")


def build_host(tmp_path):
    exe = tmp_path / "erdst_host"
    libdir = os.path.dirname(A.LIB_PATH)
    subprocess.run(["gcc", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-o", str(exe), SRC,
                    "-L", libdir, "-lermod_b200", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def write_input(path, w, params, nframes, device=0):
    t = w.topo
    ps = S.params_struct(params)
    hs = S.hist_struct(w.hist)
    frames = [w.frame(i) for i in range(nframes)]
    natp = len(frames[0][0]) // 3
    nsite = 0 if t.bfcoord is None else len(t.bfcoord) // 3
    with open(path, "wb") as f:
        np.array([t.nummol, len(t.charge), t.ljtype_max, nsite, natp, nframes, t.numslv, device],
                 dtype=np.int32).tofile(f)
        for a in (t.numsite, t.sluvid, t.uvspec):
            A.as_i32(a).tofile(f)
        A.as_f32(t.charge).tofile(f)
        A.as_i32(t.ljtype).tofile(f)
        A.as_f32(t.sitemass).tofile(f)
        A.as_f32(t.ljene_mat).tofile(f)
        A.as_f32(t.ljlensq_mat).tofile(f)
        if nsite:
            A.as_f32(t.bfcoord).tofile(f)
        f.write(bytes(ps))
        f.write(bytes(hs))
        for pos, cell in frames:
            A.as_f32(pos).tofile(f)
            A.as_f32(cell).tofile(f)
    return frames


def read_output(path):
    with open(path, "rb") as f:
        st = np.fromfile(f, dtype=np.int32, count=8)
        ermax = int(np.fromfile(f, dtype=np.int32, count=1)[0])
        edens = np.fromfile(f, dtype=np.float64, count=ermax)
        rest = np.fromfile(f, dtype=np.float64, count=5)
    return st, edens, rest[:2], rest[2], rest[3], rest[4]


def test_c_host_compiles_and_links(engine_lib, tmp_path):
    exe = build_host(tmp_path)
    out = subprocess.run(["nm", "-u", str(exe)], capture_output=True, text=True).stdout
    for name in ("ermod_enginit_mesh", "ermod_create", "ermod_engclear", "ermod_engconst", "ermod_engstore"):
        assert name in out


@pytest.mark.gpu
def test_c_host_matches_python_host(engine_lib, tmp_path):
    w = S.make_workload(2, small=True, maxins=96)
    prm = dict(w.params)
    exe = build_host(tmp_path)
    frames = write_input(tmp_path / "in.bin", w, prm, nframes=2)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    st, edens, avediv, engnorm, engsmpl, voffset = read_output(tmp_path / "out.bin")
    assert np.all(st[:3] == 0) and st[3] >= 0 and st[4] == 0
    eng = Engine(prm, w.topo, w.hist)
    eng.engclear()
    for i, (pos, cell) in enumerate(frames):
        assert eng.engconst(i + 1, pos, cell) >= 0
    norm, av = eng.engstore()
    np.testing.assert_array_equal(edens, norm["edens"])
    np.testing.assert_array_equal(avediv, av)
    assert engnorm == norm["engnorm"] and engsmpl == norm["engsmpl"] == 2 * eng.maxdst
    assert voffset == norm["voffset"]
    assert edens.sum() == pytest.approx(eng.slvmax, rel=1e-12)
