"""The C ABI without a GPU: the library loads, exports every entry point include/tgh.h
declares, and the ctypes mirror matches the C layout of every struct."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "tgh.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tgh_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point(tgh):
    lib = ctypes.CDLL(str(tgh._abi.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(tgh._abi.SIGNATURES), "the ctypes signature table must cover the header"


def test_library_loads_through_the_package(tgh):
    lib = tgh.load_library()
    assert lib.tgh_state_length is not None


def test_struct_layouts_match_the_c_compiler(tgh, tmp_path):
    abi = tgh._abi
    fields = {"tgh_config": (abi.Config, [f[0] for f in abi.Config._fields_]),
              "tgh_background": (abi.Background, [f[0] for f in abi.Background._fields_]),
              "tgh_mesh": (abi.Mesh, [f[0] for f in abi.Mesh._fields_])}
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, (_, names) in fields.items():
        src.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for n in names:
            src.append(f'printf("{cname} {n} %zu\\n", offsetof({cname}, {n}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            s, f, v = line.split()
            got[(s, f)] = int(v)
    for cname, (cls, names) in fields.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for n in names:
            assert got[(cname, n)] == getattr(cls, n).offset, (cname, n)


def test_missing_library_fails_loudly(tgh, tmp_path):
    with pytest.raises(RuntimeError, match="missing"):
        tgh._abi.load_library(tmp_path / "nope.so")


def test_config_builders(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, v=0.1, gauge="algebraic").config(4)
    assert c.bg.kind == tgh._abi.BG_KERR_SCHILD and c.bg.boost[0] == -0.1
    assert c.int_v[0] == 0.1 and c.interior == tgh._abi.INT_DAMPED and c.rho_max == 4.0
    with pytest.raises(ValueError):
        tgh.kerr_schild_case(v=0.1, gauge="sampled")


def test_forests(tgh):
    c = tgh.kerr_schild_case(M=1.0, a=0.7, halfwidth=8.0)
    f = tgh.gh_forest(c, 32, 4)
    assert f.nblocks == 64 and f.h0 == 0.125 and f.points() == 64 * 32 ** 3
    hf = tgh.hole_forest(c, 8, 2, radii=(3.0, 1.5))
    assert hf.nlevels == 3
    # 2:1 balance across faces, edges and corners
    N = hf.N
    boxes = []
    for l, cn in zip(hf.level, hf.corner):
        s = 2 ** (hf.nlevels - 1 - int(l))
        lo = [int(v) * s for v in cn]
        boxes.append((int(l), lo, [v + N * s for v in lo]))
    for (l1, lo1, hi1) in boxes:
        for (l2, lo2, hi2) in boxes:
            touch = all(lo1[d] <= hi2[d] and lo2[d] <= hi1[d] for d in range(3))
            if touch:
                assert abs(l1 - l2) <= 1


def test_noalloc_speed_refuses_bad_meshes_before_touching_the_gpu(tgh):
    """tgh_max_speed_noalloc makes tgh_problem_create's checks on the block table (null tables,
    N < 1, levels out of range, corners off the block lattice) before any CUDA call, so its
    refusals are TGH_ERR_ARG with a message even where no GPU is present."""
    lib = tgh.load_library()
    c = tgh.minkowski_case(L=1.0)
    f = tgh.gh_forest(c, 8, 2)
    cfg = c.config(4)
    err = ctypes.create_string_buffer(256)
    lam = ctypes.c_double()
    dummy = ctypes.c_void_p(1)  # never dereferenced: every case is refused first

    def call(mesh):
        return lib.tgh_max_speed_noalloc(ctypes.byref(cfg), ctypes.byref(mesh), dummy, 0.0, None,
                                         ctypes.byref(lam), err, 256)

    m = f.mesh()
    m.level = ctypes.POINTER(ctypes.c_int32)()
    assert call(m) == tgh._abi.TGH_ERR_ARG and b"must not be null" in err.value
    m = f.mesh()
    m.N = 0
    assert call(m) == tgh._abi.TGH_ERR_ARG and b"at least 1" in err.value
    lev = (ctypes.c_int32 * f.nblocks)(*([25] * f.nblocks))
    m = f.mesh()
    m.level = ctypes.cast(lev, ctypes.POINTER(ctypes.c_int32))
    assert call(m) == tgh._abi.TGH_ERR_ARG and b"out of range" in err.value
    cor = (ctypes.c_int32 * (3 * f.nblocks))(*([3] * (3 * f.nblocks)))
    m = f.mesh()
    m.corner = ctypes.cast(cor, ctypes.POINTER(ctypes.c_int32))
    assert call(m) == tgh._abi.TGH_ERR_ARG and b"multiple of N" in err.value
