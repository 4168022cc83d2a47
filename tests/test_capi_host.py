"""The C-ABI library on the CPU: it loads, exports every declared symbol, its structure
layouts match the C header, and its host helpers agree with the oracle and NumPy.
No GPU is needed for these tests."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import philox as PX
from thruster_cx_code_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pbemcs.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.PROTOTYPES, f"{n} has no ctypes prototype"
    assert lib.pb_version() >= 10000


def test_struct_layout_matches_header(tmp_path):
    fields_p = [f for f, _ in _lib.StepParams._fields_]
    fields_r = [f for f, _ in _lib.StepReport._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "pbemcs.h"', 'int main(void){',
           'printf("%zu %zu\\n", sizeof(pb_step_params), sizeof(pb_step_report));']
    for f in fields_p:
        src.append(f'printf("P {f} %zu\\n", offsetof(pb_step_params, {f}));')
    for f in fields_r:
        src.append(f'printf("R {f} %zu\\n", offsetof(pb_step_report, {f}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sp, sr = map(int, out[0].split())
    assert sp == C.sizeof(_lib.StepParams) and sr == C.sizeof(_lib.StepReport)
    for line in out[1:]:
        if not line:
            continue
        kind, name, off = line.split()
        cls = _lib.StepParams if kind == "P" else _lib.StepReport
        assert getattr(cls, name).offset == int(off), name


def _add_at(s, c, n):
    r = np.array([s], dtype=np.float32)
    np.add.at(r, np.zeros(n, dtype=np.int64), c)
    return r[0]


def test_seq_add_matches_np_add_at():
    """The run-length sum equals np.add.at on a float32 array with a Python-float value
    (float64 partial sums rounded to float32 each time), including hot cells, both
    signs, zero crossings and the ion-then-electron sequence of a deposit."""
    lib = _lib.load()
    rs = np.random.RandomState(0)
    cases = [(0.0, 0.00025568755727881564, 20000), (0.0, -0.00025568755727881564, 7000),
             (0.5, -0.0200250, 2000), (0.0, 3.3e-3, 20000), (1e-3, 1e-7, 10000), (-2.0, 0.07, 500),
             (0.0, 0.1, 100000)]
    for _ in range(200):
        s0 = float(np.float32(rs.choice([0.0, rs.uniform(-10, 10)])))
        c = float(rs.uniform(-1, 1) * 10.0 ** rs.randint(-6, 3))
        cases.append((s0, c, int(rs.randint(1, 5000))))
    for s0, c, n in cases:
        exp = _add_at(s0, c, n)
        got = np.float32(lib.pb_host_seq_add_f32d(s0, c, n))
        assert got.view(np.uint32) == exp.view(np.uint32), (s0, c, n, got, exp)
    # deposit sequence: k ions then m electrons into one cell
    cd = 0.00025568755727881564
    for k, m in [(5, 5), (7, 3), (100, 100), (3, 9), (20000, 7000), (1, 0), (0, 4)]:
        r = np.zeros(1, np.float32)
        np.add.at(r, np.zeros(k, np.int64), cd)
        np.add.at(r, np.zeros(m, np.int64), -cd)
        got = np.float32(lib.pb_host_seq_add_f32d(float(lib.pb_host_seq_add_f32d(0.0, cd, k)), -cd, m))
        assert got.view(np.uint32) == r[0].view(np.uint32), (k, m, got, r[0])


def test_host_philox_matches_oracle():
    lib = _lib.load()
    ids = np.array([0, 1, 7, 123456, 2 ** 32 - 1], dtype=np.uint64)
    for site in (PX.SITE_CEX_U, PX.SITE_ION_V, PX.SITE_CEX_FM):
        u = PX.uniforms(12345, ids, site, 77, 9)
        for k, pid in enumerate(ids):
            for j in range(9):
                assert lib.pb_host_philox_uniform(12345, int(pid), site, 77, j) == u[j, k]
        g = PX.normals(12345, ids, site, 77, 3)
        for k, pid in enumerate(ids):
            for j in range(3):
                assert lib.pb_host_philox_normal(12345, int(pid), site, 77, j) == g[j, k]


def test_host_percentile_matches_numpy():
    lib = _lib.load()
    rs = np.random.RandomState(3)
    for _ in range(400):
        n = int(rs.randint(6, 5000))
        a = np.sort((rs.rand(n) * 40).astype(np.float32))
        got = np.float32(lib.pb_host_percentile95(a.ctypes.data_as(C.c_void_p), n))
        assert got == np.float32(np.percentile(a, 95)), n


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()
