"""The C ABI from a compiled C program (tests/c_driver/cns_driver.c, gcc +
libcodens_b200.so, no Python in the process): it builds and links here; on a
GPU it runs zpres, rbord and sch_roe_euler on plain host arrays (the
copy-in/out mode, sn passed as the block's slice as the reference does) and
three fused iterations through cns_atsch_num_step_host, and its outputs equal
the oracle's bit for bit."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from codens_b200 import build as cuda_build, cases

from ._helpers import assert_equal_bits, oracle_prepared, real

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "c_driver", "cns_driver.c")
EXE = os.path.join(HERE, "c_driver", "_build", "cns_driver")
CUDA = "/usr/local/cuda"


def build_driver() -> str:
    lib = cuda_build.build()
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    libdir = os.path.dirname(lib)
    cmd = ["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(CUDA, "include"), SRC, "-o", EXE,
           "-L" + libdir, "-lcodens_b200", "-Wl,-rpath," + libdir,
           "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return EXE


def write_case(case, path):
    lay = case.layout
    ba = case.boundary_arrays()
    sc, p = case.scheme, case.phys
    scheme = [sc.ns, sc.muscl, sc.xk, sc.ilim, sc.eta, sc.kdtl, sc.dt1min, sc.lmax,
              sc.qfix_dfez, sc.precision, sc.kdefect, sc.ischema, sc.ki2, sc.ki4, sc.ncychro,
              sc.icychr0, sc.kfmg, sc.kdualns]
    with open(path, "wb") as f:
        np.array([lay.nblk, lay.ld, len(ba["type"]), len(ba["ncbd"])], np.int64).tofile(f)
        np.asarray(lay.dims_array(), np.int32).tofile(f)
        np.array([p.gam, p.pinfl, p.pr, p.prt, p.reynz, p.suth_a, p.pa1, p.aa1, p.omg],
                 np.float64).tofile(f)
        np.array(scheme, np.float64).tofile(f)
        for k, t in (("type", np.int32), ("blk", np.int32), ("face", np.int32),
                     ("mpb", np.int64), ("mmb", np.int32), ("partner", np.int32),
                     ("cosr", np.float64), ("sinr", np.float64), ("ncbd", np.int64),
                     ("ncin", np.int64)):
            np.asarray(ba[k], t).tofile(f)
        np.asarray(ba["bceqt"], np.float64).reshape(-1).tofile(f)
        for a in (case.x, case.y, case.z):
            np.asarray(a, np.float64).tofile(f)
        np.asarray(case.v0, np.float64).reshape(-1).tofile(f)


def test_driver_builds_and_links():
    exe = build_driver()
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_driver_matches_the_oracle(cuda, tmp_path):
    from oracle.oracle import lib as orc_lib
    exe = build_driver()
    # an Euler box with the flagged implimf_eu fix (the reference form turns
    # non-finite on noisy 3-D boxes), one block at offset 0
    case = cases.box_case((12, 7, 6), seed=16, skew=0.02, alpha=2.0, qfix_dfez=1)
    cpath, opath = tmp_path / "case.bin", tmp_path / "out.bin"
    write_case(case, cpath)
    r = subprocess.run([exe, str(cpath), str(opath)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    ld = case.layout.ld
    out = np.fromfile(opath, np.float64)
    u_c, v_c, norms_c = out[:5 * ld], out[5 * ld:10 * ld], out[10 * ld:].reshape(3, 5)
    rc = real(case)
    # the oracle: zpres, rbord, sch_roe_euler of block 1 on the initial state
    orc, st = oracle_prepared(case)
    L = orc_lib()
    L.orc_zpres(1, st.v, st.ps, st.temp, st.cson)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    u_o = np.zeros_like(st.u)
    L.orc_sch_roe_euler(1, u_o, st.v, st.sn, st.ps)
    assert_equal_bits(u_c.reshape(5, ld)[:, rc], u_o.reshape(5, ld)[:, rc], "sch_roe_euler u")
    # three fused iterations from the initial state
    orc, st = oracle_prepared(case)
    for _ in range(3):
        u0 = st.v.copy()
        orc.step(st)
        no = orc.norms(u0, st)
    assert_equal_bits(v_c.reshape(5, ld)[:, rc], st.v.reshape(5, ld)[:, rc], "v after 3 steps")
    np.testing.assert_allclose(norms_c, no, rtol=1e-12, atol=0)
