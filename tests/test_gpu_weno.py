"""WENO5 (sch_weno5_3d.f90, ischema 12) beyond the flux-family tests: the
flagged non-reference fix (three weighted candidates in every direction)
against the oracle bit for bit, block by block and over fused iterations; a
block one cell deep in k, where the reference's k stencil never leaves the
block; a uniform flow kept to rounding with the fix; and the mixed form
with the fix next to the FP64 one."""
from __future__ import annotations

import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib
from tests._helpers import SMALL, assert_equal_bits, oracle_prepared, real, state_err
from tests.test_gpu_parity import _gpu, _load_state, _n, _prepared_flow

pytestmark = pytest.mark.gpu


def _weno(case, fix):
    case.scheme.ischema = 12
    case.scheme.weno_fix = fix
    return case


def _block_parity(torch, case):
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    L = orc_lib()
    ld = case.layout.ld
    ns = bool(case.scheme.ns)
    u_o = np.zeros_like(st.u)
    for l in range(1, case.layout.nblk + 1):
        L.orc_sch_weno5_3d(l, u_o, st.v, st.tau, st.sn, st.ps)
    for l in range(1, case.layout.nblk + 1):
        s.u.fill_(3.0)
        torch.cuda.synchronize()
        s.sch_weno5_3d(l, s.u, s.v, s.tau, s.sn, s.pression,
                       equat=b"ns3d   " if ns else b"eu3d   ")
        s.sync()
        sel = case.layout.blocks[l - 1].real_cells()
        assert_equal_bits(_n(s.u).reshape(-1, ld)[:5, sel], u_o.reshape(-1, ld)[:5, sel],
                          f"u block {l}")
    s.close()


def _fused_parity(case, nsteps):
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    rc = real(case)
    for it in range(nsteps):
        u0 = st.v.copy()
        orc.step(st)
        no = orc.norms(u0, st)
        ng = s.atsch_num(1)
        assert np.isfinite(no).all(), it
        assert_equal_bits(_n(s.v).reshape(5, ld)[:, rc], st.v.reshape(5, ld)[:, rc],
                          f"v after step {it}")
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0, err_msg=f"norms step {it}")
    s.close()
    return no


@pytest.mark.parametrize("name", ["box_eu_qfix", "box_ns", "channel", "box_pinfl"])
def test_block_residual_parity_with_the_fix(cuda, name):
    _block_parity(cuda, _weno(SMALL[name](), 1))


@pytest.mark.parametrize("name", ["channel", "box_ns"])
def test_fused_iterations_with_the_fix(cuda, name):
    no = _fused_parity(_weno(SMALL[name](), 1), 20)
    assert no[1, 0] < 1.0


@pytest.mark.parametrize("fix", [0, 1])
def test_one_cell_deep_in_k(cuda, fix):
    """nk - 1 = 1: no interior k face, so the reference form is defined on
    every face (its 2-D use)"""
    case = _weno(cases.box_case((12, 8, 1), seed=16, skew=0.02, alpha=2.0, qfix_dfez=1), fix)
    _block_parity(cuda, case)
    _fused_parity(_weno(cases.box_case((12, 8, 1), seed=16, skew=0.02, alpha=2.0,
                                       qfix_dfez=1), fix), 5)


def test_uniform_flow_with_the_fix(cuda):
    """with all three candidates the residual of a uniform flow on an
    unskewed box is rounding (on skewed cells the stencils that wrap into the
    edge ghosts, whose pressure no routine sets, leave ~1e-8)"""
    torch = cuda
    case = _weno(cases.box_case((10, 8, 6), noise=0.0, alpha=20.0, qfix_dfez=1), 1)
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    s.sch_weno5_3d(1, s.u, s.v, s.tau, s.sn, s.pression, equat=b"eu3d   ")
    s.sync()
    ld = case.layout.ld
    rc = real(case)
    u = _n(s.u).reshape(-1, ld)[:5, rc]
    flux = float(np.abs(st.v.reshape(5, ld)[:, rc]).max())
    assert np.abs(u).max() < 1e-12 * flux, np.abs(u).max()
    s.close()


def test_mixed_form_with_the_fix_tracks_fp64(cuda):
    """precision 1 (FP32 sweeps) with the fixed WENO5 on the duct: 400
    iterations of both forms stay finite, both residuals fall, and the
    states stay close"""
    from tests.test_gpu_mixed import _duct, _solver
    a = _solver(_weno(_duct(), 1), 0)
    b = _solver(_weno(_duct(), 1), 1)
    na0 = a.atsch_num(1)
    nb0 = b.atsch_num(1)
    na = a.atsch_num(399)
    nb = b.atsch_num(399)
    assert np.isfinite(na).all() and np.isfinite(nb).all()
    assert na[1, 0] < 0.1 * na0[1, 0] and nb[1, 0] < 0.1 * nb0[1, 0], (na0, na, nb0, nb)
    case = a.case
    ld = case.layout.ld
    rc = case.layout.real_cells()
    err = state_err(_n(b.v).reshape(5, ld)[:, rc], _n(a.v).reshape(5, ld)[:, rc])
    assert err < 1e-5, err
    a.close()
    b.close()
