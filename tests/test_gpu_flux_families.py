"""GPU tests of the other flux families (HLLC, ischema 14; Rusanov,
ischema 9; AUSM+, ischema 5; WENO5, ischema 12): each block's residual
against the oracle's restatement of sch_hllc_euler / sch_hllc / sch_rusanov /
sch_ausmp / sch_weno5_3d bit for bit, and the fused iterations with each
family against the oracle's atsch_num sequence."""
from __future__ import annotations

import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib
from tests._helpers import SMALL, assert_equal_bits, max_rel_cols, oracle_prepared, real
from tests.test_gpu_parity import _gpu, _load_state, _n, _prepared_flow

pytestmark = pytest.mark.gpu

FAMILIES = {"hllc": 14, "rusanov": 9, "ausm": 5, "weno5": 12}


def with_family(case, ischema):
    case.scheme.ischema = ischema
    return case


@pytest.mark.parametrize("family", sorted(FAMILIES))
@pytest.mark.parametrize("name", ["box_eu", "box_ns", "channel", "box_pinfl"])
def test_block_residual_parity(cuda, family, name):
    torch = cuda
    if family == "ausm" and name == "box_eu":
        pytest.skip("the reference runs AUSM+ for the Navier-Stokes equations only")
    case = with_family(SMALL[name](), FAMILIES[family])
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    L = orc_lib()
    ns = bool(case.scheme.ns)
    u_o = np.zeros_like(st.u)
    for l in range(1, case.layout.nblk + 1):
        if family == "rusanov":
            L.orc_sch_rusanov(l, u_o, st.v, st.tau, st.sn, st.ps)
        elif family == "weno5":
            L.orc_sch_weno5_3d(l, u_o, st.v, st.tau, st.sn, st.ps)
        elif family == "ausm":
            L.orc_sch_ausmp(l, u_o, st.v, st.tau, st.sn, st.ps)
        elif ns:
            L.orc_sch_hllc(l, u_o, st.v, st.tau, st.sn, st.ps)
        else:
            L.orc_sch_hllc_euler(l, u_o, st.v, st.sn, st.ps)
    ld = case.layout.ld
    for l in range(1, case.layout.nblk + 1):
        s.u.fill_(7.0)
        torch.cuda.synchronize()
        if family == "rusanov":
            s.sch_rusanov(l, s.u, s.v, s.tau, s.sn, s.pression)
        elif family == "weno5":
            s.sch_weno5_3d(l, s.u, s.v, s.tau, s.sn, s.pression,
                           equat=b"ns3d   " if ns else b"eu3d   ")
        elif family == "ausm":
            s.sch_ausmp(l, s.u, s.v, s.tau, s.sn, s.pression)
        elif ns:
            s.sch_hllc(l, s.u, s.v, s.tau, s.sn, s.pression)
        else:
            s.sch_hllc_euler(l, s.u, s.v, s.sn, s.pression)
        s.sync()
        sel = case.layout.blocks[l - 1].real_cells()
        ncol = s.u.numel() // ld
        assert_equal_bits(_n(s.u).reshape(ncol, ld)[:5, sel],
                          u_o.reshape(-1, ld)[:5, sel], f"{family} u block {l}")
    s.close()


@pytest.mark.parametrize("family", sorted(FAMILIES))
@pytest.mark.parametrize("name,nsteps", [("box_ns", 5), ("channel", 5), ("box_eu_qfix", 5)])
def test_fused_steps_parity(cuda, family, name, nsteps):
    if family == "ausm" and name == "box_eu_qfix":
        pytest.skip("the reference runs AUSM+ for the Navier-Stokes equations only")
    case = with_family(SMALL[name](), FAMILIES[family])
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    rc = real(case)
    has_idd = any(b.kind == cases.BC_IDD for b in case.boundaries)
    for it in range(nsteps):
        u0 = st.v.copy()
        orc.step(st)
        no = orc.norms(u0, st)
        ng = s.atsch_num(1)
        v_g = _n(s.v).reshape(5, ld)[:, rc]
        v_o = st.v.reshape(5, ld)[:, rc]
        assert_equal_bits(v_g, v_o, f"{family} v after step {it} (injection: {has_idd})")
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0, err_msg=f"norms step {it}")
    s.close()


@pytest.mark.parametrize("family", sorted(FAMILIES))
def test_mixed_form_matches_the_fp64_converged_state(cuda, family):
    """precision 1 (FP64 residual with contraction, FP32 sweeps) with the
    other families on the duct with a unique steady state: both forms
    converge and agree within the mixed-precision tolerance"""
    if family == "weno5":
        pytest.skip("the reference WENO5 reaches no steady state (test_gpu_weno.py)")
    from tests.test_gpu_mixed import STEADY_TOL, _duct, _solver
    from tests._helpers import state_err
    a = _solver(with_family(_duct(), FAMILIES[family]), 0)
    b = _solver(with_family(_duct(), FAMILIES[family]), 1)
    na = a.atsch_num(4500)
    nb = b.atsch_num(4500)
    # AUSM+ settles near 1e-9 on this duct (FP64 and mixed alike: its
    # splitting polynomials switch at |M| = 1); the others reach rounding
    tol = 1e-8 if family == "ausm" else 1e-12
    assert na[1, 0] < tol and nb[1, 0] < tol, (na[1, 0], nb[1, 0])
    case = a.case
    ld = case.layout.ld
    rc = case.layout.real_cells()
    err = state_err(_n(b.v).reshape(5, ld)[:, rc], _n(a.v).reshape(5, ld)[:, rc])
    assert err <= STEADY_TOL, err
    a.close()
    b.close()


def test_ausm_needs_the_navier_stokes_equations(cuda):
    from codens_b200 import abi
    from codens_b200.solver import CodeNS
    case = SMALL["box_eu"]()
    s = CodeNS(case)
    sc = case.scheme
    sc.ischema = 5
    with pytest.raises(abi.CnsError) as e:
        s.set_scheme(sc)
    assert e.value.code == abi.CNS_EINVAL
    s.close()
