"""GPU parity of the Jameson scheme (ischema = 1) against the oracle, through
the C ABI: the ghost refresh before the dissipation (rfve, rfvc), the scalar
dissipation (dissip_jameson), the centred residual (sch_jameson) and the
fused iteration.  FP64 results are compared bit for bit; cases with the
injection condition (its real power is one portable implementation on both
sides) bit for bit too."""
import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib

from ._helpers import assert_equal_bits, max_rel_cols, oracle_prepared, real

pytestmark = pytest.mark.gpu

JAM = {
    # config-1b form: Euler, Jameson k2 = 0.5, k4 = 1/32, extr + periodic
    # (with the flagged fix of implimf_eu.f90:312 so that several
    # iterations stay finite)
    "box_eu": lambda: cases.box_case((12, 7, 6), seed=17, skew=0.02, alpha=2.0, ischema=1,
                                     qfix_dfez=1),
    # the reference Euler implicit phase as it is (two iterations)
    "box_eu_ref": lambda: cases.box_case((10, 6, 5), seed=18, skew=0.02, ischema=1),
    # Navier-Stokes Jameson on the multi-block channel (idd/prd/para/rc)
    "channel": lambda: cases.channel_case([9, 6, 7], 8, 5, seed=13, reynz=1.0e3, ischema=1),
}


def _gpu(case):
    from codens_b200.solver import CodeNS
    s = CodeNS(case)
    s.metric()
    s.sync()
    return s


def _t(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _n(t):
    return t.detach().cpu().numpy()


def _prepared(case):
    """oracle state after zpres, zvismo, chronos (the start of a Jameson
    iteration; ghosts as the initial state left them)"""
    orc, st = oracle_prepared(case)
    L = orc_lib()
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
        if case.scheme.ns:
            L.orc_zvismo(l, st.mu, st.temp)
        L.orc_chronos(l, st.mu, st.mut, st.v, st.dt, st.sn, st.vol, st.cson)
    return orc, st


def _load(torch, s, st):
    for nm, a in (("v", st.v), ("pression", st.ps), ("ztemp", st.temp), ("cson", st.cson),
                  ("mu", st.mu), ("mut", st.mut), ("dt", st.dt), ("tau", st.tau)):
        getattr(s, nm).copy_(_t(torch, a))
    torch.cuda.synchronize()


@pytest.mark.parametrize("name", ["box_eu", "channel"])
def test_ghost_refresh_parity(cuda, name):
    torch = cuda
    case = JAM[name]()
    orc, st = _prepared(case)
    s = _gpu(case)
    _load(torch, s, st)
    L = orc_lib()
    L.orc_rfve(st.v, st.ps, st.temp, st.cson)
    L.orc_rfvc(st.v, st.ps, st.temp, st.cson)
    s.rfve(s.v, s.pression, s.ztemp, s.cson)
    s.rfvc(s.v, s.pression, s.ztemp, s.cson)
    s.sync()
    n = case.layout.ncells
    assert_equal_bits(_n(s.v).reshape(5, -1)[:, :n], st.v.reshape(5, -1)[:, :n], "v")
    for nm, a in (("pression", st.ps), ("ztemp", st.temp), ("cson", st.cson)):
        assert_equal_bits(_n(getattr(s, nm))[:n], a[:n], nm)
    s.close()


@pytest.mark.parametrize("name", ["box_eu", "channel"])
def test_dissip_jameson_parity(cuda, name):
    torch = cuda
    case = JAM[name]()
    orc, st = _prepared(case)
    L = orc_lib()
    L.orc_rfve(st.v, st.ps, st.temp, st.cson)
    L.orc_rfvc(st.v, st.ps, st.temp, st.cson)
    s = _gpu(case)
    _load(torch, s, st)
    d_o = np.zeros_like(st.dis)
    for l in range(1, case.layout.nblk + 1):
        L.orc_dissip_jameson(l, st.v, d_o, st.sn, st.ps, st.cson)
    ld = case.layout.ld
    n = case.layout.ncells
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        s.d.fill_(7.0)
        torch.cuda.synchronize()
        s.dissip_jameson(l, s.v, s.d, s.sn, s.pression, s.cson)
        s.sync()
        if l == 0:
            sel = np.arange(n)  # ghosts zeroed too (dissip_jameson.f90:76-88)
        else:
            b = case.layout.blocks[l - 1]
            sel = np.arange(b.npc, b.npc + b.nnn)
        assert_equal_bits(_n(s.d).reshape(5, ld)[:, sel], d_o.reshape(5, ld)[:, sel],
                          f"d (l={l})")
    s.close()


@pytest.mark.parametrize("name", ["box_eu", "channel"])
def test_sch_jameson_parity(cuda, name):
    torch = cuda
    case = JAM[name]()
    orc, st = _prepared(case)
    L = orc_lib()
    L.orc_rfve(st.v, st.ps, st.temp, st.cson)
    L.orc_rfvc(st.v, st.ps, st.temp, st.cson)
    for l in range(1, case.layout.nblk + 1):
        L.orc_dissip_jameson(l, st.v, st.dis, st.sn, st.ps, st.cson)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    if case.scheme.ns:
        L.orc_zvisqc(st.v, st.mu, st.mut, st.tau, st.sn, st.vol, st.temp)
    u_o = np.zeros_like(st.u)
    for l in range(1, case.layout.nblk + 1):
        L.orc_sch_jameson(l, u_o, st.v, st.dis, st.tau, st.sn, st.ps)
    s = _gpu(case)
    _load(torch, s, st)
    s.d.copy_(_t(torch, st.dis))
    ld = case.layout.ld
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        s.u.fill_(7.0)
        torch.cuda.synchronize()
        s.sch_jameson(l, s.u, s.v, s.d, s.tau, s.sn, s.pression)
        s.sync()
        sel = real(case) if l == 0 else case.layout.blocks[l - 1].real_cells()
        assert_equal_bits(_n(s.u).reshape(5, ld)[:, sel], u_o.reshape(5, ld)[:, sel],
                          f"u (l={l})")
    s.close()


@pytest.mark.parametrize("name,nsteps", [("box_eu", 8), ("box_eu_ref", 2), ("channel", 6)])
def test_jameson_fused_steps_parity(cuda, name, nsteps):
    """the fused Jameson iteration (rfve on the first cycle only) against the
    oracle's atsch_num sequence, state and norms after every iteration"""
    case = JAM[name]()
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
        assert_equal_bits(v_g, v_o, f"v after step {it} (injection: {has_idd})")
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0, err_msg=f"norms step {it}")
    s.close()


def test_jameson_mixed_tracks_fp64(cuda):
    """the mixed form (FP64 Jameson residual, FP32 sweeps) stays within FP32
    rounding of the FP64 iteration over a few steps"""
    from codens_b200.solver import CodeNS
    outs = []
    for prec in (0, 1):
        case = JAM["box_eu"]()
        case.scheme.precision = prec
        s = CodeNS(case)
        s.metric()
        s.atsch_num(4)
        outs.append(_n(s.v).reshape(5, case.layout.ld)[:, real(case)])
        s.close()
    assert max_rel_cols(outs[1], outs[0]) < 1e-4


def test_defect_form_rejects_jameson(cuda):
    from codens_b200 import abi
    from codens_b200.solver import CodeNS
    case = JAM["box_eu"]()
    s = CodeNS(case)
    case.scheme.precision = 2
    with pytest.raises(abi.CnsError) as ei:
        s.set_scheme(case.scheme)
    assert ei.value.code == abi.CNS_EINVAL
    s.close()
