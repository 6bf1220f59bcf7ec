"""GPU parity of the turbulence-transport terms on the mean-flow path
(met_fludc, met_fludcsa, met_roe2o, met_roe2oh) against the oracle, bit for
bit, on every block at once and block by block."""
import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib

from ._helpers import assert_equal_bits, oracle_prepared

pytestmark = pytest.mark.gpu

CASES = {
    "box": lambda: cases.box_case((9, 6, 5), seed=8, noise=0.02, skew=0.02, ns=True),
    "channel": lambda: cases.channel_case([9, 6, 7], 8, 5, seed=13, reynz=1.0e3),
}
ALFAK, ALFAE, SIGMA, EPSROE = 1.0, 1.3, 2.0 / 3.0, 0.1


def _gpu(case):
    from codens_b200.solver import CodeNS
    s = CodeNS(case)
    s.metric()
    s.set_turbulence(ALFAK, ALFAE, SIGMA, EPSROE)
    s.sync()
    return s


def _t(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _transport_state(case, st, seed=31):
    """(ld, 7) state: the mean flow with its ghost cells filled by the
    boundary conditions, and two seeded transport variables"""
    ld = case.layout.ld
    L = orc_lib()
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    t = np.zeros((7, ld))
    t[:5] = st.v.reshape(5, ld)
    r = cases.splitmix64_uniform(seed, 2 * ld).reshape(2, ld)
    t[5] = t[0] * (1e-3 + 1e-3 * r[0])
    t[6] = t[0] * (0.5 + r[1])
    return t


def _fields(case, seed):
    ld = case.layout.ld
    r = cases.splitmix64_uniform(seed, 8 * ld).reshape(8, ld)
    mu = 1e-3 * (1.0 + r[0])
    mut = 1e-2 * r[1]
    fd = r[2:8] - 0.5
    return mu, mut, fd


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_fludc_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    mu, mut, fd = _fields(case, 41)
    L = orc_lib()
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        fo = fd.copy()
        blocks = range(1, case.layout.nblk + 1) if l == 0 else [l]
        for b in blocks:
            L.orc_met_fludc(b, mu, mut, *[fo[q] for q in range(6)], ALFAK, ALFAE)
        fg = [_t(torch, fd[q]) for q in range(6)]
        s.met_fludc(l, _t(torch, mu), _t(torch, mut), *fg)
        s.sync()
        for q in range(6):
            assert_equal_bits(fg[q].cpu().numpy(), fo[q], f"fd[{q}] (l={l})")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_fludcsa_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    mu, _, fd = _fields(case, 43)
    t = _transport_state(case, st)
    L = orc_lib()
    fo = fd.copy()
    for b in range(1, case.layout.nblk + 1):
        L.orc_met_fludcsa(b, t.reshape(-1), mu, *[fo[q] for q in range(6)], SIGMA)
    fg = [_t(torch, fd[q]) for q in range(6)]
    s.met_fludcsa(0, _t(torch, t.reshape(-1)), _t(torch, mu), *fg)
    s.sync()
    for q in range(6):
        assert_equal_bits(fg[q].cpu().numpy(), fo[q], f"fd[{q}]")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("harten", [False, True])
def test_met_roe2o_parity(cuda, name, harten):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    ld = case.layout.ld
    L = orc_lib()
    tg = _t(torch, t.reshape(-1))
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        d_o = np.full((7, ld), 3.0)
        blocks = range(1, case.layout.nblk + 1) if l == 0 else [l]
        for b in blocks:
            L.orc_met_roe2o(b, t.reshape(-1), d_o.reshape(-1), st.sn, int(harten), EPSROE)
        dg = _t(torch, np.full(7 * ld, 3.0))
        s.met_roe2o(l, tg, dg, s.sn, harten=harten)
        s.sync()
        assert_equal_bits(dg.cpu().numpy().reshape(7, ld), d_o, f"d (l={l})")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_samut_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    mu, _, _ = _fields(case, 47)
    L = orc_lib()
    mut_o = np.full(case.layout.ld, 5.0)
    for b in range(1, case.layout.nblk + 1):
        L.orc_met_samut(b, t.reshape(-1), mu, mut_o)
    mut_g = _t(torch, np.full(case.layout.ld, 5.0))
    s.met_samut(0, _t(torch, t.reshape(-1)), _t(torch, mu), mut_g)
    s.sync()
    assert_equal_bits(mut_g.cpu().numpy(), mut_o, "mut")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_sch_turb_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    ld = case.layout.ld
    mu, mut, fd = _fields(case, 53)
    r = cases.splitmix64_uniform(59, 4 * ld).reshape(4, ld) - 0.5
    ts6, ts7 = r[0] * 1e-3, r[1] * 1e-3
    d = np.zeros((7, ld))
    d[5], d[6] = r[2] * 1e-4, r[3] * 1e-4
    L = orc_lib()
    tg = _t(torch, t.reshape(-1))
    fdg = [_t(torch, fd[q]) for q in range(6)]
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        u_o = np.full((7, ld), 9.0)
        blocks = range(1, case.layout.nblk + 1) if l == 0 else [l]
        for b in blocks:
            L.orc_sch_turb(b, u_o.reshape(-1), t.reshape(-1), d.reshape(-1),
                           *[fd[q] for q in range(6)], ts6, ts7, st.sn, st.vol)
        ug = _t(torch, np.full(7 * ld, 9.0))
        s.sch_turb(l, ug, tg, _t(torch, d.reshape(-1)), *fdg, _t(torch, ts6), _t(torch, ts7),
                   s.sn, s.vol)
        s.sync()
        if l == 0:
            sel = np.arange(case.layout.ncells)
        else:
            b = case.layout.blocks[l - 1]
            sel = np.arange(b.npc, b.npc + b.nnn)
        assert_equal_bits(ug.cpu().numpy().reshape(7, ld)[5:, sel], u_o[5:, sel], f"u67 (l={l})")
    s.close()


def _dv_oracle(case, st, t):
    """teq_gradv of the oracle, block by block, in the global [9][ld] layout"""
    ld = case.layout.ld
    L = orc_lib()
    dv = np.zeros((9, ld))
    for l, b in enumerate(case.layout.blocks, start=1):
        loc = np.zeros(9 * b.nnn)
        L.orc_teq_gradv(l, st.sn, st.vol, t.reshape(-1), loc)
        dv[:, b.npc:b.npc + b.nnn] = loc.reshape(9, b.nnn)
    return dv


@pytest.mark.parametrize("name", sorted(CASES))
def test_teq_gradv_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    dv_o = _dv_oracle(case, st, t)
    dv_g = _t(torch, np.zeros(9 * case.layout.ld))
    s.teq_gradv(0, _t(torch, t.reshape(-1)), s.sn, s.vol, dv_g)
    s.sync()
    rc = case.layout.real_cells()
    assert_equal_bits(dv_g.cpu().numpy().reshape(9, -1)[:, rc], dv_o[:, rc], "dv")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_smsa_parity(cuda, name):
    """the SA source against the oracle: exp and the real power of
    met_smsa.f90 are one portable implementation on both sides, so bit for
    bit"""
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    ld = case.layout.ld
    mu, _, fd = _fields(case, 61)
    dist = 0.01 + cases.splitmix64_uniform(67, ld)
    dv = _dv_oracle(case, st, t)
    L = orc_lib()
    ts6_o, ts7_o, cf_o = np.full(ld, 4.0), np.full(ld, 4.0), np.full(ld, 4.0)
    for l, b in enumerate(case.layout.blocks, start=1):
        L.orc_met_smsa(l, st.sn, st.vol, t.reshape(-1), mu, dist,
                       np.ascontiguousarray(dv[:, b.npc:b.npc + b.nnn]).reshape(-1),
                       fd[0], fd[1], fd[2], ts6_o, ts7_o, cf_o)
    g = [_t(torch, np.full(ld, 4.0)) for _ in range(3)]
    s.met_smsa(0, _t(torch, t.reshape(-1)), _t(torch, mu), _t(torch, dist), s.sn, s.vol,
               _t(torch, dv.reshape(-1)), _t(torch, fd[0]), _t(torch, fd[1]), _t(torch, fd[2]),
               *g)
    s.sync()
    rc = case.layout.real_cells()
    for a, b, w in zip(g, (ts6_o, ts7_o, cf_o), ("ts6", "ts7", "cfke")):
        assert_equal_bits(a.cpu().numpy()[rc], b[rc], w)
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_impli2_eqt_3d_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    t = _transport_state(case, st)
    ld = case.layout.ld
    mu, mut, _ = _fields(case, 71)
    r = cases.splitmix64_uniform(73, 4 * ld).reshape(4, ld)
    dt = 0.01 + 0.01 * r[0]
    cfke = r[1]
    u = np.zeros((7, ld))
    u[5], u[6] = (r[2] - 0.5) * 1e-4, (r[3] - 0.5) * 1e-3
    L = orc_lib()
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        to = t.copy()
        blocks = range(1, case.layout.nblk + 1) if l == 0 else [l]
        for b in blocks:
            L.orc_impli2_eqt_3d(b, u.reshape(-1), dt, to.reshape(-1), mu, mut, cfke, st.sn,
                                st.vol, 1.0)
        tg = _t(torch, t.reshape(-1))
        s.impli2_eqt_3d(l, _t(torch, u.reshape(-1)), _t(torch, dt), tg, _t(torch, mu),
                        _t(torch, mut), _t(torch, cfke), s.sn, s.vol, 1.0)
        s.sync()
        assert_equal_bits(tg.cpu().numpy().reshape(7, ld), to, f"v (l={l})")
    s.close()
