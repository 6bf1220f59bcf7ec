"""GPU parity of the Spalart-Allmaras transport step (met_num.f90 for
1SA) against the oracle, bit for bit: the wall distance, the turbulence
ghosts, the transport-variable gradients, the diffusion-density ghosts, the
clip, the whole step and fused RANS iterations (the source term's exp and
real power are one portable implementation on both sides)."""
import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib

from ._helpers import assert_equal_bits, max_rel_cols, oracle_prepared

pytestmark = pytest.mark.gpu

CASES = {
    "plate": lambda: cases.flat_plate_case((14, 10, 4), reynz=1.0e4, dy1=2e-3, ratio=1.2,
                                           seed=5, noise=0.01),
    # three blocks: coincident joins, idd, prd and walls on both sides.
    # Unlimited MUSCL: the minmod limiter's in-place ratio recurrence is
    # discontinuous (a 1e-14 change of the state moves the next one by
    # ~1e-5); kept unlimited so that this case isolates the SA step
    "channel": lambda: cases.channel_case([9, 6, 7], 8, 5, seed=13, reynz=1.0e3, ilim=0),
}

# the wall law of the 'lp2' walls (lpsa1, lparoi1, the implicit freeze)
WALL_LAW = {
    # log law (rho u y / mu above yp0^2 in every first cell); the k faces are
    # wall-law walls too, so the corner cells take two walls' laws in order
    "plate_wl": lambda: cases.flat_plate_case((14, 10, 4), reynz=1.0e6, dy1=2e-3, ratio=1.2,
                                              seed=5, noise=0.01, wall_kind=cases.BC_LP2,
                                              side_walls=True),
    # linear law, three blocks
    "channel_wl": lambda: cases.channel_case([9, 6, 7], 8, 5, seed=13, reynz=1.0e3, ilim=0,
                                             wall_kind=cases.BC_LP2),
}
ALL = {**CASES, **WALL_LAW}


def _seven(case, seed=71):
    """the case's state with seeded transport columns when it has only 5"""
    if case.v0.shape[0] == 7:
        return case
    ld = case.layout.ld
    v = np.zeros((7, ld))
    v[:5] = case.v0
    r = cases.splitmix64_uniform(seed, 2 * ld).reshape(2, ld)
    v[5] = v[0] * (1e-3 + 1e-3 * r[0])
    v[6] = v[0] * (0.1 + r[1])
    case.v0 = v
    case.meta["rokinf"] = 2e-3
    return case


def _gpu(case):
    from codens_b200.solver import CodeNS
    s = CodeNS(case)
    s.metric()
    s.sync()
    return s


def _t(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("name", sorted(ALL))
def test_atcaldis3_parity(cuda, name):
    case = ALL[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    d_o = np.full(case.layout.ld, -1.0)
    assert orc_lib().orc_atcaldis3(st.x, st.y, st.z, d_o) == 0
    d_g = s.atcaldis3()
    s.sync()
    rc = case.layout.real_cells()
    assert_equal_bits(d_g.cpu().numpy()[rc], d_o[rc], "dist")
    assert (d_o[rc] > 0).all()
    s.close()


def test_atcaldis3_needs_a_wall(cuda):
    from codens_b200 import abi
    s = _gpu(cases.box_case((6, 5, 4), ns=True))
    with pytest.raises(abi.CnsError) as ei:
        s.atcaldis3()
    assert ei.value.code == abi.CNS_EBC
    s.close()


@pytest.mark.parametrize("name", sorted(ALL))
def test_met_bord_parity(cuda, name):
    torch = cuda
    case = _seven(ALL[name]())
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    v_o = st.v.copy()
    orc_lib().orc_met_bord(v_o, 1.25e-3, 0.5)
    vg = _t(torch, case.v0.reshape(-1))
    s.met_bord(vg, 1.25e-3, 0.5)
    s.sync()
    assert_equal_bits(vg.cpu().numpy(), v_o, "v after met_bord")
    s.close()


def _bordered(case, st):
    """(ld, 7) state whose ghost cells hold the mean-flow and turbulence
    boundary values (rbord then met_bord), as met_num sees it"""
    L = orc_lib()
    v = st.v.copy()
    ld = case.layout.ld
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, v, st.ps, st.temp, st.cson)
    L.orc_rbord(v, st.ps, st.temp, st.cson)
    L.orc_met_bord(v, case.meta["rokinf"], 0.0)
    return v.reshape(7, ld)


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_gradtr_parity(cuda, name):
    torch = cuda
    case = _seven(CASES[name]())
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    v = _bordered(case, st)
    ld = case.layout.ld
    L = orc_lib()
    vg = _t(torch, v.reshape(-1))
    for l in [0] + list(range(1, case.layout.nblk + 1)):
        fo = np.full((6, ld), 7.0)
        blocks = range(1, case.layout.nblk + 1) if l == 0 else [l]
        for b in blocks:
            L.orc_met_gradtr(b, st.sn, st.vol, v.reshape(-1), *[fo[q] for q in range(6)])
        fg = [_t(torch, np.full(ld, 7.0)) for _ in range(6)]
        s.met_gradtr(l, vg, s.sn, s.vol, *fg)
        s.sync()
        for q in range(6):
            assert_equal_bits(fg[q].cpu().numpy(), fo[q], f"fd[{q}] (l={l})")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_met_rbse_parity(cuda, name):
    torch = cuda
    case = CASES[name]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    fd = cases.splitmix64_uniform(73, 6 * ld).reshape(6, ld) - 0.5
    fo = fd.copy()
    orc_lib().orc_met_rbse(*[fo[q] for q in range(6)])
    fg = [_t(torch, fd[q]) for q in range(6)]
    s.met_rbse(*fg)
    s.sync()
    for q in range(6):
        assert_equal_bits(fg[q].cpu().numpy(), fo[q], f"fd[{q}]")
    s.close()


def test_met_cutsa_parity(cuda):
    torch = cuda
    case = CASES["channel"]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    v = np.zeros((7, ld))
    v[:5] = case.v0
    r = cases.splitmix64_uniform(79, 2 * ld).reshape(2, ld)
    v[5] = r[0] - 0.3
    v[6] = r[1]
    vo = v.reshape(-1).copy()
    for b in range(1, case.layout.nblk + 1):
        orc_lib().orc_met_cutsa(b, vo, 1e-8)
    vg = _t(torch, v.reshape(-1))
    s.met_cutsa(0, vg, 1e-8)
    s.sync()
    assert_equal_bits(vg.cpu().numpy(), vo, "v after met_cutsa")
    s.close()


def _sa_pair(case):
    """oracle and GPU solver with the SA step on, from the same state and the
    oracle's wall distance"""
    orc, st = oracle_prepared(case)
    dist = np.zeros(case.layout.ld)
    assert orc_lib().orc_atcaldis3(st.x, st.y, st.z, dist) == 0
    rok = case.meta["rokinf"]
    orc.set_sa(st, dist, rok, 0.0)
    s = _gpu(case)
    dg = _t(s.torch, dist)
    s.set_sa(dg, rok, 0.0, 1e-8)
    return orc, st, s


@pytest.mark.parametrize("name", sorted(ALL))
def test_met_num_parity(cuda, name):
    """one transport step (met_num for 1SA) on the state after the mean-flow
    thermodynamics, time step and boundary conditions"""
    case = _seven(ALL[name]())
    orc, st, s = _sa_pair(case)
    L = orc_lib()
    ld = case.layout.ld
    nb = case.layout.nblk
    for l in range(1, nb + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
        L.orc_zvismo(l, st.mu, st.temp)
        L.orc_chronos(l, st.mu, st.mut, st.v, st.dt, st.sn, st.vol, st.cson)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    # the GPU solver on the same inputs: state and the mean-flow arrays
    for name_, a in (("v", st.v), ("dt", st.dt), ("mu", st.mu), ("mut", st.mut),
                     ("pression", st.ps), ("ztemp", st.temp), ("cson", st.cson)):
        getattr(s, name_).copy_(s.torch.as_tensor(a))
    s.torch.cuda.synchronize()
    s.sync()
    L.orc_met_num(st.v, st.u, st.d, st.dt, st.mu, st.mut, st.sn, st.vol, st.temp)
    s.met_num()
    s.sync()
    rc = case.layout.real_cells()
    v_g = s.v.cpu().numpy().reshape(7, ld)
    v_o = st.v.reshape(7, ld)
    assert_equal_bits(v_g[5:6, rc], v_o[5:6, rc], "rho nu~")
    assert_equal_bits(v_g[:5], v_o[:5], "mean-flow columns untouched")
    assert_equal_bits(s.mut.cpu().numpy()[rc], st.mut[rc], "mut")
    s.close()


@pytest.mark.parametrize("name", sorted(ALL))
def test_fused_rans_iterations_parity(cuda, name):
    """fused FP64 iterations with the SA step against the oracle's
    atsch_num + met_num sequence"""
    case = _seven(ALL[name]())
    orc, st, s = _sa_pair(case)
    for _ in range(3):
        orc.step(st)
    s.atsch_num(3)
    s.sync()
    ld = case.layout.ld
    rc = case.layout.real_cells()
    v_g = s.v.cpu().numpy().reshape(7, ld)[:, rc]
    v_o = st.v.reshape(7, ld)[:, rc]
    assert_equal_bits(v_g[:6], v_o[:6], "state after 3 iterations")
    assert_equal_bits(s.mut.cpu().numpy()[rc], st.mut[rc], "mut")
    s.close()


def test_mixed_rans_iterations(cuda):
    """the mixed form with the SA step (FP32 mean-flow sweeps, everything
    else FP64) stays within FP32 reach of the FP64 iteration"""
    case = CASES["plate"]()
    orc, st, a = _sa_pair(case)
    case_b = CASES["plate"]()
    case_b.scheme.precision = 1
    from codens_b200.solver import CodeNS
    b = CodeNS(case_b)
    b.metric()
    b.set_sa(b.atcaldis3(), case.meta["rokinf"], 0.0, 1e-8)
    a.atsch_num(20)
    b.atsch_num(20)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    va = a.v.cpu().numpy().reshape(7, ld)[:, rc]
    vb = b.v.cpu().numpy().reshape(7, ld)[:, rc]
    assert np.isfinite(vb).all()
    assert max_rel_cols(vb[:6], va[:6]) < 1e-3
    a.close()
    b.close()


def test_set_sa_needs_seven_columns(cuda):
    s = _gpu(CASES["channel"]())
    with pytest.raises(ValueError):
        s.set_sa(s.vol, 1e-3, 0.0)
    s.close()


def test_met_smsa_stilde_fix_parity(cuda):
    """the flagged source fix (modified vorticity, guarded derivative) against
    the oracle's, on a state where both branches of the modified vorticity
    occur (chi = 2..6 makes fv2 < 0, so S_bar < -0.7 vort at the cells of
    small vorticity); finite everywhere, and 1e-13 like the reference form"""
    torch = cuda
    case = CASES["plate"]()
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    t = _bordered(case, st).copy()
    r = cases.splitmix64_uniform(83, 3 * ld).reshape(3, ld)
    mu = 1e-3 * (1.0 + r[0])
    t[5] = mu * (2.0 + 4.0 * r[1])              # chi in 2..6
    dist = 0.01 + r[2]
    L = orc_lib()
    b = case.layout.blocks[0]
    loc = np.zeros(9 * b.nnn)
    L.orc_teq_gradv(1, st.sn, st.vol, t.reshape(-1), loc)
    dv = np.zeros((9, ld))
    dv[:, b.npc:b.npc + b.nnn] = loc.reshape(9, b.nnn)
    fd = cases.splitmix64_uniform(89, 3 * ld).reshape(3, ld) - 0.5
    rc = case.layout.real_cells()
    # both branches of the modified vorticity are exercised
    d = dv[:, rc]
    vort = np.sqrt((d[7] - d[5]) ** 2 + (d[2] - d[6]) ** 2 + (d[3] - d[1]) ** 2)
    chi = t[5, rc] / mu[rc]
    fv1 = chi ** 3 / (chi ** 3 + 7.1 ** 3)
    sbar = (t[5, rc] / t[0, rc]) * (1.0 - chi / (1.0 + chi * fv1)) / (0.41 ** 2 * dist[rc] ** 2)
    low = sbar < -0.7 * vort
    assert low.any() and (~low).any()
    L.orc_set_sa_fix(1)
    try:
        out_o = [np.full(ld, 4.0) for _ in range(3)]
        L.orc_met_smsa(1, st.sn, st.vol, t.reshape(-1), mu, dist, loc, fd[0], fd[1], fd[2],
                       *out_o)
    finally:
        L.orc_set_sa_fix(0)
    s.set_sa(_t(torch, dist), case.meta["rokinf"], 0.0, 1e-8, stilde_fix=1)
    g = [_t(torch, np.full(ld, 4.0)) for _ in range(3)]
    s.met_smsa(0, _t(torch, t.reshape(-1)), _t(torch, mu), _t(torch, dist), s.sn, s.vol,
               _t(torch, dv.reshape(-1)), _t(torch, fd[0]), _t(torch, fd[1]), _t(torch, fd[2]),
               *g)
    s.sync()
    for a, o, w in zip(g, out_o, ("ts6", "ts7", "cfke")):
        ag = a.cpu().numpy()[rc]
        assert np.isfinite(ag).all(), w
        assert_equal_bits(ag, o[rc], w)
    s.close()


def test_fused_rans_iterations_stilde_fix_parity(cuda):
    """fused FP64 iterations with the flagged source fix against the oracle"""
    case = _seven(CASES["channel"]())
    orc, st = oracle_prepared(case)
    dist = np.zeros(case.layout.ld)
    assert orc_lib().orc_atcaldis3(st.x, st.y, st.z, dist) == 0
    rok = case.meta["rokinf"]
    orc.set_sa(st, dist, rok, 0.0, stilde_fix=1)
    s = _gpu(case)
    s.set_sa(_t(s.torch, dist), rok, 0.0, 1e-8, stilde_fix=1)
    try:
        for _ in range(3):
            orc.step(st)
    finally:
        orc.clear_sa()
    s.atsch_num(3)
    s.sync()
    ld = case.layout.ld
    rc = case.layout.real_cells()
    v_g = s.v.cpu().numpy().reshape(7, ld)[:, rc]
    v_o = st.v.reshape(7, ld)[:, rc]
    assert_equal_bits(v_g[:6], v_o[:6], "state after 3 iterations")
    s.close()


def _lp2_first_cells(case):
    ba = case.boundary_arrays()
    sel = np.flatnonzero(ba["type"] == cases.BC_LP2)
    return np.concatenate([ba["ncin"][ba["mpb"][b]:ba["mpb"][b] + ba["mmb"][b]] for b in sel])


@pytest.mark.parametrize("name", sorted(WALL_LAW))
def test_wall_law_parity(cuda, name):
    """lpsa (block by block) and cllparoi1 after zvisqc, from the same
    prepared state and a seeded eddy viscosity, bit for bit on every cell"""
    torch = cuda
    case = _seven(WALL_LAW[name]())
    orc, st = oracle_prepared(case)
    L = orc_lib()
    ld = case.layout.ld
    dist = np.zeros(ld)
    assert L.orc_atcaldis3(st.x, st.y, st.z, dist) == 0
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
        L.orc_zvismo(l, st.mu, st.temp)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    st.mut[:] = st.mu * (0.5 + cases.splitmix64_uniform(91, ld))
    s = _gpu(case)
    s.set_sa(_t(torch, dist), case.meta["rokinf"], 0.0, 1e-8)
    g = {k: _t(torch, a) for k, a in (("v", st.v), ("mu", st.mu), ("mut", st.mut),
                                      ("temp", st.temp), ("dist", dist))}
    for l in range(1, case.layout.nblk + 1):
        L.orc_lpsa(l, st.v, st.mu, st.mut, dist, st.temp, 1e-8)
        s.lpsa(l, g["v"], g["mu"], g["mut"], g["dist"], g["temp"])
    s.sync()
    ni = _lp2_first_cells(case)
    assert np.isfinite(st.v.reshape(7, ld)[5, ni]).all()
    assert_equal_bits(g["v"].cpu().numpy(), st.v, "v after lpsa")
    assert_equal_bits(g["mut"].cpu().numpy(), st.mut, "mut after lpsa")
    # the mean-flow stresses: zvisqc, then the wall law
    L.orc_zvisqc(st.v, st.mu, st.mut, st.tau, st.sn, st.vol, st.temp)
    tau = torch.zeros(9 * ld, dtype=torch.float64, device="cuda")
    s.zvisqc(g["v"], g["mu"], g["mut"], tau, s.sn, s.vol, g["temp"])
    tau_before = st.tau.copy()
    L.orc_cllparoi1(st.v, dist, st.mu, st.mut, st.tau, st.temp)
    s.cllparoi1(g["v"], g["dist"], g["mu"], g["mut"], tau, g["temp"])
    s.sync()
    assert not np.array_equal(tau_before.reshape(9, ld)[:, ni], st.tau.reshape(9, ld)[:, ni])
    assert_equal_bits(tau.cpu().numpy(), st.tau, "tau after cllparoi1")
    s.close()


def test_wall_law_needs_the_wall_distance(cuda):
    """the mean-flow wall law reads the wall distance of set_sa"""
    from codens_b200 import abi
    s = _gpu(WALL_LAW["channel_wl"]())
    with pytest.raises(abi.CnsError) as ei:
        s.atsch_num(1)
    assert ei.value.code == abi.CNS_ENOTREADY
    s.close()
