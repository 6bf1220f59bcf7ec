"""GPU parity of the k-epsilon model of Jones & Launder (met_num.f90 for
equat '2JL') against the oracle, bit for bit: the production of k, the
sources with their low-Reynolds terms (met_smke: met_exgr, met_bark,
met_bare, met_smkes), the eddy viscosity, the clip, the whole transport
step and fused iterations with it; the mixed form next to FP64."""
import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import lib as orc_lib

from ._helpers import assert_equal_bits, max_rel_cols, oracle_prepared

pytestmark = pytest.mark.gpu


def ke_state(case, seed=31, k0=1e-3, ratio=10.0):
    """the case with rho k and rho eps columns: k = k0 (1 +- 10%), eps from
    an eddy viscosity of about ratio laminar ones (cmu rho k^2 / eps)"""
    ld = case.layout.ld
    v = np.zeros((7, ld))
    v[:5] = case.v0[:5]
    r = cases.splitmix64_uniform(seed, 2 * ld).reshape(2, ld)
    rho = np.where(v[0] > 0, v[0], 1.0)
    k = k0 * (0.9 + 0.2 * r[0])
    eps = 0.09 * k * k / (ratio / case.phys.reynz) * (0.9 + 0.2 * r[1])
    v[5] = rho * k
    v[6] = rho * eps
    case.v0 = v
    case.meta["rokinf"] = float(np.median(v[5]))
    case.meta["roeinf"] = float(np.median(v[6]))
    return case


CASES = {
    "plate": lambda: ke_state(cases.flat_plate_case((14, 10, 4), reynz=1.0e4, dy1=2e-3,
                                                    ratio=1.2, seed=5, noise=0.01)),
    # three blocks, two cells in k
    "channel": lambda: ke_state(cases.channel_case([9, 6, 7], 8, 2, seed=13, reynz=1.0e3,
                                                   ilim=0)),
}
# one cell thick in k: the two sides of met_exgr read each other (the routine
# test only; the mean flow of this channel does not survive an iteration)
THIN = lambda: ke_state(cases.channel_case([9, 6, 7], 8, 1, seed=13, reynz=1.0e3, ilim=0))


def _gpu(case):
    from codens_b200.solver import CodeNS
    s = CodeNS(case)
    s.metric()
    s.sync()
    return s


def _t(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _prepared(case):
    """oracle state after zpres, zvismo, chronos, rbord and met_bord, with a
    seeded eddy viscosity"""
    orc, st = oracle_prepared(case)
    L = orc_lib()
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
        L.orc_zvismo(l, st.mu, st.temp)
        L.orc_chronos(l, st.mu, st.mut, st.v, st.dt, st.sn, st.vol, st.cson)
    L.orc_rbord(st.v, st.ps, st.temp, st.cson)
    L.orc_met_bord(st.v, case.meta["rokinf"], case.meta["roeinf"])
    st.mut[:] = st.mu * (1.0 + 4.0 * cases.splitmix64_uniform(97, case.layout.ld))
    return orc, st


@pytest.mark.parametrize("name", sorted(CASES) + ["thin"])
def test_met_prod_smke_kemut_cutke_parity(cuda, name):
    torch = cuda
    case = THIN() if name == "thin" else CASES[name]()
    orc, st = _prepared(case)
    s = _gpu(case)
    L = orc_lib()
    ld = case.layout.ld
    g = {k: _t(torch, a) for k, a in (("v", st.v), ("mu", st.mu), ("mut", st.mut))}
    dv_g = torch.zeros(9 * ld, dtype=torch.float64, device="cuda")
    tp_g = torch.zeros(ld, dtype=torch.float64, device="cuda")
    ts_g = torch.zeros(2 * ld, dtype=torch.float64, device="cuda")
    cf_g = torch.zeros(ld, dtype=torch.float64, device="cuda")
    ts_o, cf_o = np.zeros(2 * ld), np.zeros(ld)
    for l in range(1, case.layout.nblk + 1):
        b = case.layout.blocks[l - 1]
        nnn, n0 = b.nnn, b.npc
        dv_o = np.zeros(9 * nnn)
        tp_o = np.zeros(nnn)
        L.orc_teq_gradv(l, st.sn, st.vol, st.v, dv_o)
        L.orc_met_prod(l, st.mut, st.v, dv_o, tp_o)
        s.teq_gradv(l, g["v"], s.sn, s.vol, dv_g)
        s.met_prod(l, g["mut"], g["v"], dv_g, tp_g)
        s.sync()
        rc = b.real_cells()
        assert_equal_bits(tp_g.cpu().numpy()[rc], tp_o[rc - n0], f"tprod block {l}")
        L.orc_met_smke(l, st.sn, st.vol, st.v, st.mu, st.mut, tp_o, dv_o, ts_o[:ld], ts_o[ld:],
                       cf_o)
        s.met_smke(l, s.sn, s.vol, g["v"], g["mu"], g["mut"], tp_g, cf_g, dv_g, ts_g[:ld],
                   ts_g[ld:])
        s.sync()
        # met_exgr's ghosts of the nine gradients, then the sources
        keep = np.array([b.ic(i, j, k) for k in range(b.nk + 1) for j in range(b.nj + 1)
                         for i in range(b.ni + 1)])
        assert_equal_bits(dv_g.cpu().numpy().reshape(9, ld)[:, keep],
                          dv_o.reshape(9, nnn)[:, keep - n0], f"dv ghosts block {l}")
        assert_equal_bits(ts_g.cpu().numpy().reshape(2, ld)[:, rc], ts_o.reshape(2, ld)[:, rc],
                          f"sources block {l}")
        assert_equal_bits(cf_g.cpu().numpy()[rc], cf_o[rc], f"cfke block {l}")
    # eddy viscosity and the clip (some cells pushed below the floors)
    mut_o = st.mut.copy()
    v_o = st.v.copy()
    vv = v_o.reshape(7, ld)
    r = cases.splitmix64_uniform(5, ld)
    vv[5, r < 0.1] = 1e-12
    vv[6, (r > 0.5) & (r < 0.6)] = -1e-3
    vg = _t(torch, v_o)
    for l in range(1, case.layout.nblk + 1):
        L.orc_met_kemut(l, st.v, st.mu, mut_o)
        s.met_kemut(l, g["v"], g["mu"], g["mut"])
        L.orc_met_cutke(l, v_o, 1e-10, 2e-10)
        s.met_cutke(l, vg, 1e-10, 2e-10)
    s.sync()
    rc = case.layout.real_cells()
    assert_equal_bits(g["mut"].cpu().numpy()[rc], mut_o[rc], "mut")
    assert_equal_bits(vg.cpu().numpy(), v_o, "v after met_cutke")
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_turbulence_initialisation_parity(cuda, name):
    """met_inmut, met_inisa and met_ini (teq_gradv + met_brad) of every block"""
    torch = cuda
    case = CASES[name]()
    orc, st = _prepared(case)
    s = _gpu(case)
    L = orc_lib()
    ld = case.layout.ld
    g = {k: _t(torch, a) for k, a in (("v", st.v), ("mu", st.mu), ("mut", st.mut))}
    dv_g = torch.zeros(9 * ld, dtype=torch.float64, device="cuda")
    v_o, mut_o = st.v.copy(), st.mut.copy()
    for l in range(1, case.layout.nblk + 1):
        b = case.layout.blocks[l - 1]
        L.orc_met_inmut(l, st.mu, mut_o)
        s.met_inmut(l, g["mu"], g["mut"])
        L.orc_met_ini(l, v_o, mut_o, st.sn, st.vol, np.zeros(9 * b.nnn))
        s.met_ini(l, g["v"], g["mut"], g["mu"], s.sn, s.vol, dv_g)
    s.sync()
    assert_equal_bits(g["mut"].cpu().numpy(), mut_o, "mut = mu / 10")
    assert_equal_bits(g["v"].cpu().numpy(), v_o, "v after met_ini")
    for l in range(1, case.layout.nblk + 1):
        L.orc_met_inisa(l, v_o, mut_o)
        s.met_inisa(l, g["v"], g["mut"], g["mu"])
    s.sync()
    assert_equal_bits(g["v"].cpu().numpy(), v_o, "v after met_inisa")
    s.close()


def _ke_pair(case):
    orc, st = oracle_prepared(case)
    orc.set_ke(st, case.meta["rokinf"], case.meta["roeinf"])
    s = _gpu(case)
    s.set_ke(case.meta["rokinf"], case.meta["roeinf"], 1e-10, 1e-10)
    return orc, st, s


@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_ke_iterations_parity(cuda, name):
    """fused FP64 iterations with the k-epsilon step (met_num after rbord)
    against the oracle's sequence, bit for bit; the clip acts on the way"""
    case = CASES[name]()
    orc, st, s = _ke_pair(case)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    for it in range(12):
        u0 = st.v.copy()
        orc.step(st)
        no = orc.norms(u0[:5 * ld], st)
        ng = s.atsch_num(1)
        v_g = s.v.cpu().numpy().reshape(7, ld)[:, rc]
        v_o = st.v.reshape(7, ld)[:, rc]
        assert np.isfinite(v_o).all(), it
        assert_equal_bits(v_g, v_o, f"state after iteration {it}")
        assert_equal_bits(s.mut.cpu().numpy()[rc], st.mut[rc], f"mut after iteration {it}")
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0, err_msg=f"norms {it}")
    s.close()


def test_mixed_ke_iterations(cuda):
    """the mixed form with the k-epsilon step stays within FP32 reach of the
    FP64 iteration"""
    case = CASES["plate"]()
    orc, st, a = _ke_pair(case)
    case_b = CASES["plate"]()
    case_b.scheme.precision = 1
    b = _gpu(case_b)
    b.set_ke(case.meta["rokinf"], case.meta["roeinf"], 1e-10, 1e-10)
    a.atsch_num(20)
    b.atsch_num(20)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    va = a.v.cpu().numpy().reshape(7, ld)[:5, rc]
    vb = b.v.cpu().numpy().reshape(7, ld)[:5, rc]
    assert np.isfinite(vb).all()
    assert max_rel_cols(vb, va) < 1e-3
    a.close()
    b.close()


def test_ke_refuses_wall_law_walls(cuda):
    from codens_b200 import abi
    case = ke_state(cases.flat_plate_case((8, 6, 2), wall_kind=cases.BC_LP2))
    s = _gpu(case)
    with pytest.raises(abi.CnsError) as ei:
        s.set_ke(1e-3, 1e-5)
    assert ei.value.code == abi.CNS_EINVAL
    s.close()
