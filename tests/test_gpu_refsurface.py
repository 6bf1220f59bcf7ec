"""The per-routine entry points with the reference routines' argument lists:
host arrays (the copy-in/out parity mode) give the same bits as device
arrays; ityprk != 0 forms and uses the multigrid forcing function as
sch_roe.f90:1466-1481 and implimf_3d.f90:249-264 do; the nine stress arrays
may be separate; chronos uses its etal argument; unsupported equat, a wrong
lgsnlt and a forcing call without ff are refused."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from codens_b200 import abi

from ._helpers import SMALL, assert_equal_bits, real
from .test_gpu_parity import _gpu, _load_state, _n, _prepared_flow

pytestmark = pytest.mark.gpu


def _host(t):
    return np.ascontiguousarray(_n(t))


@pytest.mark.parametrize("name", ["box_ns", "channel", "box_eu_qfix"])
def test_host_arrays_give_the_device_bits(cuda, name):
    torch = cuda
    case = SMALL[name]()
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    ld = case.layout.ld
    ns = bool(case.scheme.ns)
    for l in range(1, case.layout.nblk + 1):
        # residual
        if ns:
            s.sch_roe(l, s.u, s.v, s.tau, s.sn, s.pression)
        else:
            s.sch_roe_euler(l, s.u, s.v, s.sn, s.pression)
        s.sync()
        u_dev = _host(s.u)
        u_h = np.full(s.u.numel(), 3.0)
        v_h, tau_h, sn_h, ps_h = _host(s.v), _host(s.tau), _host(s.sn), _host(s.pression)
        if ns:
            s.sch_roe(l, u_h, v_h, tau_h, sn_h, ps_h)
        else:
            s.sch_roe_euler(l, u_h, v_h, sn_h, ps_h)
        sel = case.layout.blocks[l - 1].real_cells()
        assert_equal_bits(u_h.reshape(-1, ld)[:5, sel], u_dev.reshape(-1, ld)[:5, sel],
                          f"residual block {l}")
    # implicit phase on block 1, both ways, from the same inputs
    v0, d0 = s.v.clone(), s.d.clone()
    if ns:
        s.implimf_3d(1, s.u, s.dt, s.v, s.d, s.mu, s.mut, s.sn, s.vol, s.pression, s.cson, 4)
    else:
        s.implimf_eu(1, s.u, s.dt, s.v, s.d, s.sn, s.vol, s.pression, s.cson, 4)
    s.sync()
    v_dev, d_dev = _host(s.v), _host(s.d)
    v_h, d_h = _host(v0), _host(d0)
    h = {k: _host(getattr(s, k)) for k in ("u", "dt", "sn", "vol", "pression", "cson", "mu",
                                           "mut")}
    if ns:
        s.implimf_3d(1, h["u"], h["dt"], v_h, d_h, h["mu"], h["mut"], h["sn"], h["vol"],
                     h["pression"], h["cson"], 4)
    else:
        s.implimf_eu(1, h["u"], h["dt"], v_h, d_h, h["sn"], h["vol"], h["pression"],
                     h["cson"], 4)
    rc = case.layout.blocks[0].real_cells()
    assert_equal_bits(v_h.reshape(-1, ld)[:5, rc], v_dev.reshape(-1, ld)[:5, rc], "implicit v")
    assert_equal_bits(d_h.reshape(-1, ld)[:5, rc], d_dev.reshape(-1, ld)[:5, rc], "implicit d")
    # zpres, rbord, chronos on host arrays
    n = case.layout.ncells
    ps_h, t_h, c_h = np.zeros(ld), np.zeros(ld), np.zeros(ld)
    v_h = _host(v0)
    s.zpres(0, v_h, ps_h, t_h, c_h)
    s.rbord(v_h, ps_h, t_h, c_h)
    s.v.copy_(v0)
    torch.cuda.synchronize()
    s.zpres(0, s.v, s.pression, s.ztemp, s.cson)
    s.rbord(s.v, s.pression, s.ztemp, s.cson)
    s.sync()
    assert_equal_bits(ps_h[:n], _host(s.pression)[:n], "zpres + rbord pressure")
    assert_equal_bits(v_h.reshape(-1, ld)[:5, :n], _host(s.v).reshape(-1, ld)[:5, :n], "rbord v")
    dt_h = np.zeros(ld)
    s.chronos(1, _host(s.mu), _host(s.mut), v_h, dt_h, _host(s.sn), _host(s.vol), c_h)
    s.chronos(1, s.mu, s.mut, s.v, s.dt, s.sn, s.vol, s.cson)
    s.sync()
    rc = case.layout.blocks[0].real_cells()
    assert_equal_bits(dt_h[rc], _host(s.dt)[rc], "chronos dt")
    s.close()


@pytest.mark.parametrize("name", ["box_ns", "box_eu"])
def test_flux_forcing_function(cuda, name):
    """ityprk != 0: u as with ityprk = 0, then ff -= u on the real cells"""
    torch = cuda
    case = SMALL[name]()
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    ld = case.layout.ld
    ns = bool(case.scheme.ns)
    rng = np.random.default_rng(5)
    ff0 = rng.standard_normal(s.u.numel())
    ff = torch.as_tensor(ff0, device=s.dev)
    if ns:
        s.sch_roe(1, s.u, s.v, s.tau, s.sn, s.pression)
    else:
        s.sch_roe_euler(1, s.u, s.v, s.sn, s.pression)
    s.sync()
    u0 = _host(s.u)
    if ns:
        s.sch_roe(1, s.u, s.v, s.tau, s.sn, s.pression, ityprk=1, ff=ff)
    else:
        s.sch_roe_euler(1, s.u, s.v, s.sn, s.pression, ityprk=1, ff=ff)
    s.sync()
    assert_equal_bits(_host(s.u), u0, "u with ityprk = 1")
    want = ff0.copy().reshape(-1, ld)
    rc = real(case)
    want[:5, rc] = want[:5, rc] - u0.reshape(-1, ld)[:5, rc]
    assert_equal_bits(_host(ff).reshape(-1, ld), want, "forcing function")
    s.close()


@pytest.mark.parametrize("name", ["box_ns", "box_eu_qfix"])
def test_implicit_forcing_function(cuda, name):
    """ityprk != 0: the right-hand side -u - ff, i.e. the sweeps of u + ff"""
    torch = cuda
    case = SMALL[name]()
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    if case.scheme.ns:
        s.sch_roe(0, s.u, s.v, s.tau, s.sn, s.pression)
    else:
        s.sch_roe_euler(0, s.u, s.v, s.sn, s.pression)
    s.sync()
    ff = torch.as_tensor(np.random.default_rng(6).standard_normal(s.u.numel()) * 1e-3,
                         device=s.dev)
    v0 = s.v.clone()

    def run(u, **kw):
        s.v.copy_(v0)
        s.d.zero_()
        torch.cuda.synchronize()
        if case.scheme.ns:
            s.implimf_3d(1, u, s.dt, s.v, s.d, s.mu, s.mut, s.sn, s.vol, s.pression, s.cson, 3,
                         **kw)
        else:
            s.implimf_eu(1, u, s.dt, s.v, s.d, s.sn, s.vol, s.pression, s.cson, 3, **kw)
        s.sync()
        return _host(s.v), _host(s.d)

    va, da = run(s.u, ityprk=1, ff=ff)
    vb, db = run((s.u + ff).contiguous())
    rc = case.layout.blocks[0].real_cells()
    ld = case.layout.ld
    assert_equal_bits(va.reshape(-1, ld)[:5, rc], vb.reshape(-1, ld)[:5, rc], "v")
    assert_equal_bits(da.reshape(-1, ld)[:5, rc], db.reshape(-1, ld)[:5, rc], "d")
    s.close()


def test_separate_stress_arrays(cuda):
    torch = cuda
    case = SMALL["channel"]()
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    ld = case.layout.ld
    s.sch_roe(2, s.u, s.v, s.tau, s.sn, s.pression)
    s.sync()
    u_packed = _host(s.u)
    cols = [s.tau[a * ld:(a + 1) * ld].clone() for a in range(9)]  # nine separate arrays
    snp, lg = s._sn(2, s.sn)
    ptrs = [C.c_void_p(t.data_ptr()) for t in cols]
    s.u.fill_(1.0)
    torch.cuda.synchronize()
    rc = s.lib.cns_sch_roe(s.ctx, 2, 0, C.c_void_p(s.u.data_ptr()), C.c_void_p(s.v.data_ptr()),
                           None, *ptrs, b"ns3d   ", snp, lg, *([None] * 10),
                           C.c_void_p(s.pression.data_ptr()))
    assert rc == 0
    s.sync()
    sel = case.layout.blocks[1].real_cells()
    assert_equal_bits(_host(s.u).reshape(-1, ld)[:5, sel], u_packed.reshape(-1, ld)[:5, sel],
                      "separate stress arrays")
    s.close()


def test_chronos_uses_etal(cuda):
    """dt = etal * (...): twice the CFL number gives twice every step exactly"""
    torch = cuda
    case = SMALL["box_ns"]()
    orc, st = _prepared_flow(case)
    s = _gpu(case)
    _load_state(torch, s, st)
    eta = case.scheme.eta
    s.chronos(1, s.mu, s.mut, s.v, s.dt, s.sn, s.vol, s.cson, etal=eta)
    s.sync()
    d1 = _host(s.dt)
    s.chronos(1, s.mu, s.mut, s.v, s.dt, s.sn, s.vol, s.cson, etal=2 * eta)
    s.sync()
    d2 = _host(s.dt)
    rc = real(case)
    assert_equal_bits(d2[rc], 2 * d1[rc], "dt(2 eta)")
    # the context's own eta is back for the next call
    s.chronos(1, s.mu, s.mut, s.v, s.dt, s.sn, s.vol, s.cson)
    s.sync()
    assert_equal_bits(_host(s.dt)[rc], d1[rc], "dt after")
    s.close()


def test_refused_arguments(cuda):
    case = SMALL["box_ns"]()
    s = _gpu(case)
    with pytest.raises(abi.CnsError) as e:
        s.sch_roe(1, s.u, s.v, s.tau, s.sn, s.pression, equat=b"ns2dk  ")
    assert e.value.code == abi.CNS_EINVAL
    with pytest.raises(abi.CnsError) as e:
        s.sch_roe(1, s.u, s.v, s.tau, s.sn, s.pression, ityprk=1, ff=None)
    assert e.value.code == abi.CNS_EINVAL
    snp, lg = s._sn(1, s.sn)
    rc = s.lib.cns_sch_roe_euler(s.ctx, 1, 0, C.c_void_p(s.u.data_ptr()),
                                 C.c_void_p(s.v.data_ptr()), None, b"eu3d   ", snp, lg + 1,
                                 *([None] * 10), C.c_void_p(s.pression.data_ptr()))
    assert rc == abi.CNS_EINVAL
    s.close()
