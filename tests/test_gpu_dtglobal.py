"""The global time step (kdtl = 0, chrono.f90:113-151) in the fused
iteration and as its own entry point, against the oracle; the reference's
stop when the step falls below dt1min becomes CNS_EDT."""
import numpy as np
import pytest

from oracle.oracle import lib as orc_lib

from ._helpers import SMALL, assert_equal_bits, oracle_prepared, real

pytestmark = pytest.mark.gpu


def _min_local_dt(case):
    orc, st = oracle_prepared(case)
    L = orc_lib()
    for l in range(1, case.layout.nblk + 1):
        L.orc_zpres(l, st.v, st.ps, st.temp, st.cson)
        if case.scheme.ns:
            L.orc_zvismo(l, st.mu, st.temp)
        L.orc_chronos(l, st.mu, st.mut, st.v, st.dt, st.sn, st.vol, st.cson)
    return float(st.dt[real(case)].min()), float(st.dt[real(case)].max())


@pytest.mark.parametrize("name", ["box_ns", "box_eu_qfix"])
def test_global_dt_fused_parity(cuda, name):
    from codens_b200.solver import CodeNS
    case = SMALL[name]()
    lo, _ = _min_local_dt(case)
    case.scheme.kdtl = 0
    case.scheme.dt1min = 0.5 * lo
    orc, st = oracle_prepared(case)
    s = CodeNS(case)
    s.metric()
    ld = case.layout.ld
    rc = real(case)
    for it in range(4):
        u0 = st.v.copy()
        orc.step(st)
        no = orc.norms(u0, st)
        ng = s.atsch_num(1)
        assert_equal_bits(s.v.cpu().numpy().reshape(5, ld)[:, rc], st.v.reshape(5, ld)[:, rc],
                          f"v after step {it}")
        n = case.layout.ncells
        assert_equal_bits(s.dt.cpu().numpy()[:n], st.dt[:n], f"dt after step {it}")
        np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0)
    s.close()


def test_global_dt_below_dt1min_is_an_error(cuda):
    from codens_b200 import abi
    from codens_b200.solver import CodeNS
    case = SMALL["box_ns"]()
    _, hi = _min_local_dt(case)
    case.scheme.kdtl = 0
    case.scheme.dt1min = 10.0 * hi
    s = CodeNS(case)
    s.metric()
    with pytest.raises(abi.CnsError) as ei:
        s.atsch_num(1)
    assert ei.value.code == abi.CNS_EDT
    s.close()
