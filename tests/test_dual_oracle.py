"""CPU tests of the oracle's dual time stepping restatement (sch_duin,
sch_duup, sch_duup2, sch_dual) against their formulas, and a uniform flow
kept through physical steps."""
from __future__ import annotations

import numpy as np
import pytest

from codens_b200 import cases
from oracle.oracle import Oracle, OracleState, lib as orc_lib


def small(kdualns=0):
    c = cases.box_case((6, 5, 4), seed=5, skew=0.02, alpha=1.0)
    c.scheme.kfmg, c.scheme.kdualns, c.scheme.dt1min = 3, kdualns, 0.05
    return c


@pytest.mark.parametrize("kdualns", [0, 2])
def test_physical_step_arrays_follow_their_formulas(kdualns):
    case = small(kdualns)
    orc = Oracle(case)
    st = OracleState(case)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    orc.set_dual(st, kdualns)
    v0 = st.v[:5 * ld].reshape(5, ld)[:, rc].copy()
    assert np.array_equal(st.ptdual.reshape(5, ld)[:, rc], -v0)
    for arr in (st.vdual, st.vdual1, st.vdual2):
        assert np.array_equal(arr.reshape(5, ld)[:, rc], v0)
    rng = np.random.default_rng(1)
    hist = [v0]
    for _ in range(3):
        st.v[:5 * ld].reshape(5, ld)[:, rc] = rng.standard_normal((5, rc.size))
        hist.append(st.v[:5 * ld].reshape(5, ld)[:, rc].copy())
        orc.sch_duup(st)
        vd, vd1 = hist[-1], hist[-2]
        vd2 = hist[-3] if len(hist) >= 3 else hist[0]
        if kdualns == 2:
            want = -3.0 * vd + 1.5 * vd1 - (1.0 / 3.0) * vd2
        else:
            want = -2.0 * vd + 0.5 * vd1
        assert np.array_equal(st.ptdual.reshape(5, ld)[:, rc], want)


def test_sch_dual_formula():
    case = small(0)
    Oracle(case)
    ld = case.layout.ld
    rng = np.random.default_rng(2)
    u, v, pt = (rng.standard_normal(5 * ld) for _ in range(3))
    vol = rng.uniform(0.5, 1.5, ld)
    rc = case.layout.real_cells()
    for icycle, fact in ((1, 1.0), (2, 1.5)):
        got = u.copy()
        orc_lib().orc_set_dual(3, 0, icycle, None)
        orc_lib().orc_sch_dual(1, got, v, icycle, vol, pt)
        c0 = vol[rc] * (1.0 / 0.05)
        want = u.reshape(5, ld)[:, rc] + c0 * (fact * v.reshape(5, ld)[:, rc]
                                               + pt.reshape(5, ld)[:, rc])
        assert np.array_equal(got.reshape(5, ld)[:, rc], want)


def test_uniform_flow_is_kept_by_the_physical_steps():
    case = cases.box_case((6, 5, 4), seed=5, skew=0.02, alpha=1.0, noise=0.0, ns=True)
    case.scheme.kfmg, case.scheme.dt1min = 3, 0.05
    orc = Oracle(case)
    st = OracleState(case)
    orc.metric(st)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    v0 = st.v.reshape(5, ld)[:, rc].copy()
    orc.set_dual(st, 0)
    for icycle in (1, 2, 3):
        orc.set_dual_cycle(icycle)
        for _ in range(3):
            orc.step(st)
        orc.sch_duup(st)
    assert np.max(np.abs(st.v.reshape(5, ld)[:, rc] - v0)) < 1e-12
