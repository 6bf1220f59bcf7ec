"""GPU tests of the command-deck subset: a deck read with its grid file and
finia1 runs the case the oracle runs from the same files, with the time
step kept between the iterations ncychro / icychr0 select, and a second
deck restarts from the saved fac."""
from __future__ import annotations

import numpy as np
import pytest

from codens_b200 import cases
from codens_b200.deck import Deck
from oracle.oracle import Oracle, OracleState, lib as orc_lib
from tests.test_deck import BOX_DECK

pytestmark = pytest.mark.gpu


def dt_due(n, ncychro, icychr0):
    return ncychro <= 1 or n % ncychro == 1 or n < icychr0


def _n(t):
    return t.detach().cpu().numpy()


def test_deck_run_matches_the_oracle_and_restarts(cuda, tmp_path):
    box = cases.box_case((10, 8, 5), ns=True, ilim=1, skew=0.02, alpha=-3.0)
    lay = box.layout
    assert orc_lib().orc_setup(lay.nblk, lay.dims_array(), lay.ld) == 0
    assert Oracle.writdg(str(tmp_path / "fgv"), "cvcv", box.x, box.y, box.z) == 0
    (tmp_path / "finia1").write_text("0.8 -3. 0.\n")
    (tmp_path / "flec").write_text(BOX_DECK)
    deck = Deck(str(tmp_path / "flec"))
    run = deck.run()
    s = run.solver
    case = deck.case()
    ld = lay.ld
    rc = lay.real_cells()
    # the oracle from the deck's initial state (saved before compute flow)
    orc = Oracle(case)
    st = OracleState(case)
    st.x[:], st.y[:], st.z[:] = box.x, box.y, box.z
    orc.metric(st)
    st.v[:] = 0.0
    assert Oracle.readda(str(tmp_path / "fac"), "ns3d   ", st.v, st.mut) == 0
    for n in range(1, deck.ncycle + 1):
        orc.step(st, compute_dt=dt_due(n, 2, 3))
    v_gpu = _n(s.v).reshape(5, ld)[:, rc]
    assert np.array_equal(v_gpu, st.v.reshape(5, ld)[:, rc])
    # restart: a second deck reads fac (the same initial state) and runs on
    restart = BOX_DECK.replace("init dom csvmut * 1\nsave dom csvmut cccc\n",
                               "init dom csvmut * 0\n")
    (tmp_path / "flec2").write_text(restart)
    run2 = Deck(str(tmp_path / "flec2")).run()
    assert np.array_equal(_n(run2.solver.v).reshape(5, ld)[:, rc], v_gpu)
    np.testing.assert_array_equal(run2.norms[-1], run.norms[-1])
    s.close()
    run2.solver.close()


@pytest.mark.parametrize("ncychro,icychr0", [(3, 0), (4, 3)])
def test_time_step_update_frequency_parity(cuda, ncychro, icychr0):
    """atsch_num.f90:173-178, 436: the fused iterations recompute dt only on
    the selected iterations, FP64 bit for bit with the oracle"""
    from codens_b200.solver import CodeNS
    from tests._helpers import oracle_prepared
    case = cases.box_case((10, 8, 5), ns=True, ilim=1, skew=0.02, alpha=-3.0, seed=12)
    case.scheme.ncychro, case.scheme.icychr0 = ncychro, icychr0
    orc, st = oracle_prepared(case)
    s = CodeNS(case)
    ld = case.layout.ld
    rc = case.layout.real_cells()
    for n in range(1, 9):
        orc.step(st, compute_dt=dt_due(n, ncychro, icychr0))
    s.atsch_num(3)
    s.atsch_num(5)
    assert np.array_equal(_n(s.v).reshape(5, ld)[:, rc], st.v.reshape(5, ld)[:, rc])
    s.close()


def test_time_step_frequency_in_the_mixed_form(cuda):
    """the reduced-precision graphs have their dt-kept variants too"""
    from codens_b200.solver import CodeNS
    case = cases.box_case((10, 8, 5), ns=True, ilim=1, skew=0.02, alpha=-3.0, seed=12)
    case.scheme.ncychro, case.scheme.precision = 2, 1
    s = CodeNS(case)
    n = s.atsch_num(6)
    assert np.all(np.isfinite(n))
    assert s.kernels_launched > 0
    s.close()


def test_dual_time_deck_runs_the_physical_time_loop(cuda, tmp_path):
    """a deck with fmg 3 / dual runs smg_num's physical time loop: the same
    as CodeNS.dual_time from the deck's saved initial state, bit for bit"""
    from codens_b200.solver import CodeNS
    box = cases.box_case((10, 8, 5), ns=True, ilim=1, skew=0.02, alpha=-3.0)
    lay = box.layout
    assert orc_lib().orc_setup(lay.nblk, lay.dims_array(), lay.ld) == 0
    assert Oracle.writdg(str(tmp_path / "fgv"), "cvcv", box.x, box.y, box.z) == 0
    (tmp_path / "finia1").write_text("0.8 -3. 0.\n")
    text = BOX_DECK.replace("define numerics schema 7 muscl 1 -1. 1",
                            "define numerics schema 7 muscl 1 -1. 1 fmg 3 1 0 "
                            "dual 0 1.e-2 6 1.e-3 10")
    text = text.replace("define pm_dtg kdtl 1 icychr0 3 ncychro 2",
                        "define pm_dtg kdtl 1 icychr0 3 ncychro 2 dt1min 0.02")
    (tmp_path / "flec").write_text(text)
    deck = Deck(str(tmp_path / "flec"))
    run = deck.run()
    s2 = CodeNS(deck.case())
    s2.readdg(str(tmp_path / "fgv"))
    s2.readda(str(tmp_path / "fac"), "ns3d   ")
    counts = s2.dual_time(deck.ncycle, deck.dual_niter, deck.dual_tol)
    assert run.inner == [counts]
    rc = lay.real_cells()
    assert np.array_equal(_n(run.solver.v).reshape(5, lay.ld)[:, rc],
                          _n(s2.v).reshape(5, lay.ld)[:, rc])
    run.solver.close()
    s2.close()
