"""Batching: many independent cases in one layout run in the same launches
(tile work lists over uneven blocks, one graph per iteration).  Each case's
state after the batched iterations equals, bit for bit, the state of that
case run alone (FP64); the mixed form agrees to FP32-sweep accuracy."""
import numpy as np
import pytest

from codens_b200 import cases

from ._helpers import assert_equal_bits, max_rel_cols

pytestmark = pytest.mark.gpu


def _run(case, nsteps, precision=0):
    from codens_b200.solver import CodeNS
    case.scheme.precision = precision
    s = CodeNS(case)
    s.metric()
    s.atsch_num(nsteps)
    v = s.v.cpu().numpy().reshape(5, case.layout.ld)
    s.close()
    return v


@pytest.mark.parametrize("precision", [0, 1])
def test_batched_equals_one_at_a_time(cuda, precision):
    bt = cases.batch_case(ncase=6, side=(4, 14), seed=21, qfix_dfez=1)
    vb = _run(bt, 5, precision)
    for ib in range(bt.layout.nblk):
        m = cases.batch_member(bt, ib)
        vm = _run(m, 5, precision)
        a = vb[:, bt.layout.blocks[ib].real_cells()]
        b = vm[:, m.layout.blocks[0].real_cells()]
        if precision == 0:
            assert_equal_bits(a, b, f"case {ib}")
        else:
            assert max_rel_cols(a, b) < 1e-5, f"case {ib}"
