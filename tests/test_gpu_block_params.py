"""GPU tests of the per-block scheme values eta(lm), ki2(lm), ki4(lm)
(tcmd_dfpmdtd.f90, tcmd_dfpmdsd.f90): fused iterations against the oracle
with different values on each block."""
from __future__ import annotations

import numpy as np
import pytest

from tests._helpers import SMALL, assert_equal_bits, max_rel_cols, oracle_prepared, real
from tests.test_gpu_parity import _gpu, _n

pytestmark = pytest.mark.gpu


def _steps(case, n, exact):
    orc, st = oracle_prepared(case)
    s = _gpu(case)
    ld = case.layout.ld
    rc = real(case)
    for it in range(n):
        orc.step(st)
        s.atsch_num(1)
        vg = _n(s.v).reshape(5, ld)[:, rc]
        vo = st.v.reshape(5, ld)[:, rc]
        if exact:
            assert_equal_bits(vg, vo, f"v after step {it}")
        else:
            assert max_rel_cols(vg, vo) <= 1e-12, f"step {it}"
    s.close()
    return vg


def test_per_block_eta_channel(cuda):
    case = SMALL["channel"]()
    case.scheme.eta_l = [2.0, 5.0, 3.5]
    v_blocks = _steps(case, 5, exact=False)
    uniform = SMALL["channel"]()
    uniform.scheme.eta = 5.0
    v_uniform = _steps(uniform, 5, exact=False)
    assert not np.array_equal(v_blocks, v_uniform)


def test_per_block_jameson_coefficients(cuda):
    case = SMALL["batch"]()
    case.scheme.ischema = 1
    case.scheme.eta_l = [1.5, 2.5, 3.0, 2.0]
    case.scheme.ki2_l = [0.5, 0.25, 0.75, 0.5]
    case.scheme.ki4_l = [1.0 / 32.0, 0.05, 0.02, 0.04]
    _steps(case, 4, exact=True)
