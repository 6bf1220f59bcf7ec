"""Reduced-precision forms of the fused iteration.

precision 1 (mixed): FP64 residual (face fluxes with FMA contraction),
boundary conditions, update and norms, FP32 point-Jacobi sweeps.  Its fixed
point is the FP64 steady state, so the converged state must agree with the
FP64 one to far below FP32 rounding.

precision 2 (defect correction): FP32 face fluxes, the FP64 residual every
kdefect iterations.  Its refresh iteration must use the FP64 residual.
"""
from __future__ import annotations

import numpy as np
import pytest

from codens_b200 import cases

from ._helpers import SMALL, real, state_err

pytestmark = pytest.mark.gpu

# state agreement of the converged mixed and FP64 iterations (component-
# relative); FP32 sweeps alone would leave ~1e-7
STEADY_TOL = 1e-8


def _solver(case, precision, kdefect=4):
    from codens_b200.solver import CodeNS
    case.scheme.precision = precision
    case.scheme.kdefect = kdefect
    s = CodeNS(case)
    s.metric()
    return s


def _state(s, case):
    return s.v.cpu().numpy().reshape(5, case.layout.ld)[:, real(case)]


def _residual(s, case):
    return s.u.cpu().numpy().reshape(5, case.layout.ld)[:, real(case)]


def _box_viscous():
    return cases.box_case((8, 6, 5), seed=12, ns=True, ilim=0, reynz=100.0, skew=0.02)


def _duct():
    # inlet (idd) and outlet (prd) only, j and k periodic: a unique steady
    # state (the uniform flow the inlet and outlet values set)
    return cases.channel_case([6, 8, 5], 6, 4, seed=5, reynz=100.0, ilim=0, bump=0.0,
                              walls=False)


def _assert_fp64_close(got, want, what):
    # FP64 residual with fused multiply-adds against the bit-exact one:
    # rounding-level differences, relative to each component's scale
    scale = np.maximum(np.abs(want).max(axis=1, keepdims=True), 1e-300)
    err = float((np.abs(got - want) / scale).max())
    assert err < 1e-12, (what, err)


@pytest.mark.parametrize("name", ["box_ns", "channel", "box_eu_qfix"])
def test_mixed_uses_fp64_residual(cuda, name):
    """the first mixed iteration evaluates the FP64 residual (its face fluxes
    compiled with FMA contraction: the FP64 iteration's residual to FP64
    rounding) and moves the state by an FP32-accurate step"""
    case = SMALL[name]()
    a = _solver(case, 0)
    b = _solver(SMALL[name](), 1)
    v0 = _state(a, case)
    a.atsch_num(1)
    b.atsch_num(1)
    _assert_fp64_close(_residual(b, case), _residual(a, case), "residual of the first step")
    dv64 = _state(a, case) - v0
    dv32 = _state(b, case) - v0
    scale = np.maximum(np.abs(dv64).max(axis=1, keepdims=True), 1e-300)
    assert float((np.abs(dv32 - dv64) / scale).max()) < 1e-4
    a.close()
    b.close()


def test_defect_refresh_uses_fp64_residual(cuda):
    case = SMALL["box_ns"]()
    a = _solver(case, 0)
    b = _solver(SMALL["box_ns"](), 2, kdefect=3)
    a.atsch_num(1)
    b.atsch_num(1)
    _assert_fp64_close(_residual(b, case), _residual(a, case), "refresh residual")
    # the regular iterations run on R32 + corr: finite and close to FP64
    b.atsch_num(2)
    assert np.isfinite(_state(b, case)).all()
    a.close()
    b.close()


def test_mixed_reaches_fp64_steady_state(cuda):
    """2400 iterations on a viscous box: both forms converge (L2 of the
    density increment below 1e-12), and the mixed converged state is a fixed
    point of the FP64 iteration (one FP64 iteration from it moves the state by
    FP64 rounding only).  The box's extrapolated i faces leave a family of
    steady states, so the two states themselves may differ by the path."""
    case = _box_viscous()
    a = _solver(case, 0)
    b = _solver(_box_viscous(), 1)
    na = a.atsch_num(2400)
    nb = b.atsch_num(2400)
    assert na[1, 0] < 1e-12 and nb[1, 0] < 1e-12, (na[1, 0], nb[1, 0])
    case_b = _box_viscous()
    case_b.scheme.precision = 0
    b.set_scheme(case_b.scheme)
    n1 = b.atsch_num(1)
    assert n1[1, 0] < 1e-14, n1[1, 0]
    a.close()
    b.close()


def test_mixed_matches_fp64_converged_state(cuda):
    """a case with a unique steady state: 4500 iterations converge both
    forms to FP64 rounding, and the states agree within STEADY_TOL"""
    case = _duct()
    a = _solver(case, 0)
    b = _solver(_duct(), 1)
    na = a.atsch_num(4500)
    nb = b.atsch_num(4500)
    assert na[1, 0] < 1e-13 and nb[1, 0] < 1e-13, (na[1, 0], nb[1, 0])
    err = state_err(_state(b, case), _state(a, case))
    assert err <= STEADY_TOL, err
    a.close()
    b.close()


def test_mixed_rejects_bad_precision(cuda):
    from codens_b200 import abi
    case = SMALL["box_ns"]()
    s = _solver(case, 0)
    case.scheme.precision = 3
    with pytest.raises(abi.CnsError) as ei:
        s.set_scheme(case.scheme)
    assert ei.value.code == abi.CNS_EINVAL
    case.scheme.precision = 2
    case.scheme.kdefect = 0
    with pytest.raises(abi.CnsError) as ei:
        s.set_scheme(case.scheme)
    assert ei.value.code == abi.CNS_EINVAL
    s.close()


def test_create_rejects_a_block_of_2_31_cells(cuda):
    """the kernels index a block's cells with 32-bit offsets: cns_create
    refuses a block whose (ni+2)(nj+2)(nk+2) reaches 2^31, before it
    allocates anything"""
    import ctypes as C
    from codens_b200 import abi
    s = _solver(SMALL["box_ns"](), 1)
    dims = np.array([2000, 1100, 1000], dtype=np.int32)
    lay = abi.Layout_t(1, dims.ctypes.data_as(C.POINTER(C.c_int32)), 0)
    ctx = C.c_void_p()
    rc = s.lib.cns_create(C.byref(lay), C.byref(s._phys), C.byref(s._scheme),
                          C.byref(s._bnd), C.byref(ctx))
    assert rc == abi.CNS_EINVAL and not ctx.value
    s.close()
