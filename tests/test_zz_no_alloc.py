"""The no-allocation entry point (cns_sch_roe_euler_noalloc), through the C
ABI.  It exists for callers that cannot let the library allocate device
memory (a driver owning every device array in its own pool, or running under
a hard memory cap); its intermediates live in a fixed static device array.
Its residual must equal the regular entry point's, bit for bit, on two calls
in a row (the static array keeps the previous call's contents), and calls
larger than the array must be refused before anything runs.

This file is collected last so that a failure here comes after every other
test has run; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from codens_b200 import cases

pytestmark = pytest.mark.gpu


def _inputs(case):
    from codens_b200.solver import CodeNS
    s = CodeNS(case)
    s.metric()
    s.zpres(0, s.v, s.pression, s.ztemp, s.cson)
    s.rbord(s.v, s.pression, s.ztemp, s.cson)
    s.sch_roe_euler(1, s.u, s.v, s.sn, s.pression)
    s.sync()
    return s


def _call(s, case, u, ld=None):
    b = case.layout.blocks[0]
    p, sc = case.phys, case.scheme
    return s.lib.cns_sch_roe_euler_noalloc(
        b.ni, b.nj, b.nk, case.layout.ld if ld is None else ld, p.gam, p.pinfl,
        sc.muscl, sc.xk, C.c_void_p(u.data_ptr()), C.c_void_p(s.v.data_ptr()),
        C.c_void_p(s.sn.data_ptr()), C.c_void_p(s.pression.data_ptr()),
        C.c_void_p(s.stream.cuda_stream))


@pytest.mark.parametrize("cells,pinfl,muscl,xk", [((12, 7, 6), 0.0, 1, -1.0),
                                                   ((30, 20, 16), 0.25, 1, -1.0),
                                                   ((12, 7, 6), 0.0, 0, -1.0),
                                                   ((10, 9, 7), 0.1, 1, 1.0 / 3.0)])
def test_noalloc_matches_regular_entry_point(cuda, cells, pinfl, muscl, xk):
    """first-order (muscl 0) and two kappa values of the MUSCL scheme, each
    against the regular entry point run with the same scheme"""
    torch = cuda
    case = cases.box_case(cells, seed=31, skew=0.02, alpha=3.0, pinfl=pinfl)
    case.scheme.muscl = muscl
    case.scheme.xk = xk
    s = _inputs(case)
    ref = s.u.clone()
    rc = case.layout.real_cells()
    ld = case.layout.ld
    for call in range(2):
        u = torch.full_like(s.u, float("nan"))
        torch.cuda.synchronize()
        assert _call(s, case, u) == 0
        s.sync()
        a = u.cpu().numpy().reshape(5, ld)[:, rc]
        b = ref.cpu().numpy().reshape(5, ld)[:, rc]
        assert np.array_equal(a, b), f"call {call}: residual differs"
        # the whole block is zeroed first, as the reference does
        blk = slice(0, case.layout.blocks[0].nnn)
        assert np.all(np.isfinite(u.cpu().numpy().reshape(5, ld)[:, blk]))
    s.close()


def test_noalloc_allocates_nothing(cuda):
    """after a first call (which loads the module and looks up the static
    array's address), further calls leave the device's free memory as it was"""
    torch = cuda
    case = cases.box_case((20, 14, 10), seed=33, skew=0.02, alpha=1.0)
    s = _inputs(case)
    u = torch.zeros_like(s.u)
    assert _call(s, case, u) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        assert _call(s, case, u) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    s.close()


def _call_dims(s, u, ni, nj, nk, ld):
    return s.lib.cns_sch_roe_euler_noalloc(
        ni, nj, nk, ld, 1.4, 0.0, 1, -1.0, C.c_void_p(u.data_ptr()),
        C.c_void_p(s.v.data_ptr()), C.c_void_p(s.sn.data_ptr()),
        C.c_void_p(s.pression.data_ptr()), C.c_void_p(s.stream.cuda_stream))


def test_noalloc_rejects_oversize(cuda):
    torch = cuda
    case = cases.box_case((8, 6, 5), seed=32)
    s = _inputs(case)
    u = torch.zeros_like(s.u)
    assert _call(s, case, u, ld=131072 + 1) == 1          # beyond the static array
    assert _call(s, case, u, ld=case.layout.blocks[0].nnn - 1) == 1  # arrays too short
    # sides whose ghosted size overflows 32-bit arithmetic or the array alone
    big = 2**31 - 1
    for dims in ((big, 4, 4), (4, big, 4), (4, 4, big), (131071, 3, 3), (60, 60, 60)):
        assert _call_dims(s, u, *dims, 131072) == 1, dims
    s.sync()
    assert bool((u == 0).all())  # nothing was launched
    s.close()
