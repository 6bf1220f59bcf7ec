"""codens_b200 -- B200-native (sm_100a) implementation of the CodeNS
per-iteration hot path: Roe-MUSCL / viscous residual and matrix-free
point-Jacobi implicit update on structured multi-block grids, behind the
C ABI of include/cns_abi.h.

    from codens_b200 import cases, CodeNS
    case = cases.channel_case()
    s = CodeNS(case); s.metric(); norms = s.atsch_num(100)
"""
from . import cases, layout  # noqa: F401
from .cases import Case, box_case, batch_case, channel_case  # noqa: F401


def __getattr__(name):
    # the solver (and torch) load only when asked for
    if name == "CodeNS":
        from .solver import CodeNS
        return CodeNS
    raise AttributeError(name)
