"""CPU tests: the C-ABI library loads and exports every declared symbol, and
the host-side set-up logic (layout, boundary lists, seeded cases)."""
import ctypes
import os
import re

import numpy as np
import pytest

from codens_b200 import cases
from codens_b200.layout import Layout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cns_abi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cns_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from codens_b200 import build
    path = build.build()  # nvcc cross-compiles for sm_100a without a GPU
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    from codens_b200 import abi
    assert set(declared_functions()) == set(abi.EXPORTS)


def test_layout_offsets():
    lay = Layout.from_dims([(5, 4, 3), (3, 3, 3)])
    b0, b1 = lay.blocks
    assert b0.npc == 0 and b1.npc == 7 * 6 * 5
    assert b0.ic(0, 0, 0) == 0 and b0.ic(1, 0, 0) == 1
    assert b0.ic(0, 1, 0) == 7 and b0.ic(0, 0, 1) == 42
    assert lay.nreal == 4 * 3 * 2 + 2 * 2 * 2
    assert lay.ld % 32 == 0 and lay.ld >= lay.ncells


def test_boundary_lists_follow_initis_order():
    case = cases.box_case((4, 3, 2), seed=1)
    ba = case.boundary_arrays()
    b = case.layout.blocks[0]
    # face i1: k outer, j inner; ghost at i = 0; interior at i = 1
    n = ba["mmb"][0]
    assert n == 3 * 2
    exp = [b.ic(0, j, k) for k in (1, 2) for j in (1, 2, 3)]
    assert list(ba["ncbd"][:n]) == exp
    assert list(ba["ncin"][:n]) == [e + 1 for e in exp]
    # face j2: ghost at j = nj, interior j = nj - 1, k outer, i inner
    ib = 3
    sl = slice(ba["mpb"][ib], ba["mpb"][ib] + ba["mmb"][ib])
    exp = [b.ic(i, b.nj, k) for k in (1, 2) for i in (1, 2, 3, 4)]
    assert list(ba["ncbd"][sl]) == exp
    assert list(ba["ncin"][sl]) == [e - b.nid for e in exp]
    # coincident partners are mutual and of equal size
    for i, bd in enumerate(case.boundaries):
        if bd.kind == cases.BC_RC:
            assert case.boundaries[bd.partner].partner == i
            assert ba["mmb"][bd.partner] == ba["mmb"][i]


def test_channel_joins_and_sizes():
    ni, nj, nk, seed = cases.channel_dims(seed=2)
    tot = sum(ni) * nj * nk
    assert 3.5e6 <= tot <= 4.5e6
    assert len(ni) == 8 and all(48 <= n <= 128 for n in ni)
    case = cases.channel_case([5, 4], 3, 2, seed=2)
    kinds = [b.kind for b in case.boundaries]
    assert kinds.count(cases.BC_IDD) == 1 and kinds.count(cases.BC_PRD) == 1
    assert kinds.count(cases.BC_PARA) == 4
    # the join cells line up: ghost of block 0 face i2 sits next to the
    # interior of block 1 face i1 in physical space
    ba = case.boundary_arrays()
    a, b = case.layout.blocks
    g0 = ba["ncin"][ba["mpb"][1]:ba["mpb"][1] + ba["mmb"][1]]  # block1 i1 interior
    assert all(case.x[g] >= 0 for g in g0)


def test_splitmix_deterministic():
    a = cases.splitmix64_uniform(7, 1000)
    b = cases.splitmix64_uniform(7, 1000)
    assert np.array_equal(a, b)
    assert 0.45 < a.mean() < 0.55 and a.min() >= 0 and a.max() < 1
    c = cases.splitmix64_uniform(7, 10, offset=990)
    assert np.array_equal(a[990:], c)


def test_batch_case_shapes():
    case = cases.batch_case(ncase=8, side=(16, 96), seed=4)
    assert case.layout.nblk == 8
    for b, s in zip(case.layout.blocks, case.meta["sides"]):
        assert (b.ni - 1, b.nj - 1, b.nk - 1) == tuple(s)
    assert all(0.3 <= m <= 2.0 for m in case.meta["mach"])
