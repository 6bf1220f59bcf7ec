"""GPU tests of the reference's grid and flow files through the C-ABI:
the golden files written and read byte for byte, the oracle's files at the
channel workload's full size, error cases that leave the arrays untouched,
and a restart through fac that continues the iteration bit for bit."""
from __future__ import annotations

import os
import struct

import numpy as np
import pytest

from codens_b200 import abi, cases
from codens_b200.layout import Layout
from oracle.oracle import Oracle, lib as orc_lib
from tests._helpers import SMALL
from tests.golden import file_fixtures as ff

pytestmark = pytest.mark.gpu
GOLDEN = os.path.dirname(ff.__file__)


def golden(name):
    return open(os.path.join(GOLDEN, name), "rb").read()


def fixture_solver():
    from codens_b200.solver import CodeNS
    lay = Layout.from_dims(ff.DIMS)
    z = np.zeros(lay.ld)
    case = cases.Case("files", lay, cases.Phys(), cases.Scheme(ns=1), [], z, z.copy(),
                      z.copy(), np.zeros((7, lay.ld)))
    return CodeNS(case)


def _n(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("entry", ff.FILES, ids=[f[0] for f in ff.FILES])
def test_writers_produce_the_golden_bytes(cuda, entry, tmp_path):
    torch = cuda
    name, kind, disc, equat, maxsub = entry
    s = fixture_solver()
    lay = s.case.layout
    s.set_subrecord_length(maxsub)
    out = str(tmp_path / name)
    if kind == "grid":
        for dst, src in zip((s.x, s.y, s.z), ff.fill_nodes(lay)):
            dst.copy_(torch.as_tensor(src))
        s.writdg(out, disc)
    else:
        v, mut = ff.fill_cells(lay)
        s.v.copy_(torch.as_tensor(v.reshape(-1)))
        s.mut.copy_(torch.as_tensor(mut))
        s.writda(out, equat, disc)
    assert open(out, "rb").read() == golden(name)
    s.close()


@pytest.mark.parametrize("entry", [f for f in ff.FILES if f[2] in ("cvcv", "cccc")],
                         ids=[f[0] for f in ff.FILES if f[2] in ("cvcv", "cccc")])
def test_readers_match_the_golden_files(cuda, entry):
    name, kind, disc, equat, maxsub = entry
    s = fixture_solver()
    lay = s.case.layout
    path = os.path.join(GOLDEN, name)
    if kind == "grid":
        for a in (s.x, s.y, s.z):
            a.fill_(-7.0)
        s.readdg(path)
        want = ff.fill_nodes(lay)
        idx = ff.box_index(lay, 0)
        rest = np.setdiff1d(np.arange(lay.ld), idx)
        for c, a in enumerate((s.x, s.y, s.z)):
            got = _n(a)
            assert np.array_equal(got[idx], want[c][idx])
            assert np.all(got[rest] == -7.0)
    else:
        s.v.fill_(-7.0)
        s.mut.fill_(-7.0)
        s.readda(path, equat)
        wv, wmut = ff.fill_cells(lay)
        idx = ff.box_index(lay, 1)
        v = _n(s.v).reshape(7, lay.ld)
        eq = equat.ljust(7)
        ncol = 7 if eq[5:7] == "ke" else 5
        for a in range(ncol):
            assert np.array_equal(v[a, idx], wv[a, idx])
        for a in range(ncol, 7):
            assert np.all(v[a] == -7.0)
        mut = _n(s.mut)
        if eq[:2] == "ns":
            assert np.array_equal(mut[idx], wmut[idx])
        else:
            assert np.all(mut == -7.0)
    s.close()


def test_keinit_zeroes_the_transport_columns(cuda):
    s = fixture_solver()
    lay = s.case.layout
    s.v.fill_(3.0)
    s.readda(os.path.join(GOLDEN, "fac_2blk_ns.bin"), "ns3d ke", keinit=1)
    v = _n(s.v).reshape(7, lay.ld)
    idx = ff.box_index(lay, 1)
    rest = np.setdiff1d(np.arange(lay.ld), idx)
    assert np.all(v[5:, idx] == 0.0) and np.all(v[5:, rest] == 3.0)
    wv, _ = ff.fill_cells(lay)
    assert np.array_equal(v[:5, idx], wv[:5, idx])
    s.close()


def test_read_errors_leave_the_arrays_untouched(cuda, tmp_path):
    s = fixture_solver()
    s.v.fill_(5.0)
    s.mut.fill_(5.0)
    good = golden("fac_2blk_ns.bin")
    p = tmp_path / "bad"

    def code_of(path, equat):
        with pytest.raises(abi.CnsError) as e:
            s.readda(path, equat)
        return e.value.code

    assert code_of(str(tmp_path / "none"), "ns3d   ") == abi.CNS_EIO
    p.write_bytes(good[:-10])
    assert code_of(str(p), "ns3d   ") == abi.CNS_EFORMAT
    bad = bytearray(good)
    bad[100:104] = struct.pack("<i", 95)
    p.write_bytes(bytes(bad))
    assert code_of(str(p), "ns3d   ") == abi.CNS_EFORMAT
    assert code_of(os.path.join(GOLDEN, "fac_2blk_eu.bin"), "ns3d   ") == abi.CNS_EFORMAT
    assert np.all(_n(s.v) == 5.0) and np.all(_n(s.mut) == 5.0)
    with pytest.raises(abi.CnsError) as e:
        s.writdg(str(tmp_path / "g"), "cvxx")
    assert e.value.code == abi.CNS_EINVAL
    with pytest.raises(abi.CnsError) as e:
        s.writda(str(tmp_path / "f"), "ns3d   ", "cccv")
    assert e.value.code == abi.CNS_EINVAL
    with pytest.raises(abi.CnsError) as e:
        s.set_subrecord_length(0)
    assert e.value.code == abi.CNS_EINVAL
    s.close()


def test_a_longer_record_is_read_up_to_its_need(cuda, tmp_path):
    s = fixture_solver()
    lay = s.case.layout
    recs = ff.records("flow", "cccc", "eu3d   ")
    p = tmp_path / "long"
    p.write_bytes(b"".join(ff.frame(np.append(r, [1.5, 2.5]).astype("<f8").tobytes(), 1 << 30)
                           for r in recs))
    s.readda(str(p), "eu3d   ")
    wv, _ = ff.fill_cells(lay)
    idx = ff.box_index(lay, 1)
    assert np.array_equal(_n(s.v).reshape(7, lay.ld)[:5, idx], wv[:5, idx])
    s.close()


def test_channel_files_match_the_oracle_at_full_size(cuda, tmp_path):
    """the channel workload (8 blocks, about 4M cells): fac (with mut) and
    fgcf written by the GPU equal the oracle's files byte for byte, and fac
    read back restores every real cell"""
    torch = cuda
    from codens_b200.solver import CodeNS
    case = cases.channel_case()
    lay = case.layout
    s = CodeNS(case)
    s.metric()   # extrapolates the ghost nodes that fgcf's centres use
    g = torch.Generator(device=s.dev).manual_seed(7)
    s.v.copy_(torch.rand(s.v.numel(), generator=g, device=s.dev, dtype=torch.float64))
    s.mut.copy_(torch.rand(s.mut.numel(), generator=g, device=s.dev, dtype=torch.float64))
    fa, fb = str(tmp_path / "fac_gpu"), str(tmp_path / "fac_orc")
    s.writda(fa, "ns3d   ")
    v, mut = _n(s.v), _n(s.mut)
    assert orc_lib().orc_setup(lay.nblk, lay.dims_array(), lay.ld) == 0
    assert Oracle.writda(fb, "cccc", "ns3d   ", v, mut) == 0
    assert os.path.getsize(fa) == 6 * (8 * lay.nreal + 8 * lay.nblk)
    assert open(fa, "rb").read() == open(fb, "rb").read()
    ga, gb = str(tmp_path / "fgcf_gpu"), str(tmp_path / "fgcf_orc")
    s.writdg(ga, "cvcf")
    assert Oracle.writdg(gb, "cvcf", _n(s.x), _n(s.y), _n(s.z)) == 0
    assert open(ga, "rb").read() == open(gb, "rb").read()
    s.v.zero_()
    s.mut.zero_()
    s.readda(fb, "ns3d   ")
    rc = lay.real_cells()
    assert np.array_equal(_n(s.v).reshape(5, lay.ld)[:, rc], v.reshape(5, lay.ld)[:, rc])
    assert np.array_equal(_n(s.mut)[rc], mut[rc])
    s.close()


@pytest.mark.parametrize("name", ["channel", "box_ns"])
def test_restart_through_fac_continues_bit_for_bit(cuda, name, tmp_path):
    """iterate, save fac (svfw), restart a fresh solver from it (readda) and
    iterate on: the state equals the uninterrupted run's bit for bit, since
    every ghost cell is rebuilt from the real cells each iteration"""
    from codens_b200.solver import CodeNS
    case = SMALL[name]()
    equat = "ns3d   " if case.scheme.ns else "eu3d   "
    a = CodeNS(case)
    a.atsch_num(5)
    path = str(tmp_path / "fac")
    a.writda(path, equat)
    na = a.atsch_num(5)
    b = CodeNS(case)
    b.readda(path, equat)
    nb = b.atsch_num(5)
    rc = case.layout.real_cells()
    ld = case.layout.ld
    assert np.array_equal(_n(a.v).reshape(5, ld)[:, rc], _n(b.v).reshape(5, ld)[:, rc])
    np.testing.assert_array_equal(na, nb)
    a.close()
    b.close()
