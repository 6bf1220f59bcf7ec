"""CPU tests of the reference's grid and flow files: the golden files, and
the oracle's restatement of readdg / svgr / readda / svfw read and written
against them (including gfortran's subrecords and the error cases)."""
from __future__ import annotations

import hashlib
import json
import os
import struct

import numpy as np
import pytest

from codens_b200.layout import Layout
from oracle.oracle import Oracle, lib as orc_lib
from tests.golden import file_fixtures as ff

GOLDEN = os.path.dirname(ff.__file__)
MANIFEST = json.load(open(os.path.join(GOLDEN, "files.json")))
ENTRIES = {e["file"]: e for e in MANIFEST["files"]}


def layout():
    lay = Layout.from_dims(ff.DIMS)
    assert orc_lib().orc_setup(lay.nblk, lay.dims_array(), lay.ld) == 0
    return lay


def golden(name):
    return open(os.path.join(GOLDEN, name), "rb").read()


def test_golden_files_match_their_manifest_and_generator():
    assert MANIFEST["dims"] == [list(d) for d in ff.DIMS]
    for name, kind, disc, equat, maxsub in ff.FILES:
        data = golden(name)
        e = ENTRIES[name]
        assert hashlib.sha256(data).hexdigest() == e["sha256"]
        assert data == ff.file_bytes(kind, disc, equat, maxsub)


def test_record_framing_follows_gfortran_subrecords():
    data = golden("fac_2blk_ke_sub20.bin")
    # block 1's first record: 3*2*2 cells = 96 bytes in 20-byte subrecords
    marks, pos = [], 0
    for _ in range(5):
        lead = struct.unpack_from("<i", data, pos)[0]
        trail = struct.unpack_from("<i", data, pos + 4 + abs(lead))[0]
        marks.append((lead, trail))
        pos += 8 + abs(lead)
    assert marks == [(-20, 20), (-20, -20), (-20, -20), (-20, -20), (16, -16)]
    # the single-subrecord form: both markers hold the byte count
    d2 = golden("fac_2blk_ns.bin")
    assert struct.unpack_from("<ii", d2, 0)[0] == 96
    assert struct.unpack_from("<i", d2, 100)[0] == 96


@pytest.mark.parametrize("entry", ff.FILES, ids=[f[0] for f in ff.FILES])
def test_oracle_writes_the_golden_bytes(entry, tmp_path):
    name, kind, disc, equat, maxsub = entry
    lay = layout()
    out = str(tmp_path / name)
    if kind == "grid":
        x, y, z = ff.fill_nodes(lay)
        assert Oracle.writdg(out, disc, x, y, z, maxsub) == 0
    else:
        v, mut = ff.fill_cells(lay)
        assert Oracle.writda(out, disc, equat, v.reshape(-1), mut, maxsub) == 0
    assert open(out, "rb").read() == golden(name)


@pytest.mark.parametrize("entry", [f for f in ff.FILES if f[2] in ("cvcv", "cccc")],
                         ids=[f[0] for f in ff.FILES if f[2] in ("cvcv", "cccc")])
def test_oracle_reads_the_golden_files(entry):
    name, kind, disc, equat, maxsub = entry
    lay = layout()
    path = os.path.join(GOLDEN, name)
    if kind == "grid":
        got = [np.full(lay.ld, -7.0) for _ in range(3)]
        assert Oracle.readdg(path, *got) == 0
        want = ff.fill_nodes(lay)
        idx = ff.box_index(lay, 0)
        rest = np.setdiff1d(np.arange(lay.ld), idx)
        for c in range(3):
            assert np.array_equal(got[c][idx], want[c][idx])
            assert np.all(got[c][rest] == -7.0)
    else:
        v = np.full(7 * lay.ld, -7.0)
        mut = np.full(lay.ld, -7.0)
        assert Oracle.readda(path, equat, v, mut) == 0
        wv, wmut = ff.fill_cells(lay)
        idx = ff.box_index(lay, 1)
        v = v.reshape(7, lay.ld)
        eq = equat.ljust(7)
        ncol = 7 if eq[5:7] == "ke" else 5
        for a in range(ncol):
            assert np.array_equal(v[a, idx], wv[a, idx])
        for a in range(ncol, 7):
            assert np.all(v[a] == -7.0)
        if eq[:2] == "ns":
            assert np.array_equal(mut[idx], wmut[idx])
        else:
            assert np.all(mut == -7.0)


def test_oracle_keinit_zeroes_the_transport_columns():
    """readda.f90:123-131: equat 'ke' with keinit >= 1 reads no v6, v7 records
    and zeroes both on the real cells"""
    lay = layout()
    v = np.full(7 * lay.ld, 3.0)
    mut = np.zeros(lay.ld)
    assert Oracle.readda(os.path.join(GOLDEN, "fac_2blk_ns.bin"), "ns3d ke", v, mut, 1) == 0
    v = v.reshape(7, lay.ld)
    idx = ff.box_index(lay, 1)
    assert np.all(v[5:, idx] == 0.0)
    rest = np.setdiff1d(np.arange(lay.ld), idx)
    assert np.all(v[5:, rest] == 3.0)


def test_oracle_file_errors(tmp_path):
    lay = layout()
    v = np.zeros(7 * lay.ld)
    mut = np.zeros(lay.ld)
    good = golden("fac_2blk_ns.bin")
    # missing file
    assert Oracle.readda(str(tmp_path / "none"), "ns3d   ", v, mut) == 8
    # truncated inside the last record
    p = tmp_path / "cut"
    p.write_bytes(good[:-10])
    assert Oracle.readda(str(p), "ns3d   ", v, mut) == 9
    # a trailing marker that disagrees with its leading one
    bad = bytearray(good)
    bad[100:104] = struct.pack("<i", 95)
    p.write_bytes(bytes(bad))
    assert Oracle.readda(str(p), "ns3d   ", v, mut) == 9
    # an Euler file (5 records per block) read as Navier-Stokes (6)
    assert Oracle.readda(os.path.join(GOLDEN, "fac_2blk_eu.bin"), "ns3d   ", v, mut) == 9
    # unknown discretisation keys
    x = np.zeros(lay.ld)
    assert Oracle.writdg(str(tmp_path / "g"), "cvxx", x, x, x) == 1
    assert Oracle.writda(str(tmp_path / "f"), "cccv", "ns3d   ", v, mut) == 1


def test_oracle_skips_the_rest_of_a_longer_record(tmp_path):
    """a Fortran READ of fewer items than the record holds skips the rest"""
    lay = layout()
    recs = ff.records("flow", "cccc", "eu3d   ")
    data = b"".join(ff.frame(np.append(r, [1.5, 2.5]).astype("<f8").tobytes(), 1 << 30)
                    for r in recs)
    p = tmp_path / "long"
    p.write_bytes(data)
    v = np.zeros(7 * lay.ld)
    mut = np.zeros(lay.ld)
    assert Oracle.readda(str(p), "eu3d   ", v, mut) == 0
    wv, _ = ff.fill_cells(lay)
    idx = ff.box_index(lay, 1)
    assert np.array_equal(v.reshape(7, lay.ld)[:5, idx], wv[:5, idx])
