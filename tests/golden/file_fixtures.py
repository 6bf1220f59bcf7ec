"""Golden files of the reference's grid and flow formats, and the script
that writes them (``python tests/golden/file_fixtures.py``).

No file written by the reference itself exists (it ships no grids, decks
or restart files, and there is no Fortran compiler here), so these files are
built from two published facts, with numpy and struct only:

* gfortran's layout of unformatted sequential files: a logical record is
  one or more subrecords, each a 4-byte leading marker, the data and a
  4-byte trailing marker (little-endian here); a marker holds the
  subrecord's byte count, negated on the leading marker when another
  subrecord follows and on the trailing marker when one precedes; a
  subrecord holds at most 2147483639 bytes (``-fmax-subrecord-length``
  lowers that, which the ``sub20`` file uses to exercise the split);
* the record order of the reference's writers: for every block in order,
  ``writdg.f90:46-48`` writes x, y, z over the box that ``chdgcv.f90``
  chose (real nodes for cvcv, real cells for cvcc, cells with the ghost
  layer for cvcf; cell centres are ``.125*(sum of the 8 nodes)`` in
  ``cvccg.f90``'s order), and ``writda.f90:78-97`` writes v1..v5, then mut
  when ``equat(1:2) = 'ns'``, then v6, v7 when ``equat(6:7) = 'ke'``, over
  the box of ``chdacc.f90`` (real cells for cccc, with the ghost layer for
  cccf).  Every record loops i fastest, then j, then k.

The values are smooth functions of (block, i, j, k) with no exact binary
form, so a reader or writer that visits the box in another order, or sums
the centre's nodes in another order, changes the bytes.
"""
from __future__ import annotations

import hashlib
import json
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DIMS = [(4, 3, 3), (3, 3, 2)]   # real nodes ni, nj, nk of the two blocks
MAXSUB = 2147483639

FILES = [
    # name, kind, disc, equat, maxsub
    ("fgv_2blk.bin", "grid", "cvcv", "", MAXSUB),
    ("fgc_2blk.bin", "grid", "cvcc", "", MAXSUB),
    ("fgcf_2blk.bin", "grid", "cvcf", "", MAXSUB),
    ("fac_2blk_eu.bin", "flow", "cccc", "eu3d   ", MAXSUB),
    ("fac_2blk_ns.bin", "flow", "cccc", "ns3d   ", MAXSUB),
    ("fac_2blk_ke_sub20.bin", "flow", "cccc", "ns3d ke", 20),
    ("facf_2blk_ns.bin", "flow", "cccf", "ns3d   ", MAXSUB),
]


def node_value(c: int, b: int, i, j, k):
    """coordinate c (0 x, 1 y, 2 z) of node (i, j, k) of block b, ghosts too"""
    i, j, k = (np.asarray(a, dtype=np.float64) for a in (i, j, k))
    return (0.7 * (c + 1) + b + 0.1 * i + 0.01 * j * (c + 1) + 0.001 * k
            + 1.0e-4 * i * j * k / 3.0)


def cell_value(a: int, b: int, i, j, k):
    """column a (0..6 of v; 7 = mut) of cell (i, j, k) of block b, ghosts too"""
    i, j, k = (np.asarray(q, dtype=np.float64) for q in (i, j, k))
    return (1.0 + 0.3 * a + 0.05 * b + 0.02 * i / 3.0 + 0.004 * j + 0.0007 * k * (a + 1)
            + 1.0e-5 * i * j * k)


def box(dims, what):
    """(lo, hi) of a record's box: 0 real nodes, 1 real cells, 2 cells with
    the ghost layer"""
    lo = [0 if what == 2 else 1] * 3
    hi = [n - 1 if what == 1 else n for n in dims]
    return lo, hi


def box_ijk(dims, what):
    """i, j, k of the box's points in record order (i fastest)"""
    lo, hi = box(dims, what)
    k, j, i = np.meshgrid(*(np.arange(lo[a], hi[a] + 1) for a in (2, 1, 0)), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()


def centre_value(c, b, i, j, k):
    """cvccg.f90: .125*(x(n)+x(n+inc3)+x(n+inc1)+x(n+inc1+inc3)+x(n+inc2)
    +x(n+inc2+inc3)+x(n+inc1+inc2)+x(n+inc1+inc2+inc3)), summed left to right"""
    terms = [(0, 0, 0), (0, 0, 1), (1, 0, 0), (1, 0, 1), (0, 1, 0), (0, 1, 1), (1, 1, 0),
             (1, 1, 1)]
    s = None
    for di, dj, dk in terms:
        t = node_value(c, b, i + di, j + dj, k + dk)
        s = t if s is None else s + t
    return 0.125 * s


def records(kind, disc, equat):
    """the data of every record of a file, in order"""
    out = []
    eq = equat.ljust(7)
    for b, dims in enumerate(DIMS):
        if kind == "grid":
            what = {"cvcv": 0, "cvcc": 1, "cvcf": 2}[disc]
            i, j, k = box_ijk(dims, what)
            for c in range(3):
                out.append(node_value(c, b, i, j, k) if what == 0 else centre_value(c, b, i, j, k))
        else:
            what = {"cccc": 1, "cccf": 2}[disc]
            i, j, k = box_ijk(dims, what)
            cols = list(range(5))
            if eq[0:2] == "ns":
                cols.append(7)
            if eq[5:7] == "ke":
                cols += [5, 6]
            for a in cols:
                out.append(cell_value(a, b, i, j, k))
    return out


def frame(data: bytes, maxsub: int) -> bytes:
    """one logical record in gfortran's subrecord framing"""
    out, pos, first = [], 0, True
    while True:
        chunk = data[pos:pos + maxsub]
        pos += len(chunk)
        more = pos < len(data)
        out.append(struct.pack("<i", -len(chunk) if more else len(chunk)))
        out.append(chunk)
        out.append(struct.pack("<i", len(chunk) if first else -len(chunk)))
        first = False
        if not more:
            return b"".join(out)


def file_bytes(kind, disc, equat, maxsub) -> bytes:
    return b"".join(frame(np.asarray(r, "<f8").tobytes(), maxsub)
                    for r in records(kind, disc, equat))


def write_all():
    manifest = []
    for name, kind, disc, equat, maxsub in FILES:
        data = file_bytes(kind, disc, equat, maxsub)
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)
        manifest.append(dict(file=name, kind=kind, disc=disc, equat=equat, maxsub=maxsub,
                             records=len(records(kind, disc, equat)), bytes=len(data),
                             sha256=hashlib.sha256(data).hexdigest()))
    with open(os.path.join(HERE, "files.json"), "w") as f:
        json.dump(dict(dims=DIMS, files=manifest), f, indent=1)
        f.write("\n")


# the arrays of a layout filled from the same functions (for the readers'
# expected results and the writers' inputs)
def fill_nodes(layout):
    """x, y, z (ld,) with every node of every block, ghosts included"""
    out = [np.zeros(layout.ld) for _ in range(3)]
    for b, blk in enumerate(layout.blocks):
        k, j, i = np.meshgrid(np.arange(blk.nkd), np.arange(blk.njd), np.arange(blk.nid),
                              indexing="ij")
        n = blk.ic(i, j, k).ravel()
        for c in range(3):
            out[c][n] = node_value(c, b, i.ravel(), j.ravel(), k.ravel())
    return out


def fill_cells(layout, ncol=7):
    """v (ncol, ld) and mut (ld,) at every cell of every block"""
    v = np.zeros((ncol, layout.ld))
    mut = np.zeros(layout.ld)
    for b, blk in enumerate(layout.blocks):
        k, j, i = np.meshgrid(np.arange(blk.nkd), np.arange(blk.njd), np.arange(blk.nid),
                              indexing="ij")
        n = blk.ic(i, j, k).ravel()
        for a in range(ncol):
            v[a, n] = cell_value(a, b, i.ravel(), j.ravel(), k.ravel())
        mut[n] = cell_value(7, b, i.ravel(), j.ravel(), k.ravel())
    return v, mut


def box_index(layout, what):
    """flat indices of every block's box (0 real nodes, 1 real cells, 2 cells
    with the ghost layer)"""
    idx = []
    for blk in layout.blocks:
        i, j, k = box_ijk((blk.ni, blk.nj, blk.nk), what)
        idx.append(blk.ic(i, j, k))
    return np.concatenate(idx)


if __name__ == "__main__":
    write_all()
