"""Per-block array layout of the CodeNS structured solver.

Mirrors the reference's block creation (crdms.f90:125-158): block ``l`` has
real nodes ``i = 1..ni`` (``ii1=1``, ``ii2=ni``) with one ghost layer
(``nfi=1``, ``id1=0``, ``id2=ni+1``), nodes and cells share one index space,
and blocks are stacked one after another at running offsets ``npc(l)``.  The
cell ``(i, j, k)`` of block ``l`` lives at the 0-based flat index
``npc + i + j*nid + k*nid*njd`` (sch_roe.f90:1487-1491 with 0-based storage).

Cell ``(i, j, k)`` with ``1 <= i <= ni-1`` (etc.) is a real cell; its lower
face in direction ``d`` is the face whose area vector is stored at the same
index in ``sn`` (norm.f90:70-75).  The normals of block ``l`` occupy
``sn[9*npc(l) : 9*npc(l)+9*nnn(l)]`` as ``sn(nnn, 3 directions, 3 components)``
column-major (atsch_num.f90:470-479).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np


@dataclass(frozen=True)
class Block:
    ni: int
    nj: int
    nk: int
    npc: int

    @property
    def nid(self) -> int:
        return self.ni + 2

    @property
    def njd(self) -> int:
        return self.nj + 2

    @property
    def nkd(self) -> int:
        return self.nk + 2

    @property
    def nijd(self) -> int:
        return self.nid * self.njd

    @property
    def nnn(self) -> int:
        return self.nijd * self.nkd

    @property
    def nreal(self) -> int:
        return (self.ni - 1) * (self.nj - 1) * (self.nk - 1)

    def ic(self, i, j, k):
        """0-based flat index of cell/node (i, j, k) (Fortran index values)."""
        return self.npc + i + j * self.nid + k * self.nijd

    def real_cells(self) -> np.ndarray:
        """Flat indices of the real cells in (k, j, i) loop order."""
        k, j, i = np.meshgrid(np.arange(1, self.nk), np.arange(1, self.nj),
                              np.arange(1, self.ni), indexing="ij")
        return self.ic(i, j, k).ravel()


@dataclass
class Layout:
    blocks: List[Block]
    ld: int  # leading dimension ip11 of the (ld, ncol) state arrays

    @staticmethod
    def from_dims(dims: Sequence[Tuple[int, int, int]], ld: int | None = None,
                  align: int = 32) -> "Layout":
        blocks, off = [], 0
        for (ni, nj, nk) in dims:
            if min(ni, nj, nk) < 2:
                raise ValueError("each block needs at least 2 nodes per direction")
            b = Block(int(ni), int(nj), int(nk), off)
            blocks.append(b)
            off += b.nnn
        if ld is None:
            ld = (off + align - 1) // align * align
        if ld < off:
            raise ValueError("ld smaller than the total cell count")
        return Layout(blocks, int(ld))

    @property
    def nblk(self) -> int:
        return len(self.blocks)

    @property
    def ncells(self) -> int:
        b = self.blocks[-1]
        return b.npc + b.nnn

    @property
    def nreal(self) -> int:
        return sum(b.nreal for b in self.blocks)

    def dims_array(self) -> np.ndarray:
        return np.array([[b.ni, b.nj, b.nk] for b in self.blocks],
                        dtype=np.int32).ravel()

    def real_cells(self) -> np.ndarray:
        return np.concatenate([b.real_cells() for b in self.blocks])
