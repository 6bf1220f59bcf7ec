"""Seeded synthetic cases for the CodeNS hot path.

The reference ships no decks, meshes or sample flows, so every workload here
is generated: structured blocks of node coordinates, a uniform freestream
(normalised as in utinia.f90:58-66, stagnation density and sound speed 1)
with seeded uniform noise, and the boundary topology the reference builds in
crbds.f90/initis.f90 (ghost-cell lists) and inbdb.f90/initbs.f90 (adjacent
interior cells).

All randomness comes from a counter-based SplitMix64 stream, so a case is a
pure function of its parameters and seed.

Workloads (sizes are cells):
  * ``box_case``      -- one sinusoidally stretched box, extrapolation on the
                         i faces, self-periodic j and k (64x32x32 by default);
  * ``channel_case``  -- blocks in a row forming a channel with a Gaussian
                         bump on the lower wall: injection / outlet pressure /
                         adiabatic walls / periodic k, coincident joins;
  * ``batch_case``    -- many independent boxes of random sides and Mach;
  * ``flat_plate_case`` -- one wall-bounded block with geometric wall
                         stretching and the two Spalart-Allmaras transport
                         columns: injection / outlet / adiabatic plate /
                         extrapolated top / periodic span.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .layout import Layout

# boundary kinds (rbord.f90:144-424): extr, rc (coincident join), para
# (adiabatic wall), idd (injection), prd (imposed pressure)
BC_EXTR, BC_RC, BC_PARA, BC_IDD, BC_PRD = 1, 2, 3, 4, 5
BC_LP2 = 6  # adiabatic wall with the wall law ('lp2': rbord.f90:374-388)
FACES = {"i1": 0, "i2": 1, "j1": 2, "j2": 3, "k1": 4, "k2": 5}

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64_uniform(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Uniform doubles in [0, 1) from a counter-based SplitMix64 stream."""
    with np.errstate(over="ignore"):
        k = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class Phys:
    gam: float = 1.4
    pinfl: float = 0.0
    pr: float = 0.72
    prt: float = 1.0
    reynz: float = 1.0e12
    suth_a: float = 110.4 / 288.15   # zvismo.f90:79, a = 110.4/tnz
    pa1: float = 1.0 / 1.4           # c_nzst.f90:59 with roa1 = ta1 = 1
    aa1: float = 1.0
    omg: float = 0.0


@dataclass
class Scheme:
    ns: int = 0          # equat(1:2) == 'ns'
    muscl: int = 1
    xk: float = -1.0
    ilim: int = 0
    eta: float = 5.0
    kdtl: int = 1        # local time step
    dt1min: float = 0.0
    lmax: int = 10
    qfix_dfez: int = 0   # non-reference: restore the *wi of implimf_eu.f90:312
    precision: int = 0   # fused step: 0 FP64, 1 mixed (FP32 sweeps), 2 defect correction
    kdefect: int = 4     # precision 2: FP64 residual / defect refresh period
    ischema: int = 7     # 7 Roe (sch_roe*), 1 Jameson (dissip_jameson + sch_jameson)
    ki2: float = 0.5     # Jameson 2nd-difference coefficient ki2(lm)
    ki4: float = 1.0 / 32.0  # Jameson 4th-difference coefficient ki4(lm)
    ncychro: int = 1     # time step recomputed when n mod ncychro = 1 or n < icychr0
    icychr0: int = 0     # (atsch_num.f90:173-178, 436); ncychro <= 1: every iteration
    kfmg: int = 0        # 3: dual time stepping, physical time step dt1min
    kdualns: int = 0     # dual time order: 0, 1 second (BDF2), 2 third
    eta_l: Optional[Sequence[float]] = None   # per block eta(lm) (else eta for all)
    ki2_l: Optional[Sequence[float]] = None   # per block ki2(lm)
    ki4_l: Optional[Sequence[float]] = None   # per block ki4(lm)
    weno_fix: int = 0    # non-reference: WENO5 sums all three candidates everywhere


@dataclass
class Boundary:
    block: int          # 0-based block
    face: str           # 'i1' ... 'k2'
    kind: int
    partner: int = -1   # boundary index of the coincident partner
    tper: float = 0.0   # periodic rotation angle of this boundary (rbvc.f90:46)
    values: Tuple[float, ...] = ()   # bceqt values: idd (rpi, rti, d0x, d0y, d0z); prd (p,)


@dataclass
class Case:
    name: str
    layout: Layout
    phys: Phys
    scheme: Scheme
    boundaries: List[Boundary]
    x: np.ndarray        # node coordinates (ld,), real nodes filled
    y: np.ndarray
    z: np.ndarray
    v0: np.ndarray       # (5, ld) initial conserved state
    meta: Dict = field(default_factory=dict)

    # ------------------------------------------------------------------
    def boundary_arrays(self):
        """Flat boundary tables in the reference's list order (initis.f90)."""
        lay = self.layout
        nb = len(self.boundaries)
        btype = np.zeros(nb, np.int32)
        bblk = np.zeros(nb, np.int32)
        bface = np.zeros(nb, np.int32)
        mpb = np.zeros(nb, np.int64)
        mmb = np.zeros(nb, np.int32)
        part = np.full(nb, -1, np.int32)
        cosr = np.ones(nb)
        sinr = np.zeros(nb)
        ncbd, ncin, vals = [], [], []
        off = 0
        for ib, bd in enumerate(self.boundaries):
            b = lay.blocks[bd.block]
            g, inner = _face_cells(b, bd.face)
            btype[ib] = bd.kind
            bblk[ib] = bd.block + 1
            bface[ib] = FACES[bd.face]
            mpb[ib] = off
            mmb[ib] = g.size
            part[ib] = bd.partner
            cosr[ib] = math.cos(bd.tper)
            sinr[ib] = math.sin(bd.tper)
            ncbd.append(g)
            ncin.append(inner)
            val = np.zeros((g.size, 5))
            for a, x in enumerate(bd.values):
                val[:, a] = x
            vals.append(val)
            off += g.size
        for ib, bd in enumerate(self.boundaries):
            if bd.kind == BC_RC:
                p = bd.partner
                if p < 0 or mmb[p] != mmb[ib]:
                    raise ValueError(f"coincident boundary {ib} has no matching partner")
        ncbd = np.concatenate(ncbd).astype(np.int64) if ncbd else np.zeros(0, np.int64)
        ncin = np.concatenate(ncin).astype(np.int64) if ncin else np.zeros(0, np.int64)
        bceqt = (np.concatenate(vals, axis=0) if vals else np.zeros((0, 5)))
        bceqt = np.ascontiguousarray(bceqt.T)   # (5, nlist): column-major nlist x 5
        return dict(type=btype, blk=bblk, face=bface, mpb=mpb, mmb=mmb,
                    partner=part, cosr=cosr, sinr=sinr, ncbd=ncbd, ncin=ncin,
                    bceqt=bceqt)


def _face_cells(b, face: str):
    """Ghost cells of a whole block face and their interior neighbours.

    Order of initis.f90:26-99: i faces loop k then j, j and k faces loop
    (k or j) then i; ncin = ncbd +/- the index increment (initbs.f90:18-27).
    """
    ni, nj, nk = b.ni, b.nj, b.nk
    if face[0] == "i":
        k, j = np.meshgrid(np.arange(1, nk), np.arange(1, nj), indexing="ij")
        ig = 0 if face == "i1" else ni
        g = b.ic(ig, j, k).ravel()
        inc = 1
    elif face[0] == "j":
        k, i = np.meshgrid(np.arange(1, nk), np.arange(1, ni), indexing="ij")
        jg = 0 if face == "j1" else nj
        g = b.ic(i, jg, k).ravel()
        inc = b.nid
    else:
        j, i = np.meshgrid(np.arange(1, nj), np.arange(1, ni), indexing="ij")
        kg = 0 if face == "k1" else nk
        g = b.ic(i, j, kg).ravel()
        inc = b.nijd
    sgn = 1 if face[1] == "1" else -1
    return g.astype(np.int64), (g + sgn * inc).astype(np.int64)


def freestream(phys: Phys, mach: float, alpha_deg: float = 0.0,
               beta_deg: float = 0.0):
    """Conserved freestream of utinia.f90:58-71 (stagnation-normalised)."""
    gam = phys.gam
    gam1 = gam - 1.0
    gam2 = 0.5 * gam1
    gam4 = 1.0 / gam1
    ro = 1.0 / (1.0 + gam2 * mach ** 2) ** gam4
    a = phys.aa1 / (1.0 + gam2 * mach ** 2) ** 0.5
    p = (1.0 + gam2 * mach ** 2) ** (-gam / gam1) / gam
    q = mach * a
    al, be = math.radians(alpha_deg), math.radians(beta_deg)
    u = q * math.cos(al) * math.cos(be)
    v = -q * math.sin(be)
    w = q * math.sin(al) * math.cos(be)
    return ro, u, v, w, p


def _fill_state(lay: Layout, blocks, prim, seed: int, noise: float) -> np.ndarray:
    """Noisy primitive state on every cell (ghosts included) -> conserved."""
    v0 = np.zeros((5, lay.ld))
    gam = prim["gam"]
    pinfl = prim["pinfl"]
    for ib in blocks:
        b = lay.blocks[ib]
        ro, u, vv, w, p = prim["state"][ib]
        q = math.sqrt(u * u + vv * vv + w * w) or 1.0
        n = b.nnn
        r = splitmix64_uniform(seed + 7919 * ib, 5 * n).reshape(5, n)
        e = noise * (2.0 * r - 1.0)
        rho = ro * (1.0 + e[0])
        uu = u + q * e[1]
        vy = vv + q * e[2]
        wz = w + q * e[3]
        pp = p * (1.0 + e[4])
        sl = slice(b.npc, b.npc + n)
        v0[0, sl] = rho
        v0[1, sl] = rho * uu
        v0[2, sl] = rho * vy
        v0[3, sl] = rho * wz
        v0[4, sl] = pp / (gam - 1.0) + pinfl + 0.5 * rho * (uu * uu + vy * vy + wz * wz)
    return v0


def _stretch(xi: np.ndarray, s: float = 0.5) -> np.ndarray:
    return xi - s / (2.0 * math.pi) * np.sin(2.0 * math.pi * xi)


def _box_coords(lay: Layout, ib: int, lengths=(2.0, 1.0, 1.0), s: float = 0.5,
                skew: float = 0.0, origin=(0.0, 0.0, 0.0)):
    b = lay.blocks[ib]
    i = np.arange(1, b.ni + 1)
    j = np.arange(1, b.nj + 1)
    k = np.arange(1, b.nk + 1)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    xi = (I - 1) / (b.ni - 1)
    eta = (J - 1) / (b.nj - 1)
    zeta = (K - 1) / (b.nk - 1)
    X = origin[0] + lengths[0] * _stretch(xi, s)
    Y = origin[1] + lengths[1] * _stretch(eta, s)
    Z = origin[2] + lengths[2] * _stretch(zeta, s)
    if skew:
        X = X + skew * np.sin(2 * math.pi * eta) * np.sin(2 * math.pi * zeta)
        Y = Y + skew * np.sin(2 * math.pi * xi) * np.sin(2 * math.pi * zeta)
        Z = Z + skew * np.sin(2 * math.pi * xi) * np.sin(2 * math.pi * eta)
    return b.ic(I, J, K).ravel(), X.ravel(), Y.ravel(), Z.ravel()


def box_case(cells=(64, 32, 32), mach: float = 0.8, seed: int = 1,
             noise: float = 0.01, ns: bool = False, ilim: int = 0,
             skew: float = 0.0, lmax: int = 10, eta: float = 5.0,
             pinfl: float = 0.0, reynz: float = 1.0e12, alpha: float = 0.0,
             qfix_dfez: int = 0, ischema: int = 7, name: str = "box") -> Case:
    """Single stretched box: extr on i faces, self-periodic j and k."""
    ni, nj, nk = (c + 1 for c in cells)
    lay = Layout.from_dims([(ni, nj, nk)])
    phys = Phys(pinfl=pinfl, reynz=reynz)
    scheme = Scheme(ns=int(ns), ilim=ilim, lmax=lmax, eta=eta, qfix_dfez=qfix_dfez,
                    ischema=ischema)
    x = np.zeros(lay.ld); y = np.zeros(lay.ld); z = np.zeros(lay.ld)
    idx, X, Y, Z = _box_coords(lay, 0, skew=skew)
    x[idx], y[idx], z[idx] = X, Y, Z
    st = freestream(phys, mach, alpha)
    v0 = _fill_state(lay, [0], dict(gam=phys.gam, pinfl=pinfl,
                                    state={0: st}), seed, noise)
    bnd = [Boundary(0, "i1", BC_EXTR), Boundary(0, "i2", BC_EXTR),
           Boundary(0, "j1", BC_RC, partner=3), Boundary(0, "j2", BC_RC, partner=2),
           Boundary(0, "k1", BC_RC, partner=5), Boundary(0, "k2", BC_RC, partner=4)]
    return Case(name, lay, phys, scheme, bnd, x, y, z, v0,
                meta=dict(mach=mach, seed=seed, cells=tuple(cells)))


C1_SUBRUNS = ("1a", "1b", "1c")


def c1_case(sub: str, qfix_dfez: int = 0, seed: int = 1, lmax: int = 10) -> Case:
    """The 64x32x32-cell stretched box at Mach 0.8 (extr i faces, periodic j
    and k, 1% noise, CFL 5) as one of its three reference-path sub-runs:
    1a Euler Roe with the unlimited kappa = -1 MUSCL (sch_roe_euler +
    implimf_eu), 1b Euler Jameson with ki2 = 0.5, ki4 = 1/32 (dissip_jameson +
    sch_jameson + implimf_eu), 1c the Navier-Stokes path at Re 1e12 with the
    minmod limiter (sch_roe + implimf_3d).  qfix_dfez = 1 restores the factor
    implimf_eu.f90:312 lacks (non-reference; the reference form of 1a and 1b
    turns non-finite within a few iterations)."""
    if sub == "1a":
        return box_case((64, 32, 32), mach=0.8, seed=seed, lmax=lmax, qfix_dfez=qfix_dfez,
                        name="c1a")
    if sub == "1b":
        c = box_case((64, 32, 32), mach=0.8, seed=seed, lmax=lmax, qfix_dfez=qfix_dfez,
                     ischema=1, name="c1b")
        c.scheme.ki2, c.scheme.ki4 = 0.5, 1.0 / 32.0
        return c
    if sub == "1c":
        return box_case((64, 32, 32), mach=0.8, seed=seed, lmax=lmax, ns=True, ilim=1,
                        reynz=1.0e12, name="c1c")
    raise ValueError(f"unknown sub-run {sub!r}")


def batch_case(ncase: int = 64, side=(16, 96), seed: int = 4,
               noise: float = 0.01, lmax: int = 10, eta: float = 5.0,
               mach_range=(0.3, 2.0), alpha_range=(-5.0, 5.0),
               qfix_dfez: int = 0) -> Case:
    """Independent single-block Euler boxes run as one multi-block layout."""
    r = splitmix64_uniform(seed, 5 * ncase).reshape(ncase, 5)
    lo, hi = side
    sides = (lo + np.floor(r[:, :3] * (hi - lo + 1))).astype(int)
    machs = mach_range[0] + r[:, 3] * (mach_range[1] - mach_range[0])
    alphas = alpha_range[0] + r[:, 4] * (alpha_range[1] - alpha_range[0])
    lay = Layout.from_dims([tuple(int(s) + 1 for s in sd) for sd in sides])
    phys = Phys()
    scheme = Scheme(ns=0, lmax=lmax, eta=eta, qfix_dfez=qfix_dfez)
    x = np.zeros(lay.ld); y = np.zeros(lay.ld); z = np.zeros(lay.ld)
    states = {}
    bnd: List[Boundary] = []
    for ib in range(ncase):
        idx, X, Y, Z = _box_coords(lay, ib, origin=(0.0, 0.0, 0.0))
        x[idx], y[idx], z[idx] = X, Y, Z
        states[ib] = freestream(phys, float(machs[ib]), float(alphas[ib]))
        base = len(bnd)
        bnd += [Boundary(ib, "i1", BC_EXTR), Boundary(ib, "i2", BC_EXTR),
                Boundary(ib, "j1", BC_RC, partner=base + 3),
                Boundary(ib, "j2", BC_RC, partner=base + 2),
                Boundary(ib, "k1", BC_RC, partner=base + 5),
                Boundary(ib, "k2", BC_RC, partner=base + 4)]
    v0 = _fill_state(lay, range(ncase), dict(gam=phys.gam, pinfl=0.0,
                                              state=states), seed, noise)
    return Case("batch", lay, phys, scheme, bnd, x, y, z, v0,
                meta=dict(seed=seed, sides=sides.tolist(), mach=machs.tolist(),
                          alpha=alphas.tolist()))


def batch_member(batch: Case, ib: int) -> Case:
    """Case ib of a batch as a case of its own: the same block dimensions,
    coordinates, state and boundary conditions in a one-block layout."""
    import copy
    b = batch.layout.blocks[ib]
    lay = Layout.from_dims([(b.ni, b.nj, b.nk)])
    sl = slice(b.npc, b.npc + b.nnn)
    x = np.zeros(lay.ld); y = np.zeros(lay.ld); z = np.zeros(lay.ld)
    x[:b.nnn], y[:b.nnn], z[:b.nnn] = batch.x[sl], batch.y[sl], batch.z[sl]
    v0 = np.zeros((5, lay.ld))
    v0[:, :b.nnn] = batch.v0[:, sl]
    own = [q for q, bd in enumerate(batch.boundaries) if bd.block == ib]
    remap = {q: r for r, q in enumerate(own)}
    bnd = [Boundary(0, batch.boundaries[q].face, batch.boundaries[q].kind,
                    partner=remap.get(batch.boundaries[q].partner, -1),
                    tper=batch.boundaries[q].tper, values=batch.boundaries[q].values)
           for q in own]
    return Case(f"{batch.name}[{ib}]", lay, copy.deepcopy(batch.phys),
                copy.deepcopy(batch.scheme), bnd, x, y, z, v0,
                meta=dict(batch=batch.name, member=ib))


def channel_dims(nblk: int = 8, seed: int = 2, lo: int = 48, hi: int = 128,
                 target=(3.5e6, 4.5e6)):
    """Block sizes of the bump channel: n_i per block and a shared n_j, n_k,
    redrawn with seed+1 until the total cell count is inside ``target``."""
    s = seed
    while True:
        r = splitmix64_uniform(s, nblk + 2)
        ni = (lo + np.floor(r[:nblk] * (hi - lo + 1))).astype(int)
        nj = int(lo + math.floor(r[nblk] * (hi - lo + 1)))
        nk = int(lo + math.floor(r[nblk + 1] * (hi - lo + 1)))
        tot = int(ni.sum()) * nj * nk
        if target[0] <= tot <= target[1] or target is None:
            return [int(a) for a in ni], nj, nk, s
        s += 1


def channel_case(ni_cells: Optional[Sequence[int]] = None, nj_cells: int = 0,
                 nk_cells: int = 0, seed: int = 2, mach: float = 0.5,
                 reynz: float = 1.0e4, noise: float = 0.01, lmax: int = 10,
                 eta: float = 5.0, ilim: int = 1, bump: float = 0.1,
                 length: float = 8.0, span: float = 0.5, walls: bool = True,
                 ischema: int = 7, alpha: float = 0.0, wall=None,
                 wall_kind: int = BC_PARA, name: str = "channel") -> Case:
    """Bump channel: blocks along x joined by coincident faces.

    Lower wall y_w(x) = bump*exp(-((x-x_c)/0.25)^2) with x_c at mid-length,
    upper wall y = 1; nodes interpolated algebraically wall to wall with a
    mild tanh clustering at both walls; z periodic over ``span``.
    Boundary kinds: idd at the inlet face (total pressure / temperature of the
    freestream, flow along +x), prd at the outlet (freestream static
    pressure), para on both walls, periodic k on every block.  walls=False
    makes j periodic too (a duct with inlet and outlet only; with bump=0 its
    steady state is the uniform flow set by the inlet and outlet values).
    alpha: inlet flow angle in the x-y plane (degrees); wall: the lower-wall
    height of every node column along x (sum(ni_cells) + 1 values) instead
    of the bump formula; wall_kind: BC_LP2 gives both walls the wall law.
    """
    if ni_cells is None:
        ni_cells, nj_cells, nk_cells, seed = channel_dims(seed=seed)
    nblk = len(ni_cells)
    dims = [(int(n) + 1, nj_cells + 1, nk_cells + 1) for n in ni_cells]
    lay = Layout.from_dims(dims)
    phys = Phys(reynz=reynz)
    scheme = Scheme(ns=1, ilim=ilim, lmax=lmax, eta=eta, ischema=ischema)
    x = np.zeros(lay.ld); y = np.zeros(lay.ld); z = np.zeros(lay.ld)
    ntot = int(sum(ni_cells))
    xc = 0.5 * length
    beta = 1.5
    i0 = 0
    for ib, b in enumerate(lay.blocks):
        i = np.arange(1, b.ni + 1)
        j = np.arange(1, b.nj + 1)
        k = np.arange(1, b.nk + 1)
        K, J, I = np.meshgrid(k, j, i, indexing="ij")
        X = length * (i0 + I - 1) / ntot
        eta_ = (J - 1) / (b.nj - 1)
        s = 0.5 * (1.0 + np.tanh(beta * (2.0 * eta_ - 1.0)) / math.tanh(beta))
        if wall is None:
            yw = bump * np.exp(-((X - xc) / 0.25) ** 2)
        else:
            yw = np.asarray(wall, dtype=float)[i0 + I - 1]
        Y = yw + (1.0 - yw) * s
        Z = span * (K - 1) / (b.nk - 1)
        idx = b.ic(I, J, K).ravel()
        x[idx], y[idx], z[idx] = X.ravel(), Y.ravel(), Z.ravel()
        i0 += b.ni - 1
    st = freestream(phys, mach)
    v0 = _fill_state(lay, range(nblk), dict(gam=phys.gam, pinfl=0.0,
                                             state={ib: st for ib in range(nblk)}),
                     seed, noise)
    bnd: List[Boundary] = []
    # joins first so partner indices are easy: boundary 2*ib = i2 of block ib,
    # 2*ib+1 = i1 of block ib+1
    for ib in range(nblk - 1):
        a = len(bnd)
        bnd.append(Boundary(ib, "i2", BC_RC, partner=a + 1))
        bnd.append(Boundary(ib + 1, "i1", BC_RC, partner=a))
    p_inf = st[4]
    bnd.append(Boundary(0, "i1", BC_IDD, values=(1.0, 1.0, math.cos(math.radians(alpha)),
                                                 math.sin(math.radians(alpha)), 0.0)))
    bnd.append(Boundary(nblk - 1, "i2", BC_PRD, values=(p_inf,)))
    for ib in range(nblk):
        if walls:
            bnd.append(Boundary(ib, "j1", wall_kind))
            bnd.append(Boundary(ib, "j2", wall_kind))
        else:
            a = len(bnd)
            bnd.append(Boundary(ib, "j1", BC_RC, partner=a + 1))
            bnd.append(Boundary(ib, "j2", BC_RC, partner=a))
        a = len(bnd)
        bnd.append(Boundary(ib, "k1", BC_RC, partner=a + 1))
        bnd.append(Boundary(ib, "k2", BC_RC, partner=a))
    return Case(name, lay, phys, scheme, bnd, x, y, z, v0,
                meta=dict(mach=mach, seed=seed, reynz=reynz, alpha=alpha,
                          ni=list(ni_cells), nj=nj_cells, nk=nk_cells, length=length,
                          span=span, bump=bump, beta=beta))


def sutherland_mu(phys: Phys, temp: float) -> float:
    """zvismo.f90:90-104 (air): mu = T^1.5 (1 + a) / (T + a) / Re"""
    a = phys.suth_a
    return (1.0 / phys.reynz) * temp * math.sqrt(temp) * (1.0 + a) / (temp + a)


def flat_plate_case(cells=(256, 128, 64), mach: float = 0.3, reynz: float = 1.0e6,
                    dy1: float = 1.0e-5, ratio: float = 1.1, length: float = 1.0,
                    span: float = 0.1, nut_ratio: float = 3.0, seed: int = 3,
                    noise: float = 0.0, lmax: int = 10, eta: float = 5.0,
                    wall_kind: int = BC_PARA, side_walls: bool = False,
                    name: str = "flat_plate") -> Case:
    """RANS flat plate: one block of cells[0] x cells[1] x cells[2] cells.

    x uniform over ``length`` (the plate spans the whole lower face, leading
    edge at the inlet), y geometric from the wall (first spacing dy1, growth
    ratio), z uniform over ``span``.  Boundaries: idd at i1 (freestream total
    pressure / temperature along +x), prd at i2 (freestream static
    pressure), para (adiabatic wall) at j1, extr at j2, periodic k.  The
    state has 7 columns: the freestream (uniform unless ``noise`` > 0) and
    the Spalart-Allmaras variable rho nu~ = nut_ratio * mu_inf (v(:,7) = 0),
    as met_inisa.f90 leaves it for a uniform mut.  meta['rokinf'] is the
    freestream rho nu~ the injection ghosts take (met_bord.f90:60-63).
    With the reference's Spalart-Allmaras source the iteration of the
    full-size plate fails once S~ (negative in the freestream, where fv2 < 0)
    crosses zero at some cell; run it with the flagged source fix
    (CodeNS.set_sa(..., stilde_fix=1)).  wall_kind: BC_LP2 puts the wall law
    on the plate; side_walls: the k faces are walls of that kind too instead
    of periodic (cells along the corners then have two walls).
    """
    ni, nj, nk = (c + 1 for c in cells)
    lay = Layout.from_dims([(ni, nj, nk)])
    phys = Phys(reynz=reynz)
    scheme = Scheme(ns=1, ilim=0, lmax=lmax, eta=eta)
    x = np.zeros(lay.ld); y = np.zeros(lay.ld); z = np.zeros(lay.ld)
    b = lay.blocks[0]
    i = np.arange(1, ni + 1)
    j = np.arange(1, nj + 1)
    k = np.arange(1, nk + 1)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    X = length * (I - 1) / (ni - 1)
    Y = dy1 * (ratio ** (J - 1) - 1.0) / (ratio - 1.0)
    Z = span * (K - 1) / (nk - 1)
    idx = b.ic(I, J, K).ravel()
    x[idx], y[idx], z[idx] = X.ravel(), Y.ravel(), Z.ravel()
    st = freestream(phys, mach)
    v5 = _fill_state(lay, [0], dict(gam=phys.gam, pinfl=0.0, state={0: st}), seed, noise)
    t_inf = phys.gam * st[4] / st[0]
    mu_inf = sutherland_mu(phys, t_inf)
    rokinf = nut_ratio * mu_inf
    v0 = np.zeros((7, lay.ld))
    v0[:5] = v5
    r = splitmix64_uniform(seed + 104729, b.nnn)
    v0[5, b.npc:b.npc + b.nnn] = rokinf * (1.0 + noise * (2.0 * r - 1.0))
    bnd = [Boundary(0, "i1", BC_IDD, values=(1.0, 1.0, 1.0, 0.0, 0.0)),
           Boundary(0, "i2", BC_PRD, values=(st[4],)),
           Boundary(0, "j1", wall_kind), Boundary(0, "j2", BC_EXTR)]
    if side_walls:
        bnd += [Boundary(0, "k1", wall_kind), Boundary(0, "k2", wall_kind)]
    else:
        bnd += [Boundary(0, "k1", BC_RC, partner=5), Boundary(0, "k2", BC_RC, partner=4)]
    return Case(name, lay, phys, scheme, bnd, x, y, z, v0,
                meta=dict(mach=mach, reynz=reynz, seed=seed, cells=tuple(cells), dy1=dy1,
                          ratio=ratio, length=length, span=span, rokinf=rokinf,
                          mu_inf=mu_inf, nut_ratio=nut_ratio))
