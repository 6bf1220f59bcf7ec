"""Discrete adjoint of the steady Euler Roe solution on the bump channel:
gradients of the wall pressure force with respect to the inflow Mach number,
the inflow angle and the lower-wall node heights, behind a
``torch.autograd.Function``.

Problem (configuration 5 form): the bump channel of ``cases.channel_case`` as
an extruded 2-D Euler flow -- injection at the inlet (total pressure and
temperature, flow direction (cos a, sin a, 0), clidd.f90), imposed static
pressure p_inf(M) at the outlet (clprd.f90), slip walls (clpara.f90),
periodic span -- solved to a steady state by the FP64 Roe iteration
(sch_roe_euler, implimf_eu with the flagged qfix_dfez = 1 that keeps its
implicit phase linear in the increment).  The reconstruction is first order
by default: with the unlimited kappa = -1 MUSCL the iteration on this channel
settles into a limit cycle at L2 ~1e-6 and never reaches the steady state an
adjoint linearises about; muscl = 1 is accepted where it converges.

Functional (utitfr.f90:287-327): the x component of the pressure force on
the lower wall, J = sum over wall faces of (gam p_inf - gam p_ghost) *
|dS_yz| * sign(n_x), the face area projection from the face's four nodes.

Gradient: with u(W; x, M, a) = 0 the converged residual, lambda solves
A^T lambda = dJ/dW (A = du/dW) and dJ/dtheta = dJ/dtheta|_W - lambda^T
du/dtheta.  The CUDA library supplies A^T lambda (exact, from the scheme's
own expressions in dual numbers) and L^T, the transposed linearised implicit
phase; lambda iterates lambda += L^T (dJ/dW - A^T lambda), the transpose of
the primal iteration, so it converges at the primal's rate.  The small local
maps around the residual -- the pressure of a cell (zpres), the ghost cells
as functions of the interior (the boundary conditions), the face areas and
the boundary normals as functions of the nodes, the functional -- are
restated here in torch and differentiated by autograd; their Jacobians are
linearised once per gradient.

This module is the thin PyTorch binding of the adjoint; the primal and the
transposed products run in the CUDA library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import cases
from .solver import CodeNS


# ---------------------------------------------------------------------------
# problem definition
# ---------------------------------------------------------------------------
@dataclass
class Design:
    ni: int = 512            # cells along the channel (one block)
    nj: int = 256            # cells wall to wall
    nk: int = 4              # cells across the (periodic) span
    mach: float = 0.5
    alpha: float = 0.0       # inlet flow angle, degrees
    bump: float = 0.1
    length: float = 8.0
    span: float = 0.5
    seed: int = 5
    lmax: int = 10
    eta: float = 5.0
    muscl: int = 0           # 0: first-order reconstruction, 1: kappa = -1 MUSCL
    precision: int = 0       # 0 FP64; 1 mixed: FP32 primal sweeps and FP32 transposed
                             # sweeps of the adjoint (FP64 residual and A^T lambda)

    def wall(self) -> np.ndarray:
        """lower-wall height of every node column (ni + 1 values)"""
        x = self.length * np.arange(self.ni + 1) / self.ni
        return self.bump * np.exp(-((x - 0.5 * self.length) / 0.25) ** 2)

    def case(self, mach=None, alpha=None, wall=None) -> cases.Case:
        c = cases.channel_case([self.ni], self.nj, self.nk, seed=self.seed,
                               mach=self.mach if mach is None else float(mach),
                               reynz=1.0e12, noise=0.0, lmax=self.lmax, eta=self.eta,
                               ilim=0, length=self.length, span=self.span,
                               alpha=self.alpha if alpha is None else float(alpha),
                               wall=self.wall() if wall is None else np.asarray(wall))
        c.scheme.ns = 0
        c.scheme.qfix_dfez = 1
        c.scheme.muscl = self.muscl
        c.scheme.precision = self.precision
        return c


def p_inf(mach, gam=1.4):
    """outlet static pressure of the stagnation-normalised freestream
    (utinia.f90:58-71)"""
    return (1.0 + 0.5 * (gam - 1.0) * mach ** 2) ** (-gam / (gam - 1.0)) / gam


# ---------------------------------------------------------------------------
# primal
# ---------------------------------------------------------------------------
def solve_primal(case, tol=1e-13, max_iter=20000, chunk=200, solver=None):
    """iterate the FP64 scheme until the L2 norm of the density increment is
    below tol; returns (solver, iterations, last L2)"""
    s = solver if solver is not None else CodeNS(case)
    if solver is None:
        s.metric()
    it = 0
    l2 = float("inf")
    while it < max_iter:
        n = s.atsch_num(chunk)
        it += chunk
        l2 = float(n[1, 0])
        if not math.isfinite(l2):
            raise RuntimeError("primal iteration diverged")
        if l2 < tol:
            break
    return s, it, l2


# ---------------------------------------------------------------------------
# torch restatements of the local maps (for their derivatives)
# ---------------------------------------------------------------------------
class _Maps:
    """Index tables of one case and the torch functions of (state, nodes,
    parameters) around the residual."""

    def __init__(self, case, torch, dev):
        self.torch = torch
        self.dev = dev
        self.case = case
        lay = case.layout
        self.ld = lay.ld
        b = lay.blocks[0]
        self.b = b
        self.gam = case.phys.gam
        self.gam1 = case.phys.gam - 1.0
        self.pinfl = case.phys.pinfl
        ba = case.boundary_arrays()
        self.ba = ba
        L = lambda a: torch.as_tensor(np.asarray(a), device=dev)
        self.real = L(lay.real_cells())
        self.ncbd = L(ba["ncbd"])
        self.ncin = L(ba["ncin"])
        nb = len(case.boundaries)
        ent_b = np.concatenate([np.full(int(m), q) for q, m in enumerate(ba["mmb"])])
        self.ent_b = ent_b
        self.kind = ba["type"][ent_b]
        part_in = np.zeros(len(ent_b), np.int64)
        for q in range(nb):
            if ba["type"][q] == cases.BC_RC:
                p = ba["partner"][q]
                m0, mm = ba["mpb"][q], ba["mmb"][q]
                part_in[m0:m0 + mm] = ba["ncin"][ba["mpb"][p]:ba["mpb"][p] + mm]
        self.part_in = L(part_in)
        # the boundary entries' scatter targets in layers with distinct cells
        # (a cell's first entry in list order in layer 0, its second in
        # layer 1, ...; only block corners and edges have more than one), so
        # every layer is a scatter-add without colliding indices and the
        # layers add in a fixed order: deterministic sums
        def layers(dest, use):
            seen = {}
            lay_of = np.full(len(dest), -1)
            for e in np.flatnonzero(use):
                c = int(dest[e])
                lay_of[e] = seen.get(c, 0)
                seen[c] = lay_of[e] + 1
            return [L(np.flatnonzero(lay_of == q)) for q in range(int(lay_of.max()) + 1)]
        self.in_layers = layers(ba["ncin"], np.ones(len(ent_b), bool))
        self.part_layers = layers(part_in, ba["type"][ent_b] == cases.BC_RC)
        ghost = np.ones(self.ld, bool)
        ghost[lay.real_cells()] = False
        self.not_real = L(ghost)
        self.face = ba["face"][ent_b]
        self.sel = {k: L(np.flatnonzero(self.kind == k)) for k in
                    (cases.BC_RC, cases.BC_PARA, cases.BC_IDD, cases.BC_PRD, cases.BC_EXTR)}
        self.bceqt = L(ba["bceqt"])            # (5, nlist)
        # lower-wall (j1) entries for the functional
        self.wall_ent = L(np.flatnonzero((self.kind == cases.BC_PARA) & (self.face == 2)))

    # -- geometry -----------------------------------------------------------
    def nodes(self, wall):
        """node coordinates of the channel as functions of the wall heights
        (the grid formula of cases.channel_case)"""
        torch = self.torch
        m = self.case.meta
        b = self.b
        ni, nj, nk = b.ni, b.nj, b.nk
        i = torch.arange(1, ni + 1, device=self.dev, dtype=torch.float64)
        j = torch.arange(1, nj + 1, device=self.dev, dtype=torch.float64)
        k = torch.arange(1, nk + 1, device=self.dev, dtype=torch.float64)
        K, J, I = torch.meshgrid(k, j, i, indexing="ij")
        X = m["length"] * (I - 1) / (ni - 1)
        eta = (J - 1) / (nj - 1)
        beta = m["beta"]
        s = 0.5 * (1.0 + torch.tanh(beta * (2.0 * eta - 1.0)) / math.tanh(beta))
        yw = wall[(I - 1).long()]
        Y = yw + (1.0 - yw) * s
        Z = m["span"] * (K - 1) / (nk - 1)
        idx = torch.as_tensor(b.ic(np.arange(1, ni + 1)[None, None, :],
                                   np.arange(1, nj + 1)[None, :, None],
                                   np.arange(1, nk + 1)[:, None, None]).ravel(),
                              device=self.dev)
        P = torch.zeros((3, self.ld), dtype=torch.float64, device=self.dev)
        P = P.index_put((torch.zeros_like(idx), idx), X.reshape(-1))
        P = P.index_put((torch.ones_like(idx), idx), Y.reshape(-1))
        P = P.index_put((torch.full_like(idx, 2), idx), Z.reshape(-1))
        return P

    def _offs(self, dir):
        b = self.b
        nid, nijd = b.nid, b.nijd
        e = {0: (0, 1, 1), 1: (1, 0, 1), 2: (1, 1, 0)}[dir]
        f = {0: (0, 0, 1), 1: (0, 0, 1), 2: (0, 1, 0)}[dir]
        g = {0: (0, 1, 0), 1: (1, 0, 0), 2: (1, 0, 0)}[dir]
        o = lambda t: t[0] + t[1] * nid + t[2] * nijd
        return o(e), o(f), o(g)

    def face_cells(self, dir):
        """cell indices of the faces of a direction the residual uses (face
        index 1..nd along dir, the other two indices real)"""
        b = self.b
        r = [np.arange(1, b.ni), np.arange(1, b.nj), np.arange(1, b.nk)]
        r[dir] = np.arange(1, [b.ni, b.nj, b.nk][dir] + 1)
        K, J, I = np.meshgrid(r[2], r[1], r[0], indexing="ij")
        return self.torch.as_tensor(b.ic(I, J, K).ravel(), device=self.dev)

    def face_normals(self, P, dir, n):
        """0.5 (d1 x d2) of the faces at cells n (the oriented sign applied by
        the caller), the expressions of norm.f90"""
        torch = self.torch
        e, f, g = self._offs(dir)
        d1 = P[:, n + e] - P[:, n]
        d2 = P[:, n + f] - P[:, n + g]
        return 0.5 * torch.stack([d1[1] * d2[2] - d1[2] * d2[1],
                                  d1[2] * d2[0] - d1[0] * d2[2],
                                  d1[0] * d2[1] - d1[1] * d2[0]])

    def boundary_normals(self, P, sgn):
        """unit boundary normals of every list entry (boundary_geom of the
        metric): the face area at the face cell, +/- by the face side"""
        torch = self.torch
        face = torch.as_tensor(self.face, device=self.dev)
        upper = (face % 2) == 1
        fc = torch.where(upper, self.ncbd, self.ncin)
        out = torch.zeros((3, len(self.face)), dtype=torch.float64, device=self.dev)
        for dir in range(3):
            m = (face // 2) == dir
            if not bool(m.any()):
                continue
            S = sgn[dir] * self.face_normals(P, dir, fc[m])
            isg = torch.where(upper[m], -1.0, 1.0).to(torch.float64)
            nx = isg * S
            nn = torch.sqrt((nx * nx).sum(0))
            out[:, m] = nx / nn
        return out

    # -- thermodynamics and boundary conditions ------------------------------
    def pressure(self, W):
        return self.gam1 * (W[4] - 0.5 * (W[1] ** 2 + W[2] ** 2 + W[3] ** 2) / W[0] - self.pinfl)

    def ghosts(self, Wi, pi, Wp, pp, nrm, bceqt):
        """ghost states and pressures of every list entry from the interior
        cell (Wi, pi), the coincident partner's interior (Wp, pp), the unit
        normals and the boundary values (k_rbord / rbord.f90)"""
        torch = self.torch
        gam, gam1, pinfl = self.gam, self.gam1, self.pinfl
        nl = Wi.shape[1]
        Wg = torch.zeros((5, nl), dtype=torch.float64, device=self.dev)
        pg = torch.zeros(nl, dtype=torch.float64, device=self.dev)
        s = self.sel[cases.BC_RC]
        if len(s):
            Wg[:, s] = 0.5 * (Wi[:, s] + Wp[:, s])
            pg[s] = 0.5 * (pi[s] + pp[s])
        s = self.sel[cases.BC_EXTR]
        if len(s):
            Wg[:, s] = Wi[:, s]
            pg[s] = pi[s]
        s = self.sel[cases.BC_PARA]
        if len(s):
            v1, v2, v3, v4, v5 = Wi[:, s]
            Wg[0, s] = v1
            Wg[4, s] = v5 - 0.5 * (v2 ** 2 + v3 ** 2 + v4 ** 2) / v1
            pg[s] = pi[s]
        s = self.sel[cases.BC_PRD]
        if len(s):
            v1, v2, v3, v4, v5 = Wi[:, s]
            pres = bceqt[0, s]
            qxs, qys, qzs = v2 / v1, v3 / v1, v4 / v1
            p = gam1 * (v5 - 0.5 * v1 * (qxs ** 2 + qys ** 2 + qzs ** 2) - pinfl)
            cs2 = gam * p / v1
            roc0 = torch.sqrt(gam * p * v1)
            dqn = (pres - p) / roc0
            qx = qxs + dqn * nrm[0, s]
            qy = qys + dqn * nrm[1, s]
            qz = qzs + dqn * nrm[2, s]
            rho = v1 + (pres - p) / cs2
            Wg[0, s] = rho
            Wg[1, s] = rho * qx
            Wg[2, s] = rho * qy
            Wg[3, s] = rho * qz
            Wg[4, s] = pres / gam1 + pinfl + 0.5 * rho * (qx ** 2 + qy ** 2 + qz ** 2)
            pg[s] = pres
        s = self.sel[cases.BC_IDD]
        if len(s):
            Wg_s, pg_s = self._idd(Wi[:, s], nrm[:, s], bceqt[:, s])
            Wg[:, s] = Wg_s
            pg[s] = pg_s
        return Wg, pg

    def _idd(self, Wi, nrm, bc, nitn=None):
        """clidd.f90:50-170 (omg = 0): Newton on the normal velocity, the
        whole boundary stopping together once every update is below 1e-7"""
        torch = self.torch
        gam, gam1, pinfl = self.gam, self.gam1, self.pinfl
        aa1 = self.case.phys.aa1
        pa1 = self.case.phys.pa1
        gam6 = gam / gam1
        gamt = gam / aa1 ** 2
        gam2t = 0.5 * gam1 / aa1 ** 2
        rpi, rti, d0x, d0y, d0z = bc
        nx, ny, nz = nrm
        usdn = 1.0 / (d0x * nx + d0y * ny + d0z * nz)
        usdn2 = usdn ** 2
        v1, v2, v3, v4, v5 = Wi
        qxs, qys, qzs = v2 / v1, v3 / v1, v4 / v1
        qn = qxs * nx + qys * ny + qzs * nz
        ps = gam1 * (v5 - 0.5 * (qxs * v2 + qys * v3 + qzs * v4) - pinfl)
        roc0 = -torch.sqrt(gam * ps * v1)
        am0 = ps + roc0 * qn
        if nitn is None:
            # the iteration count of the discrete map (data-dependent, fixed here)
            with torch.no_grad():
                q = qn.detach().clone()
                nitn, res = 0, 1.0
                while res > 1e-7 and nitn < 20:
                    b = 1.0 / (1.0 + gam2t / rti.detach() * usdn2.detach() * q ** 2)
                    p = pa1 * rpi.detach() * b ** gam6
                    ro = gamt * p / (b * rti.detach())
                    f = p + roc0.detach() * q - am0.detach()
                    df = roc0.detach() - ro * q * usdn2.detach()
                    dq = -f / df
                    res = float((dq.abs() / q).max())
                    q = q + dq
                    nitn += 1
            self.idd_nitn = nitn
        for _ in range(nitn):
            b = 1.0 / (1.0 + gam2t / rti * usdn2 * qn ** 2)
            p = pa1 * rpi * b ** gam6
            ro = gamt * p / (b * rti)
            f = p + roc0 * qn - am0
            df = roc0 - ro * qn * usdn2
            qn = qn - f / df
        b = 1.0 / (1.0 + gam2t / rti * usdn2 * qn ** 2)
        p = pa1 * rpi * b ** gam6
        ro = gamt * p / (b * rti)
        w = qn * usdn
        m1, m2, m3 = ro * (w * d0x), ro * (w * d0y), ro * (w * d0z)
        E = p / gam1 + pinfl + 0.5 * (m1 ** 2 + m2 ** 2 + m3 ** 2) / ro
        return torch.stack([ro, m1, m2, m3, E]), p

    def functional(self, W, pg_wall, P, mach, sgn_nx):
        """x pressure force on the lower wall (utitfr.f90:287-327) with the
        reference pressure gam * p_inf(M)"""
        torch = self.torch
        b = self.b
        g = self.ncbd[self.wall_ent]
        n1 = g + b.nid                       # node (i, 1, k)
        n2 = n1 + 1                          # (i+1, 1, k)
        n3 = n1 + 1 + b.nijd                 # (i+1, 1, k+1)
        n4 = n1 + b.nijd                     # (i, 1, k+1)
        d1 = P[:, n3] - P[:, n1]
        d2 = P[:, n4] - P[:, n2]
        dsyz = torch.abs(d1[1] * d2[2] - d1[2] * d2[1]) / 2.0
        p0spi0 = self.gam * p_inf(mach, self.gam)
        return ((p0spi0 - self.gam * pg_wall) * dsyz * sgn_nx).sum()


# ---------------------------------------------------------------------------
# gradient
# ---------------------------------------------------------------------------
class WallForceGradient:
    """Primal solve, functional and adjoint gradient for one design."""

    def __init__(self, design: Design, mach: float, alpha: float, wall: np.ndarray,
                 tol=1e-13, max_iter=40000, adj_tol=1e-12, adj_max=40000, check=100):
        import torch
        self.torch = torch
        self.design = design
        self.mach, self.alpha = float(mach), float(alpha)
        self.wall = np.asarray(wall, dtype=float)
        self.case = design.case(mach, alpha, self.wall)
        self.s, self.iters, self.l2 = solve_primal(self.case, tol=tol, max_iter=max_iter)
        self.maps = _Maps(self.case, torch, self.s.dev)
        self.adj_tol, self.adj_max, self.check = adj_tol, adj_max, check
        self._setup()

    def close(self):
        self.s.close()

    def _setup(self):
        torch = self.torch
        s, M = self.s, self.maps
        dev = s.dev
        # orientation of the face areas (norm.f90's psk/psj/psi) from the
        # library's metric
        P0 = M.nodes(torch.as_tensor(self.wall, device=dev))
        sn = s.sn.detach()
        b = M.b
        self.sgn = []
        for dir in range(3):
            n = M.face_cells(dir)
            S = M.face_normals(P0, dir, n)
            ref = torch.stack([sn[9 * b.npc + c * 3 * b.nnn + dir * b.nnn + (n - b.npc)]
                               for c in range(3)])
            sg = 1.0 if float((S * ref).sum()) >= 0 else -1.0
            err = float((sg * S - ref).abs().max())
            if err > 1e-12 * float(ref.abs().max()):
                raise RuntimeError(f"torch face areas differ from the metric ({err:.2e})")
            self.sgn.append(sg)
        nrm = M.boundary_normals(P0, self.sgn)
        self.nrm = nrm
        self.sgn_nx = torch.sign(nrm[0, M.wall_ent]).detach()
        self._linearise()

    def _linearise(self):
        """the iteration's inputs and Jacobians at the solver's current state:
        the library's face-flux Jacobians and implicit coefficients
        (cns_adjoint_prepare), the interior pressure derivative (zpres) and
        the boundary-map Jacobians"""
        torch = self.torch
        s, M = self.s, self.maps
        s.adjoint_prepare()
        s.sync()
        W = s.v.detach().reshape(5, M.ld).clone()
        self.W = W
        Wr = W.clone().requires_grad_(True)
        self.dp_dW = torch.autograd.functional.jacobian(
            lambda w: M.pressure(w).sum(), Wr)       # (5, ld)
        self._bc_jac(W, self.nrm)

    def _bc_inputs(self, W):
        M = self.maps
        Wi = W[:, M.ncin]
        Wp = W[:, M.part_in]
        return Wi, M.pressure(Wi), Wp, M.pressure(Wp)

    def _bc_jac(self, W, nrm):
        """Jacobians of every ghost (W 5, p 1) w.r.t. its interior cell and its
        coincident partner's interior (10 forward tangents)"""
        torch = self.torch
        M = self.maps
        nl = len(M.kind)
        bce = M.bceqt
        Wi0, _, Wp0, _ = self._bc_inputs(W)
        jac = torch.zeros((nl, 6, 10), dtype=torch.float64, device=W.device)
        for t in range(10):
            dWi = torch.zeros_like(Wi0)
            dWp = torch.zeros_like(Wp0)
            (dWi if t < 5 else dWp)[t % 5] = 1.0

            def f(wi, wp):
                g, pg = M.ghosts(wi, M.pressure(wi), wp, M.pressure(wp), nrm, bce)
                return torch.cat([g, pg[None]], 0)

            _, tan = torch.func.jvp(f, (Wi0, Wp0), (dWi, dWp))
            jac[:, :, t] = tan.T
        self.bcJ = jac

    def _chain(self, wbar):
        """A^T lambda on the real cells from the library's per-cell (W, p)
        parts: the pressure part through zpres on real cells, the ghost parts
        through the boundary maps to the interior"""
        torch = self.torch
        M = self.maps
        ld = M.ld
        wb = wbar.reshape(6, ld)
        out = wb[:5] + wb[5:6] * self.dp_dW
        g = torch.cat([wb[:5, M.ncbd], wb[5:6, M.ncbd]], 0)           # (6, nl)
        back = torch.einsum("eoi,oe->ie", self.bcJ, g)                # (10, nl)
        # layer by layer (one atomic scatter over all entries would sum the
        # two contributions of a block-corner cell in a varying order)
        for e in M.in_layers:
            out = out.index_add(1, M.ncin[e], back[:5, e])
        for e in M.part_layers:
            out = out.index_add(1, M.part_in[e], back[5:, e])
        return out.masked_fill(M.not_real, 0.0)

    def value_and_partials(self):
        """J and its explicit derivatives (state at real cells, wall nodes,
        Mach) at the converged state"""
        torch = self.torch
        M = self.maps
        dev = self.s.dev
        W = self.W.clone().requires_grad_(True)
        wall = torch.as_tensor(self.wall, device=dev).requires_grad_(True)
        mach = torch.tensor(self.mach, dtype=torch.float64, device=dev, requires_grad=True)
        P = M.nodes(wall)
        pg = M.pressure(W[:, M.ncin[M.wall_ent]])        # slip wall: ghost p = interior p
        J = M.functional(W, pg, P, mach, self.sgn_nx)
        gW, gwall, gm = torch.autograd.grad(J, (W, wall, mach))
        gW = gW.detach().clone()
        keep = torch.zeros_like(gW)
        keep[:, M.real] = gW[:, M.real]
        return float(J.detach()), keep, gwall, gm

    def solve_adjoint(self, g):
        """lambda += L^T (g - A^T lambda) until the relative residual is below
        adj_tol; one iteration (A^T lambda in the library, the boundary-map
        chain in torch, L^T in the library) is captured into a CUDA graph on
        the solver's stream and replayed"""
        torch = self.torch
        s = self.s
        ld = self.maps.ld
        lam = torch.zeros(5 * ld, dtype=torch.float64, device=s.dev)
        wbar = torch.zeros(6 * ld, dtype=torch.float64, device=s.dev)
        r = torch.zeros(5 * ld, dtype=torch.float64, device=s.dev)
        dl = torch.zeros(5 * ld, dtype=torch.float64, device=s.dev)
        gflat = g.reshape(-1).contiguous()
        gn = float(gflat.norm())

        def step():
            s.adjoint_rt(lam, wbar)
            r.copy_(gflat - self._chain(wbar).reshape(-1))
            s.adjoint_lt(r, dl)
            lam.add_(dl)

        hist = []
        it = 0
        graph = None
        if self.adj_max > 0:
            with torch.cuda.stream(s.stream):
                step()
            it = 1
            s.sync()
            try:
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph, stream=s.stream):
                    step()  # recorded, not run
            except Exception:
                graph = None
        while it < self.adj_max:
            with torch.cuda.stream(s.stream):
                if graph is not None:
                    graph.replay()
                else:
                    step()
            it += 1
            if it % self.check == 0:
                s.sync()
                rn = float(r.norm()) / max(gn, 1e-300)
                hist.append(rn)
                if not math.isfinite(rn):
                    raise RuntimeError("adjoint iteration diverged")
                if rn < self.adj_tol:
                    break
        s.sync()
        self.adj_iters = it
        self.adj_hist = hist
        return lam

    def gradient(self):
        """(J, dJ/dM, dJ/dalpha [per degree], dJ/dwall)"""
        torch = self.torch
        M = self.maps
        s = self.s
        dev = s.dev
        ld = M.ld
        J, gW, gwall_J, gm_J = self.value_and_partials()
        lam = self.solve_adjoint(gW)
        wbar = torch.zeros(6 * ld, dtype=torch.float64, device=dev)
        sbar = torch.zeros(9 * ld, dtype=torch.float64, device=dev)
        s.adjoint_rt(lam, wbar, sbar)
        s.sync()
        gwall_u, gm_u, ga_u = self._lin_grads(wbar, sbar)
        gwall = gwall_J - gwall_u
        gm = gm_J - gm_u
        ga = -ga_u
        return J, float(gm), float(ga), gwall.detach()

    def _lin_grads(self, wbar, sbar):
        """d(lambda^T u)/d(wall heights, Mach, angle) at the linearisation
        state self.W, from the library's per-cell wbar and per-face sbar of
        lambda: through the face areas and the boundary maps"""
        torch = self.torch
        M = self.maps
        dev = self.s.dev
        ld = M.ld
        wall = torch.as_tensor(self.wall, device=dev).requires_grad_(True)
        mach = torch.tensor(self.mach, dtype=torch.float64, device=dev, requires_grad=True)
        alpha = torch.tensor(self.alpha, dtype=torch.float64, device=dev, requires_grad=True)
        P = M.nodes(wall)
        sb = sbar.reshape(3, 3, ld)
        lin = torch.zeros((), dtype=torch.float64, device=dev)
        for dir in range(3):
            n = M.face_cells(dir)
            S = self.sgn[dir] * M.face_normals(P, dir, n)
            lin = lin + (S * sb[dir][:, n]).sum()
        nrm = M.boundary_normals(P, self.sgn)
        bce = M.bceqt.clone()
        s_prd = M.sel[cases.BC_PRD]
        s_idd = M.sel[cases.BC_IDD]
        bce = bce.index_put((torch.zeros_like(s_prd), s_prd),
                            p_inf(mach, M.gam).expand(len(s_prd)))
        ar = alpha * (math.pi / 180.0)
        bce = bce.index_put((torch.full_like(s_idd, 2), s_idd), torch.cos(ar).expand(len(s_idd)))
        bce = bce.index_put((torch.full_like(s_idd, 3), s_idd), torch.sin(ar).expand(len(s_idd)))
        Wi, pi, Wp, pp = self._bc_inputs(self.W)
        Wg, pg = M.ghosts(Wi, pi, Wp, pp, nrm, bce)
        wb = wbar.reshape(6, ld)
        lin = lin + (Wg * wb[:5, M.ncbd]).sum() + (pg * wb[5, M.ncbd]).sum()
        gwall_u, gm_u, ga_u = torch.autograd.grad(lin, (wall, mach, alpha), allow_unused=True)
        zero = torch.zeros((), dtype=torch.float64, device=dev)
        gm_u = zero if gm_u is None else gm_u
        ga_u = zero if ga_u is None else ga_u
        return gwall_u.detach(), gm_u.detach(), ga_u.detach()


class CheckpointedGradient(WallForceGradient):
    """Reverse accumulation of J(W_N) through N pseudo-time iterations of the
    primal, W_{n+1} = W_n + d(W_n) with d the implicit phase's increment,
    with pseudo-time checkpointing: the forward run keeps the state every
    `every` iterations; the reverse sweep takes the segments from the last to
    the first, recomputes each segment's states from its checkpoint, and
    steps back through them -- at most N/every + every states in memory
    instead of N.  Each reverse step linearises the iteration at its state
    W_n (library face-flux Jacobians and implicit coefficients, torch
    boundary maps):

        mu_n   = L_n^T wbar_{n+1}
        wbar_n = wbar_{n+1} - A_n^T mu_n
        dJ/dtheta -= d(mu_n^T u)/dtheta at W_n,

    from wbar_N = dJ/dW at W_N; L_n is the implicit phase linearised at
    d = 0, whose own dependence on the state is not differentiated (it
    multiplies the residual, zero at a steady state).  Over a converged
    history the sum of the mu_n after N reverse steps is the steady adjoint's
    lambda after N of its iterations, so the gradient tends to
    WallForceGradient's; for a history that has not converged it is the
    derivative of the truncated iteration with the implicit phase frozen.
    The start state is held fixed.  The adjoint states do not depend on
    `every` (the recomputed states are the forward run's, bit for bit); the
    parameter gradients agree to rounding (torch's scatter-adds into the wall
    nodes sum in a varying order)."""

    def __init__(self, design: Design, mach: float, alpha: float, wall: np.ndarray,
                 n_iter: int, every: int, start=None):
        import torch
        if n_iter < 1 or every < 1:
            raise ValueError("n_iter and every must be positive")
        self.torch = torch
        self.design = design
        self.mach, self.alpha = float(mach), float(alpha)
        self.wall = np.asarray(wall, dtype=float)
        self.case = design.case(mach, alpha, self.wall)
        self.n_iter, self.every = int(n_iter), int(every)
        s = CodeNS(self.case)
        s.metric()
        if start is not None:
            s.v.copy_(torch.as_tensor(np.ascontiguousarray(start).reshape(-1), device=s.dev))
            torch.cuda.synchronize()
        self.s = s
        self.maps = _Maps(self.case, torch, s.dev)
        # forward: checkpoints at n = 0, every, 2 every, ...
        self.ckpt = {}
        n = 0
        while n < self.n_iter:
            s.sync()
            self.ckpt[n] = s.v.detach().clone()
            k = min(self.every, self.n_iter - n)
            self.l2 = float(s.atsch_num(k)[1, 0])
            n += k
        s.sync()
        self.iters = self.n_iter
        self.max_states = 0  # the most states held at once in the reverse sweep
        self._setup()        # orientation and the linearisation at W_N

    def _set_state(self, W):
        self.s.sync()
        self.s.v.copy_(W)
        self.s.sync()

    def gradient(self):
        """(J(W_N), dJ/dM, dJ/dalpha [per degree], dJ/dwall) by reverse
        accumulation over the checkpointed history"""
        torch = self.torch
        M = self.maps
        s = self.s
        dev = s.dev
        ld = M.ld
        J, gW, gwall, gm = self.value_and_partials()      # at W_N (the last _setup)
        gwall = gwall.detach().clone()
        gm = gm.detach().clone()
        ga = torch.zeros((), dtype=torch.float64, device=dev)
        wb_state = gW.reshape(-1).contiguous()
        mu = torch.zeros(5 * ld, dtype=torch.float64, device=dev)
        wbar = torch.zeros(6 * ld, dtype=torch.float64, device=dev)
        sbar = torch.zeros(9 * ld, dtype=torch.float64, device=dev)
        self.mu_sum = torch.zeros(5 * ld, dtype=torch.float64, device=dev)
        for n0 in sorted(self.ckpt, reverse=True):
            k = min(self.every, self.n_iter - n0)
            # recompute the segment's states W_n0 .. W_{n0+k-1}
            states = [self.ckpt[n0]]
            self._set_state(self.ckpt[n0])
            for _ in range(k - 1):
                s.atsch_num(1)
                s.sync()
                states.append(s.v.detach().clone())
            self.max_states = max(self.max_states, len(states) + len(self.ckpt))
            for W_n in reversed(states):
                self._set_state(W_n)
                self._linearise()
                s.adjoint_lt(wb_state, mu)
                s.adjoint_rt(mu, wbar, sbar)
                s.sync()
                a = self._chain(wbar).reshape(-1)
                wb_state = (wb_state - a).contiguous()
                self.mu_sum += mu
                gw_u, gm_u, ga_u = self._lin_grads(wbar, sbar)
                gwall -= gw_u
                gm -= gm_u
                ga -= ga_u
        return J, float(gm), float(ga), gwall.detach()


def wall_force(design: Design, mach: float, alpha: float, wall: np.ndarray, **kw) -> float:
    """J at a design, from a converged primal (for finite differences).
    state: a converged (5, ld) state computed elsewhere (e.g. by the CPU
    restatement of the reference) to evaluate J at instead of solving"""
    g = WallForceGradient.__new__(WallForceGradient)
    import torch
    g.torch = torch
    g.design = design
    g.mach, g.alpha = float(mach), float(alpha)
    g.wall = np.asarray(wall, dtype=float)
    g.case = design.case(mach, alpha, g.wall)
    if kw.get("state") is not None:
        g.s = CodeNS(g.case)
        g.s.metric()
        g.s.v.copy_(torch.as_tensor(np.ascontiguousarray(kw["state"]).reshape(-1),
                                    device=g.s.dev))
        torch.cuda.synchronize()
        g.iters, g.l2 = 0, float("nan")
    else:
        g.s, g.iters, g.l2 = solve_primal(g.case, tol=kw.get("tol", 1e-13),
                                          max_iter=kw.get("max_iter", 40000))
    g.maps = _Maps(g.case, torch, g.s.dev)
    g.W = g.s.v.detach().reshape(5, g.maps.ld).clone()
    P0 = g.maps.nodes(torch.as_tensor(g.wall, device=g.s.dev))
    sn = g.s.sn.detach()
    b = g.maps.b
    g.sgn = []
    for dir in range(3):
        n = g.maps.face_cells(dir)
        S = g.maps.face_normals(P0, dir, n)
        ref = torch.stack([sn[9 * b.npc + c * 3 * b.nnn + dir * b.nnn + (n - b.npc)]
                           for c in range(3)])
        g.sgn.append(1.0 if float((S * ref).sum()) >= 0 else -1.0)
    nrm = g.maps.boundary_normals(P0, g.sgn)
    g.sgn_nx = torch.sign(nrm[0, g.maps.wall_ent])
    J = g.value_and_partials()[0]
    g.s.close()
    return J


def make_function():
    """torch.autograd.Function: J(mach, alpha, wall) with the adjoint in
    backward (design parameters other than these fixed by a Design)"""
    import torch

    class WallForce(torch.autograd.Function):
        @staticmethod
        def forward(ctx, mach, alpha, wall, design):
            # the local maps are differentiated with autograd inside (forward
            # runs with gradients disabled)
            with torch.enable_grad():
                g = WallForceGradient(design, float(mach), float(alpha),
                                      wall.detach().cpu().numpy())
                J, gm, ga, gw = g.gradient()
                g.close()
            ctx.save_for_backward(torch.tensor([gm, ga], dtype=torch.float64), gw.cpu())
            return torch.tensor(J, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gJ):
            gma, gw = ctx.saved_tensors
            return gJ * gma[0], gJ * gma[1], gJ * gw, None

    return WallForce
