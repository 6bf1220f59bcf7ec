"""Reference command decks (the ``flec`` file): a subset of the reference's
commands, enough to set up, run, save and restart a case of the hot path
from the reference's own deck, grid file and flow file.

Reading follows gtcmd.f90 / splcmd.f90: a line whose first character is
``#`` is a comment; ``&`` continues a command on the next line (the ``&``
itself becomes a blank and the rest of the line is dropped); words are
separated by blanks; carriage returns are ignored; an empty line is an
empty command.  Commands are interpreted in order (solve.f90:437-860) with
the reference's defaults (inimem.f90, defdfnm.f90, defdfph.f90,
defdfpmdtd.f90, defdfpmimd.f90, defdfpmdsd.f90, defdfpmdtg.f90,
defdffw.f90, defsecpfw.f90):

    create dom st l ni nj nk                      tcmd_crdms.f90 (real node counts)
    create boundary st mfbe kini l imin imax jmin jmax kmin kmax indmf
                                                  tcmd_crbds.f90, initis.f90
    define physics  [iflu i] [gammal g] [rgazl r] [pinfl p] [ql q]
                    [prandtll pr] [prandtlt prt] [reyref re]   tcmd_dfph.f90
    define numerics [nfi n] [fmg kfmg lgx kcg] [schema s] [muscl m xk ilim]
                    [prcd kprec cte kvisq] [dual kdualns tol niter tolke nitur]
                                                  tcmd_dfnm.f90 (fmg 3: dual time stepping,
                                                  compute flow = smg_num's physical time loop)
    define state n [ktype t] [roi r] [ai a] [ti t] [long l] [mach m]
                   [alpha a] [beta b]                          tcmd_dfst.f90
    define normaliz n                             tcmd_dfnzst.f90, dfnzst.f90, c_nzst.f90
    define flow [equat e] [krotation k] [vrotation w]           tcmd_dffw.f90
    define pm_dtd ldom l|* lgr g|* eta e          tcmd_dfpmdtd.f90
    define pm_dtg [kdtl k] [icychr0 i] [ncychro n] [dt1min d]   tcmd_dfpmdtg.f90
                    (the time step is recomputed on the iterations atsch_num.f90:173-178,
                    436 selects and kept in between)
    define pm_numd ldom l|* lgr g|* [ki2 a] [ki4 b]             tcmd_dfpmdsd.f90
    define pm_numi ldom l|* lgr g|* [kmf k] [lmax n]            tcmd_dfpmimd.f90
    init boundary basic mfbe|* clmf kibdb [file n] [state n | val/usi v.. | val/ref v..]
                                                  tcmd_inbdb.f90, inbdb.f90, inbdbst.f90, inbdbdf.f90
    init boundary coin mfbea frc mfbeb kibdc k [krr 0 ptc i j k dir ti tj tk | krr 1 epsmsh e]
                                                  tcmd_inbdc.f90
    init dom xyz ldom|* king                      tcmd_ingr.f90 (king /= 0: read fgv)
    init dom csvmut ldom|* kina [keinit k]        tcmd_infw.f90 (kina 0: read fac;
                                                  1: utinia.f90 from finia1)
    set env_cpfw [lgr g|* ncycle n] [...]         tcmd_secpfw.f90
    compute flow                                  cpfw.f90: ncycle iterations
    save dom xyz disc | save dom csvmut disc      tcmd_svgr.f90 / tcmd_svfw.f90
    end
    define title / define geometry / display / alloc / init boundary norm / partition
                                                  accepted, no effect on this path

What the subset does not handle raises ``DeckError`` naming the command:
boundary kinds other than extr, para, idd, prd and coincident joins;
boundaries that do not cover a whole block face; coincident joins whose
index directions are not the identity; turbulence models (equat(6:7) =
'ke'), multigrid (kfmg 1, 2), preconditioning (kprec /= 0),
explicit stepping (kmf = 0), rotating frames, and values of lmax that differ
between domains (eta, ki2 and ki4 may differ).  Files are the reference's
names in the deck's directory (fgv, fgc, fgcf, fac, facf, finia1).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from .cases import (BC_EXTR, BC_IDD, BC_LP2, BC_PARA, BC_PRD, BC_RC, Boundary, Case, Phys,
                    Scheme)
from .layout import Layout

REELMX = 1.7976931348623157e308   # huge(1.) with default real*8 (inimem.f90:119)
INTMX = 2147483647                # huge(1) (inimem.f90:118)
SUTHERLAND_C = 110.4              # zvismo.f90:79: 110.4/tnz


class DeckError(ValueError):
    pass


@dataclass
class Command:
    words: List[str]
    line: int

    def __str__(self):
        return f"line {self.line}: {' '.join(self.words)}"


def read_commands(text: str) -> List[Command]:
    """gtcmd.f90 + splcmd.f90: the deck's commands as word lists"""
    out: List[Command] = []
    lines = text.split("\n")
    p = 0
    while p < len(lines):
        first = p + 1
        buf = []
        while p < len(lines):
            line = lines[p].replace("\r", "")
            p += 1
            if line[:1] == "#":
                buf = None
                break
            amp = line.find("&")
            if amp >= 0:
                buf.append(line[:amp])
                continue
            buf.append(line)
            break
        if buf is None:
            continue
        words = [w for w in " ".join(buf).split(" ") if w]
        if words:
            out.append(Command(words, first))
    return out


def _int(cmd: Command, k: int) -> int:
    try:
        return int(cmd.words[k])
    except (IndexError, ValueError):
        raise DeckError(f"{cmd}: integer expected at word {k + 1}") from None


def _real(cmd: Command, k: int) -> float:
    try:
        return float(cmd.words[k].replace("d", "e").replace("D", "e"))
    except (IndexError, ValueError):
        raise DeckError(f"{cmd}: real expected at word {k + 1}") from None


def _word(cmd: Command, k: int) -> str:
    if k >= len(cmd.words):
        raise DeckError(f"{cmd}: word {k + 1} missing")
    return cmd.words[k]


def _list(cmd: Command, k: int, every: List[int]) -> List[int]:
    """lentier.f90: '*' is every entry, else one integer"""
    return list(every) if _word(cmd, k) == "*" else [_int(cmd, k)]


@dataclass
class DeckRun:
    """what running a deck produced"""
    solver: object
    norms: List[np.ndarray] = field(default_factory=list)   # after each compute flow
    files: List[str] = field(default_factory=list)          # files written
    inner: List[List[int]] = field(default_factory=list)    # dual time: inner iterations
    dual_started: bool = False


class Deck:
    """A parsed deck: the case it defines and the actions it asks for."""

    def __init__(self, path: str):
        self.path = os.path.abspath(path)
        self.dir = os.path.dirname(self.path)
        self.domains: Dict[int, tuple] = {}
        self.bnds: Dict[int, dict] = {}     # mfbe -> l, face, box (creation order)
        self.bc: Dict[int, tuple] = {}      # mfbe -> (clmf, values)
        self.coin: Dict[int, int] = {}      # mfbe -> partner mfbe
        self.states: Dict[int, dict] = {}
        # physics (defdfph.f90, defdfnm.f90)
        self.gam, self.rd, self.pinfl, self.pr, self.prt = 1.4, 287.13, 1.0, 0.72, 1.0
        self.reynz = REELMX
        self.tnz: Optional[float] = None
        self.equat = "eu3d   "
        self.omg = 0.0
        # numerics (defdfnm.f90, defdfpm*.f90)
        self.nfi, self.kfmg, self.lgx = 1, 0, 1
        self.kdualns, self.dual_tol, self.dual_niter = 0, 0.0, 1
        self.ischema, self.muscl, self.xk, self.ilim, self.kprec = 1, 0, 0.0, 0, 0
        self.eta: Dict[int, float] = {}
        self.lmax: Dict[int, int] = {}
        self.kmf: Dict[int, int] = {}
        self.ki2: Dict[int, float] = {}
        self.ki4: Dict[int, float] = {}
        self.kdtl, self.dt1min, self.ncychro, self.icychr0 = INTMX, REELMX, INTMX, 10
        self.ncycle = INTMX
        self.actions: List[tuple] = []
        with open(self.path) as f:
            for cmd in read_commands(f.read()):
                self._do(cmd)

    # ------------------------------------------------------------------
    def _do(self, c: Command):
        w = c.words
        head = w[0]
        two = w[1] if len(w) > 1 else ""
        if head == "#":
            return
        if head == "create" and two == "dom":
            if _word(c, 2) != "st":
                raise DeckError(f"{c}: 'create dom st' expected")
            self.domains[_int(c, 3)] = (_int(c, 4), _int(c, 5), _int(c, 6))
        elif head == "create" and two == "boundary":
            if _word(c, 2) != "st":
                raise DeckError(f"{c}: 'create boundary st' expected")
            mfbe, l = _int(c, 3), _int(c, 5)
            box = [_int(c, q) for q in range(6, 12)]
            face = _word(c, 12)
            self.bnds[mfbe] = dict(l=l, face=face, box=box, cmd=c)
        elif head == "define":
            self._define(c)
        elif head == "init" and two == "boundary":
            kind = _word(c, 2)
            if kind == "basic":
                self._inbdb(c)
            elif kind == "coin":
                self._inbdc(c)
            elif kind != "norm":
                raise DeckError(f"{c}: boundary initialisation not handled")
        elif head == "init" and two == "dom":
            kind = _word(c, 2)
            doms = _list(c, 3, sorted(self.domains))
            if kind == "xyz":
                self.actions.append(("ingr", doms, _int(c, 4), c))
            elif kind == "csvmut":
                keinit = 0
                if len(w) > 6 and w[5] == "keinit":
                    keinit = _int(c, 6)
                self.actions.append(("infw", doms, _int(c, 4), keinit, c))
            elif kind != "numt":
                raise DeckError(f"{c}: domain initialisation not handled")
        elif head == "set" and two == "env_cpfw":
            k = 2
            while k < len(w):
                if w[k] == "lgr" and k + 2 < len(w) and w[k + 2] == "ncycle":
                    self.ncycle = _int(c, k + 3)
                    k += 4
                else:
                    k += 2
        elif head == "compute" and two == "flow":
            self.actions.append(("cpfw", c))
        elif head == "save" and two == "dom":
            kind = _word(c, 2)
            if kind not in ("xyz", "csvmut"):
                raise DeckError(f"{c}: save not handled")
            self.actions.append(("svgr" if kind == "xyz" else "svfw", _word(c, 3), c))
        elif head == "end":
            self.actions.append(("end", c))
        elif head in ("display", "alloc", "partition"):
            return
        else:
            raise DeckError(f"{c}: command not handled")

    def _keywords(self, c: Command, table: dict, start: int = 2):
        """keyword-value pairs (tcmd_df*.f90): table maps a keyword to a
        setter taking the command and the index of its first value and
        returning the number of values consumed"""
        k = start
        w = c.words
        while k < len(w):
            f = table.get(w[k])
            if f is None:
                raise DeckError(f"{c}: unknown keyword {w[k]!r}")
            k += 1 + f(c, k + 1)

    def _define(self, c: Command):
        what = _word(c, 1)
        doms = sorted(self.domains)

        def setattr_(name, conv):
            def f(cc, k):
                setattr(self, name, conv(cc, k))
                return 1
            return f

        if what == "physics":
            self._keywords(c, {"iflu": lambda cc, k: 1, "gammal": setattr_("gam", _real),
                               "rgazl": setattr_("rd", _real), "pinfl": setattr_("pinfl", _real),
                               "ql": lambda cc, k: 1, "prandtll": setattr_("pr", _real),
                               "prandtlt": setattr_("prt", _real),
                               "reyref": setattr_("reynz", _real)})
        elif what == "numerics":
            def fmg(cc, k):
                self.kfmg, self.lgx = _int(cc, k), _int(cc, k + 1)
                return 3

            def muscl(cc, k):
                self.muscl, self.xk, self.ilim = _int(cc, k), _real(cc, k + 1), _int(cc, k + 2)
                return 3

            def prcd(cc, k):
                self.kprec = _int(cc, k)
                return 3

            def dual(cc, k):
                # kdualns tol niter tolke nitur (tolke, nitur: the transport
                # equations' inner loop, not handled here)
                self.kdualns, self.dual_tol = _int(cc, k), _real(cc, k + 1)
                self.dual_niter = _int(cc, k + 2)
                return 5

            self._keywords(c, {"nfi": setattr_("nfi", _int), "fmg": fmg,
                               "schema": setattr_("ischema", _int), "muscl": muscl,
                               "prcd": prcd, "dual": dual})
        elif what == "state":
            nst = _int(c, 2)
            st = self.states.setdefault(nst, {})
            k = 3
            if len(c.words) > k and c.words[k] == "ktype":
                k += 2
            names = ("roi", "ai", "ti", "long", "mach", "alpha", "beta")

            def val(name):
                def f(cc, q):
                    st[name] = _real(cc, q)
                    return 1
                return f
            self._keywords(c, {n: val(n) for n in names}, start=k)
        elif what == "normaliz":
            # dfnzst.f90 + c_nzst.f90: the state's density and temperature are
            # the reference values, so roa1 = aa1 = ta1 = 1 and pa1 = 1/gam
            st = self.states.get(_int(c, 2))
            if st is None or "ti" not in st:
                raise DeckError(f"{c}: the normalising state needs ti")
            self.tnz = st["ti"]
            self.ronz = st.get("roi", 1.0)
        elif what == "flow":
            def equat(cc, k):
                self.equat = _word(cc, k).ljust(7)[:7]
                return 1

            def krot(cc, k):
                if _int(cc, k) != 0:
                    raise DeckError(f"{cc}: rotating frames not handled")
                return 1
            self._keywords(c, {"equat": equat, "krotation": krot,
                               "vrotation": lambda cc, k: 1})
        elif what in ("pm_dtd", "pm_numd", "pm_numi"):
            per = {"pm_dtd": {"eta": (self.eta, _real)},
                   "pm_numd": {"ki2": (self.ki2, _real), "ki4": (self.ki4, _real)},
                   "pm_numi": {"kmf": (self.kmf, _int), "lmax": (self.lmax, _int)}}[what]
            sel = {"doms": doms}

            def ldom(cc, k):
                sel["doms"] = _list(cc, k, doms)
                return 1

            def one(dst, conv):
                def f(cc, k):
                    for l in sel["doms"]:
                        dst[l] = conv(cc, k)
                    return 1
                return f
            table = {"ldom": ldom, "lgr": lambda cc, k: 1}
            table.update({n: one(*v) for n, v in per.items()})
            self._keywords(c, table)
        elif what == "pm_dtg":
            self._keywords(c, {"kdtl": setattr_("kdtl", _int),
                               "icychr0": setattr_("icychr0", _int),
                               "ncychro": setattr_("ncychro", _int),
                               "dt1min": setattr_("dt1min", _real)})
        elif what in ("pm_turbn", "pm_turbp"):
            raise DeckError(f"{c}: turbulence models not handled")
        elif what in ("title", "geometry", "pm_cfg"):
            return
        else:
            raise DeckError(f"{c}: define {what} not handled")

    def _inbdb(self, c: Command):
        """tcmd_inbdb.f90 + inbdb.f90: boundary kind and values"""
        ids = _list(c, 3, sorted(self.bnds))
        clmf = _word(c, 4)[:4].ljust(4)
        k = 6
        w = c.words
        if len(w) > k and w[k] == "file":
            raise DeckError(f"{c}: boundary values from a file not handled")
        vals: List[float] = []
        ibddim = 0
        if len(w) > k:
            if w[k] == "state":
                vals, ibddim = self._bc_from_state(c, clmf, _int(c, k + 1)), 1
            elif w[k] in ("val/usi", "val/ref"):
                vals = [_real(c, q) for q in range(k + 1, len(w))]
                ibddim = 1 if w[k] == "val/usi" else 0
            else:
                raise DeckError(f"{c}: unknown value form {w[k]!r}")
        vals = self._bc_dimensions(c, clmf, ibddim, vals)
        for m in ids:
            if m not in self.bnds:
                raise DeckError(f"{c}: boundary {m} was not created")
            self.bc[m] = (clmf, vals)

    def _bc_from_state(self, c, clmf, nst):
        """inbdbst.f90"""
        st = self.states.get(nst)
        if st is None:
            raise DeckError(f"{c}: state {nst} not defined")
        gam = self.gam
        roist, tist = st.get("roi", 0.0), st.get("ti", 0.0)
        mast, alst, btst = st.get("mach", 0.0), st.get("alpha", 0.0), st.get("beta", 0.0)
        pist = roist * (1.0 / gam) * tist
        if clmf[:3] == "idd":
            return [pist, tist, alst, btst]
        if clmf in ("prd ", "prdp"):
            pspi = (1.0 + 0.5 * (gam - 1.0) * mast ** 2) ** (gam / (1.0 - gam))
            return [pspi * pist]
        return []

    def _bc_dimensions(self, c, clmf, ibddim, vals):
        """inbdbdf.f90 for the kinds handled here"""
        if clmf[:3] == "idd":
            if len(vals) < 2:
                raise DeckError(f"{c}: idd needs pi, ti")
            pdim, tdim = (1.0, 1.0) if ibddim == 0 else self._pt_ref(c)
            v = list(vals) + [0.0] * 5
            rpi, rti = v[0] / pdim, v[1] / tdim
            if len(vals) > 2:
                alf0 = v[2] * math.atan(1.0) / 45.0
                bet0 = v[3] * math.atan(1.0) / 45.0
            else:
                alf0 = bet0 = 0.0
            return [rpi, rti, math.cos(alf0) * math.cos(bet0), -math.cos(alf0) * math.sin(bet0),
                    math.sin(alf0)]
        if clmf in ("prd ", "prdp"):
            if clmf == "prdp":
                raise DeckError(f"{c}: boundary kind {clmf.strip()!r} not handled")
            if not vals:
                raise DeckError(f"{c}: prd needs a pressure")
            pdim = 1.0 if ibddim == 0 else self._pt_ref(c)[0]
            return [vals[0] / pdim * (1.0 / self.gam)]   # pa1 = roa1 ta1 / gam
        if clmf in ("extr", "para", "lp2 "):
            return []
        raise DeckError(f"{c}: boundary kind {clmf.strip()!r} not handled")

    def _pt_ref(self, c):
        """pnz, tnz of dfnzst.f90"""
        if self.tnz is None:
            raise DeckError(f"{c}: dimensional values need 'define normaliz' first")
        anz = math.sqrt(self.gam * self.rd * self.tnz)
        return self.ronz * anz ** 2 / self.gam, self.tnz

    def _inbdc(self, c: Command):
        """tcmd_inbdc.f90: mfbea frc mfbeb kibdc k [krr 0 ptc i j k dir ti tj tk |
        krr 1 epsmsh e]; only joins whose lists run in the same order"""
        a = _int(c, 3)
        if _word(c, 4) != "frc":
            raise DeckError(f"{c}: 'frc' expected")
        b = _int(c, 5)
        w = c.words
        if "krr" in w:
            q = w.index("krr")
            if _int(c, q + 1) == 0:
                if "dir" not in w:
                    raise DeckError(f"{c}: krr 0 needs dir")
                d = w.index("dir")
                dirs = [_word(c, d + 1), _word(c, d + 2), _word(c, d + 3)]
                for want, got in zip("ijk", dirs):
                    if got not in ("fa", "+" + want):
                        raise DeckError(f"{c}: index directions other than the identity "
                                        "not handled")
        for m in (a, b):
            if m not in self.bnds:
                raise DeckError(f"{c}: boundary {m} was not created")
        self.coin[a] = b
        self.bc[a] = ("rc  ", [])

    # ------------------------------------------------------------------
    def _uniform(self, name, per, default):
        vals = {per.get(l, default) for l in self.domains}
        if len(vals) > 1:
            raise DeckError(f"{name} differs between domains: not handled")
        return vals.pop() if vals else default

    def scheme(self) -> Scheme:
        if self.equat[2:4] != "3d":
            raise DeckError(f"equat {self.equat!r}: only 3-D equations are handled")
        if self.equat[5:7] == "ke":
            raise DeckError("turbulence models (equat 'ke') not handled")
        if self.nfi != 1 or self.kfmg not in (0, 3) or self.lgx != 1:
            raise DeckError("nfi 1, kfmg 0 or 3 (dual time) and one grid level only")
        if self.kfmg == 3 and self.dt1min == REELMX:
            raise DeckError("dual time stepping needs the physical step (pm_dtg dt1min)")
        if self.kprec != 0:
            raise DeckError("preconditioning (kprec) not handled")
        if self.ischema not in (1, 5, 7, 9, 14):
            raise DeckError(f"schema {self.ischema} not handled (1 Jameson, 5 AUSM+, 7 Roe, "
                            "9 Rusanov, 14 HLLC)")
        if self.ischema == 5 and self.equat[:2] != "ns":
            raise DeckError("schema 5 (AUSM+) runs with the Navier-Stokes equations only")
        if self._uniform("kmf", self.kmf, 1) != 1:
            raise DeckError("explicit stepping (kmf 0) not handled")
        ls = sorted(self.domains)
        per = {n: [getattr(self, n).get(l, dflt) for l in ls]
               for n, dflt in (("eta", 1.0), ("ki2", 0.0), ("ki4", 0.032))}
        return Scheme(ns=1 if self.equat[:2] == "ns" else 0, muscl=self.muscl, xk=self.xk,
                      ilim=self.ilim, eta=per["eta"][0] if ls else 1.0,
                      eta_l=per["eta"] if len(set(per["eta"])) > 1 else None,
                      ki2_l=per["ki2"] if len(set(per["ki2"])) > 1 else None,
                      ki4_l=per["ki4"] if len(set(per["ki4"])) > 1 else None,
                      kdtl=0 if self.kdtl == 0 else 1,
                      dt1min=self.dt1min if self.dt1min != REELMX else 0.0,
                      lmax=self._uniform("lmax", self.lmax, 10), ischema=self.ischema,
                      ki2=per["ki2"][0] if ls else 0.0,
                      ki4=per["ki4"][0] if ls else 0.032, ncychro=self.ncychro,
                      icychr0=self.icychr0, kfmg=self.kfmg, kdualns=self.kdualns)

    def phys(self) -> Phys:
        if self.tnz is None and self.equat[:2] == "ns":
            raise DeckError("Navier-Stokes needs 'define normaliz' (Sutherland's 110.4/tnz)")
        tnz = self.tnz if self.tnz is not None else 288.15
        return Phys(gam=self.gam, pinfl=self.pinfl, pr=self.pr, prt=self.prt,
                    reynz=self.reynz, suth_a=SUTHERLAND_C / tnz, pa1=1.0 / self.gam, aa1=1.0,
                    omg=self.omg)

    def layout(self) -> Layout:
        if not self.domains:
            raise DeckError("no domain created")
        ls = sorted(self.domains)
        if ls != list(range(1, len(ls) + 1)):
            raise DeckError("domains must be numbered 1..n")
        return Layout.from_dims([self.domains[l] for l in ls])

    def boundaries(self) -> List[Boundary]:
        kinds = {"extr": BC_EXTR, "para": BC_PARA, "idd ": BC_IDD, "prd ": BC_PRD,
                 "rc  ": BC_RC, "lp2 ": BC_LP2}
        order = list(self.bnds)
        pos = {m: q for q, m in enumerate(order)}
        out = []
        for m in order:
            bd = self.bnds[m]
            if m not in self.bc:
                raise DeckError(f"{bd['cmd']}: boundary {m} has no initialisation")
            clmf, vals = self.bc[m]
            l, face, box = bd["l"], bd["face"], bd["box"]
            ni, nj, nk = self.domains.get(l, (0, 0, 0))
            n = {"i": ni, "j": nj, "k": nk}
            want = []
            for q, ax in enumerate("ijk"):
                if ax == face[0]:
                    p = 1 if face[1] == "1" else n[ax]
                    want += [p, p]
                else:
                    want += [1, n[ax]]
            if face not in ("i1", "i2", "j1", "j2", "k1", "k2") or box != want:
                raise DeckError(f"{bd['cmd']}: only whole block faces are handled")
            partner = -1
            if clmf == "rc  ":
                other = self.coin[m]
                partner = pos[other]
            out.append(Boundary(l - 1, face, kinds[clmf], partner=partner,
                                values=tuple(vals)))
        for m, other in self.coin.items():
            if self.coin.get(other) != m:
                raise DeckError(f"coincident boundary {m}: its partner {other} must name it "
                                "back")
        return out

    def case(self) -> Case:
        lay = self.layout()
        z = np.zeros(lay.ld)
        return Case("deck", lay, self.phys(), self.scheme(), self.boundaries(), z, z.copy(),
                    z.copy(), np.zeros((5, lay.ld)), meta=dict(deck=self.path))

    # ------------------------------------------------------------------
    def utinia(self, solver) -> None:
        """utinia.f90:58-99: the finia1 state (mach, alpha, beta) on the real
        cells, computed on the host in the reference's expression order"""
        with open(os.path.join(self.dir, "finia1")) as f:
            rmach, alpha, beta = (float(t.replace("d", "e")) for t in f.read().split()[:3])
        ph = solver.case.phys
        gam = ph.gam
        gam1 = gam - 1.0
        gam2 = 0.5 * gam1
        gam4 = 1.0 / gam1
        roa1 = aa1 = 1.0
        ro = roa1 / (1.0 + gam2 * rmach ** 2) ** gam4
        a = aa1 / (1.0 + gam2 * rmach ** 2) ** 0.5
        p = (1.0 + gam2 * rmach ** 2) ** (-gam / gam1) / gam
        q = rmach * a
        degrad = math.atan2(1.0, 0.0) / 90.0
        alphar, betar = alpha * degrad, beta * degrad
        rou = ro * q * math.cos(alphar) * math.cos(betar)
        rov = -ro * q * math.sin(betar)
        row = ro * q * math.sin(alphar) * math.cos(betar)
        lay = solver.case.layout
        y = solver.y.cpu().numpy()
        z = solver.z.cpu().numpy()
        v = solver.v.cpu().numpy().reshape(solver.ncol, lay.ld).copy()
        for b in lay.blocks:
            n = b.real_cells()
            ci, cj, ck = 1, b.nid, b.nijd
            ym = 0.125 * (y[n] + y[n + ci] + y[n + cj] + y[n + ci + cj] + y[n + ck]
                          + y[n + ci + ck] + y[n + cj + ck] + y[n + ci + cj + ck])
            zm = 0.125 * (z[n] + z[n + ci] + z[n + cj] + z[n + ci + cj] + z[n + ck]
                          + z[n + ci + ck] + z[n + cj + ck] + z[n + ci + cj + ck])
            v[0, n] = ro
            v[1, n] = rou
            v[2, n] = rov + (ro * zm * ph.omg)
            v[3, n] = row - (ro * ym * ph.omg)
            v[4, n] = p / gam1 + ph.pinfl + 0.5 * (v[1, n] ** 2 + v[2, n] ** 2
                                                   + v[3, n] ** 2) / ro
        solver.v.copy_(solver.torch.as_tensor(v.reshape(-1)))
        if self.equat[:2] == "ns":
            solver.mut.zero_()

    def run(self, device: int | None = None) -> DeckRun:
        """execute the deck's actions on one GPU"""
        from .solver import CodeNS
        case = self.case()
        s = CodeNS(case, device=device)
        out = DeckRun(s)
        files = {"cvcv": "fgv", "cvcc": "fgc", "cvcf": "fgcf", "cccc": "fac", "cccf": "facf"}
        grid_read = False
        for act in self.actions:
            kind, cmd = act[0], act[-1]
            if kind == "ingr":
                doms, king = act[1], act[2]
                if king == 0:
                    raise DeckError(f"{cmd}: generated grids (king 0) not handled")
                if doms != sorted(self.domains):
                    raise DeckError(f"{cmd}: the grid is read for every domain at once")
                s.readdg(os.path.join(self.dir, "fgv"))
                grid_read = True
            elif kind == "infw":
                doms, kina, keinit = act[1], act[2], act[3]
                if doms != sorted(self.domains):
                    raise DeckError(f"{cmd}: the flow is initialised for every domain at once")
                if not grid_read:
                    raise DeckError(f"{cmd}: init dom xyz first")
                if kina == 0:
                    s.readda(os.path.join(self.dir, "fac"), self.equat, keinit=keinit)
                elif kina == 1:
                    self.utinia(s)
                else:
                    raise DeckError(f"{cmd}: kina {kina} not handled")
            elif kind == "cpfw":
                if self.ncycle == INTMX:
                    raise DeckError(f"{cmd}: set env_cpfw ... ncycle n first")
                if self.kfmg == 3:
                    # smg_num.f90:130-470: ncycle physical steps of at most
                    # niter inner iterations
                    out.inner.append(s.dual_time(self.ncycle, self.dual_niter, self.dual_tol,
                                                 start=not out.dual_started))
                    out.dual_started = True
                    out.norms.append(s.last_norms())
                else:
                    out.norms.append(s.atsch_num(self.ncycle))
            elif kind in ("svgr", "svfw"):
                disc = act[1]
                if disc not in files:
                    raise DeckError(f"{cmd}: disc {disc!r} not handled")
                path = os.path.join(self.dir, files[disc])
                if kind == "svgr":
                    s.writdg(path, disc)
                else:
                    s.writda(path, self.equat, disc)
                out.files.append(path)
            elif kind == "end":
                break
        return out
