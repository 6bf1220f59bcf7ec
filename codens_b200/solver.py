"""Host-side mirror of the reference's call surface for the hot path.

``CodeNS`` holds one case on one GPU: the context (what the Fortran reference
keeps in its modules) and the device arrays of the reference's flat layout,
allocated through torch (device memory and streams only).  Its methods carry
the reference routine names and argument meaning:

    zpres(l, v, pression, ztemp, cson)              zpres.f90
    zvismo(l, mu, v, ztemp)                         zvismo.f90
    chronos(l, mu, mut, v, dt, sn, vol, cson)       chronos.f90
    rbord(v, pression, ztemp, cson)                 rbord.f90
    sch_roe_euler(l, u, v, sn, ps)                  sch_roe_euler.f90
    sch_roe(l, u, v, tau, sn, ps)                   sch_roe.f90
    zvisqc(v, mu, mut, tau, sn, vol, ztemp)         zvisqc.f90
    implimf_eu(l, u, dt, v, d, sn, vol, ps, cson, lmx)
    implimf_3d(l, u, dt, v, d, mu, mut, sn, vol, ps, cson, lmx)
    rscpsv(u0, v, dt) -> (3, 5) L1/L2/Linf         rscpsv.f90 + residu.f90
    atsch_num(nsteps) -> norms of the last step     atsch_num.f90 (fused, graph)
    readdg(path) / writdg(path, disc)               readdg.f90 / svgr.f90 (fgv, fgc, fgcf)
    readda(path, equat) / writda(path, equat, disc) readda.f90 / svfw.f90 (fac, facf)

Block numbers are 1-based like the reference; ``l = 0`` runs every block in
one launch.  Every array argument is a float64 CUDA tensor in the reference
layout (column-major (ld, ncol) flattened).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .cases import Case


def _ptr(t):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype.is_floating_point and t.is_contiguous()):
        raise ValueError("arrays must be contiguous float64 CUDA tensors")
    return C.c_void_p(t.data_ptr())


def _arr(a):
    """a device tensor or a host numpy array (the copy-in/out parity mode of
    the per-routine entry points) as a pointer"""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise ValueError("host arrays must be contiguous float64")
        return C.c_void_p(a.ctypes.data)
    return _ptr(a)


def _offset(p, elems: int):
    return None if p is None else C.c_void_p(p.value + 8 * elems)


def _check_ke(equat: str, v, ld: int):
    if equat.ljust(7)[5:7] == "ke" and v.numel() < 7 * ld:
        raise ValueError("equat 'ke' reads and writes v(:,6:7): v must be (ld, 7)")


class CodeNS:
    def __init__(self, case: Case, device: int | None = None, stream=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("codens_b200 needs a CUDA device: there is no CPU path")
        self.torch = torch
        if device is not None:
            torch.cuda.set_device(device)
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self.lib = abi.load()
        self.case = case
        lay = case.layout
        self.ld = ld = lay.ld
        self.nreal = lay.nreal
        # host copies kept alive for the lifetime of the context
        self._dims = np.ascontiguousarray(lay.dims_array())
        ba = case.boundary_arrays()
        self._ba = {k: np.ascontiguousarray(v) for k, v in ba.items()}
        self._ba["bceqt"] = np.ascontiguousarray(ba["bceqt"].reshape(-1))
        self.nlist = len(self._ba["ncbd"])
        self._layout = abi.Layout_t(lay.nblk, self._dims.ctypes.data_as(C.POINTER(C.c_int32)), ld)
        p = case.phys
        self._phys = abi.Phys_t(p.gam, p.pinfl, p.pr, p.prt, p.reynz, p.suth_a, p.pa1,
                                p.aa1, p.omg)
        self._scheme = self._scheme_t(case.scheme)
        b = self._ba

        def ip(a, t):
            return a.ctypes.data_as(C.POINTER(t))

        self._bnd = abi.Bnd_t(len(b["type"]), ip(b["type"], C.c_int32), ip(b["blk"], C.c_int32),
                              ip(b["face"], C.c_int32), ip(b["mpb"], C.c_int64),
                              ip(b["mmb"], C.c_int32), ip(b["partner"], C.c_int32),
                              ip(b["cosr"], C.c_double), ip(b["sinr"], C.c_double),
                              self.nlist, ip(b["ncbd"], C.c_int64), ip(b["ncin"], C.c_int64),
                              ip(b["bceqt"], C.c_double))
        ctx = C.c_void_p()
        rc = self.lib.cns_create(C.byref(self._layout), C.byref(self._phys),
                                 C.byref(self._scheme), C.byref(self._bnd), C.byref(ctx))
        if rc:
            raise abi.CnsError(rc, "cns_create")
        self.ctx = ctx
        # every call of this solver is ordered on one stream (its own unless
        # the caller passes one, e.g. to serialise several solvers)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self._check(self.lib.cns_set_stream(ctx, C.c_void_p(self.stream.cuda_stream)),
                    "cns_set_stream")
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.x = torch.as_tensor(case.x, **f64).contiguous()
        self.y = torch.as_tensor(case.y, **f64).contiguous()
        self.z = torch.as_tensor(case.z, **f64).contiguous()
        # (ld, 5) conserved state, or (ld, 7) with the two transport variables
        self.ncol = ncol = int(case.v0.shape[0])
        self.v = torch.as_tensor(case.v0.reshape(-1), **f64).contiguous()
        self.u = torch.zeros(ncol * ld, **f64)
        self.d = torch.zeros(ncol * ld, **f64)
        self.dt = torch.zeros(ld, **f64)
        self.sn = torch.zeros(9 * ld, **f64)
        self.vol = torch.zeros(ld, **f64)
        self.pression = torch.zeros(ld, **f64)
        self.ztemp = torch.zeros(ld, **f64)
        self.cson = torch.zeros(ld, **f64)
        self.mu = torch.zeros(ld, **f64)
        self.mut = torch.zeros(ld, **f64)
        self.tau = torch.zeros(9 * ld, **f64)
        # dual time stepping: the physical-step arrays of smg_num.f90, (ld, 5)
        if int(getattr(case.scheme, "kfmg", 0)) == 3:
            self.ptdual, self.vdual, self.vdual1, self.vdual2 = (
                torch.zeros(5 * ld, **f64) for _ in range(4))
        else:
            self.ptdual = self.vdual = self.vdual1 = self.vdual2 = None
        torch.cuda.synchronize()
        st = abi.State_t(*[C.c_void_p(t.data_ptr()) if t is not None else None for t in
                           (self.v, self.u, self.d, self.dt, self.sn, self.vol,
                            self.pression, self.ztemp, self.cson, self.mu, self.mut,
                            self.tau, self.ptdual, self.vdual, self.vdual1, self.vdual2)])
        self._check(self.lib.cns_bind_state(ctx, C.byref(st)), "cns_bind_state")
        self._metric_done = False

    # ------------------------------------------------------------------
    @staticmethod
    def _scheme_t(s, qfix_dfez: int = 0):
        # per-block eta(lm), ki2(lm), ki4(lm): ctypes arrays kept on the struct
        keep = {}
        for name in ("eta_l", "ki2_l", "ki4_l"):
            vals = getattr(s, name, None)
            keep[name] = (C.c_double * len(vals))(*map(float, vals)) if vals is not None else None
        st = CodeNS._scheme_fields(s, qfix_dfez, keep)
        st._keep = keep
        return st

    @staticmethod
    def _scheme_fields(s, qfix_dfez, keep):
        return abi.Scheme_t(int(s.ns), int(s.muscl), float(s.xk), int(s.ilim), float(s.eta),
                            int(s.kdtl), float(s.dt1min), int(s.lmax),
                            int(getattr(s, "qfix_dfez", qfix_dfez)),
                            int(getattr(s, "precision", 0)), int(getattr(s, "kdefect", 4)),
                            int(getattr(s, "ischema", 7)), float(getattr(s, "ki2", 0.5)),
                            float(getattr(s, "ki4", 1.0 / 32.0)),
                            int(getattr(s, "ncychro", 1)), int(getattr(s, "icychr0", 0)),
                            int(getattr(s, "kfmg", 0)), int(getattr(s, "kdualns", 0)),
                            *(C.cast(keep[n], C.POINTER(C.c_double)) if keep[n] is not None
                              else None for n in ("eta_l", "ki2_l", "ki4_l")),
                            int(getattr(s, "weno_fix", 0)))

    def _check(self, rc: int, where: str):
        if rc:
            detail = self.lib.cns_last_error(self.ctx).decode() if getattr(self, "ctx", None) else ""
            raise abi.CnsError(rc, where, detail)

    def close(self):
        if getattr(self, "ctx", None):
            self.stream.synchronize()
            self.lib.cns_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_scheme(self, scheme, qfix_dfez: int = 0):
        self._scheme = self._scheme_t(scheme, qfix_dfez)
        self._check(self.lib.cns_set_scheme(self.ctx, C.byref(self._scheme)), "cns_set_scheme")

    def sync(self):
        self.stream.synchronize()

    @property
    def scratch_bytes(self) -> int:
        return int(self.lib.cns_scratch_bytes(self.ctx))

    def sweep_tiles(self, precision: int = 0):
        """(ti, tj, kc, tuned) of the Jacobi sweep tiling of a precision"""
        cfg = (C.c_int32 * 4)()
        self._check(self.lib.cns_sweep_tiles(self.ctx, precision, cfg), "cns_sweep_tiles")
        return tuple(int(x) for x in cfg)

    def set_sweep_tiles(self, precision: int, ti: int, tj: int, kc: int):
        self._check(self.lib.cns_set_sweep_tiles(self.ctx, precision, ti, tj, kc),
                    "cns_set_sweep_tiles")

    def set_tune_cache(self, path):
        """the sweep-tiling cache file (None: off); a configuration found there
        is used without timing"""
        self._check(self.lib.cns_set_tune_cache(self.ctx, None if path is None
                                                else str(path).encode()),
                    "cns_set_tune_cache")

    def residual_tiles(self):
        """(ti, tj, kc) of the fused residual, or zeros for the face kernels"""
        cfg = (C.c_int32 * 3)()
        self._check(self.lib.cns_residual_tiles(self.ctx, cfg), "cns_residual_tiles")
        return tuple(int(x) for x in cfg)

    @property
    def sweep_staging(self) -> int:
        """how the FP32 sweeps stage a plane: 0 tensor boxes, 1 cp.async"""
        m = C.c_int32()
        self._check(self.lib.cns_sweep_staging(self.ctx, C.byref(m)), "cns_sweep_staging")
        return int(m.value)

    def set_sweep_staging(self, mode: int):
        """0: tensor-box staging (the default); 1: cp.async element copies
        (the same bits)"""
        self._check(self.lib.cns_set_sweep_staging(self.ctx, mode), "cns_set_sweep_staging")

    def set_residual_tiles(self, ti: int, tj: int = 0, kc: int = 0):
        """ti = 0: the face kernels + accumulation; else the fused kernel"""
        self._check(self.lib.cns_set_residual_tiles(self.ctx, ti, tj, kc),
                    "cns_set_residual_tiles")

    @property
    def kernels_launched(self) -> int:
        """kernels launched so far by the fused-step graphs of this solver"""
        return int(self.lib.cns_kernels_launched(self.ctx))

    # ---- set-up -------------------------------------------------------
    def metric(self):
        """metric.f90: ghost nodes, sn, vol and the boundary-entry geometry."""
        self._check(self.lib.cns_metric(self.ctx, _ptr(self.x), _ptr(self.y), _ptr(self.z),
                                        _ptr(self.sn), _ptr(self.vol)), "cns_metric")
        self._metric_done = True

    def boundary_geom(self):
        out = [np.zeros(max(self.nlist, 1)) for _ in range(5)]
        self._check(self.lib.cns_boundary_geom(
            self.ctx, *[o.ctypes.data_as(C.POINTER(C.c_double)) for o in out]),
            "cns_boundary_geom")
        return [o[: self.nlist] for o in out]

    # ---- reference call surface ----------------------------------------
    # The C entry points take the reference routines' argument lists:
    # equat, the block's sn slice with lgsnlt = nnn(lm), the nine stress
    # arrays toxx..qcz, ityprk and ff, work arrays (passed as NULL here).
    def _equat(self, ns=None) -> bytes:
        ns = self.case.scheme.ns if ns is None else ns
        return b"ns3d   " if ns else b"eu3d   "

    def _sn(self, l, sn):
        """sn(npsn): the block's slice (lm >= 1) or the whole array (lm = 0),
        and lgsnlt"""
        if l == 0:
            return _arr(sn), self.ld
        b = self.case.layout.blocks[l - 1]
        return _offset(_arr(sn), 9 * b.npc), b.nnn

    def _tau9(self, tau):
        base = _arr(tau)
        if base is None:
            return [None] * 9
        return [_offset(base, a * self.ld) for a in range(9)]

    def zpres(self, l, v, pression, ztemp, cson):
        self._check(self.lib.cns_zpres(self.ctx, l, _arr(v), _arr(pression), _arr(ztemp),
                                       _arr(cson)), "cns_zpres")

    def zvismo(self, l, mu, v, ztemp):
        self._check(self.lib.cns_zvismo(self.ctx, l, _arr(mu), _arr(v), _arr(ztemp)),
                    "cns_zvismo")

    def chronos(self, l, mu, mut, v, dt, sn, vol, cson, etal=None):
        """chronos.f90 with the CFL etal (default: the block's eta)"""
        if etal is None:
            sc = self.case.scheme
            etal = sc.eta_l[l - 1] if (sc.eta_l is not None and l >= 1) else sc.eta
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_chronos(self.ctx, l, float(etal), _arr(mu), _arr(mut), _arr(v),
                                         _arr(dt), self._equat(), snp, lg, _arr(vol), None,
                                         None, None, None, _arr(cson)), "cns_chronos")

    def rbord(self, v, pression, ztemp, cson):
        self._check(self.lib.cns_rbord(self.ctx, _arr(v), _arr(pression), _arr(ztemp),
                                       _arr(cson)), "cns_rbord")

    def _flux_euler(self, fn, name, l, u, v, sn, ps, ityprk, ff, equat):
        snp, lg = self._sn(l, sn)
        self._check(fn(self.ctx, l, ityprk, _arr(u), _arr(v), _arr(ff), equat or b"eu3d   ",
                       snp, lg, *([None] * 10), _arr(ps)), name)

    def _flux_ns(self, fn, name, l, u, v, tau, sn, ps, ityprk, ff, equat, d=()):
        snp, lg = self._sn(l, sn)
        dd = [_arr(d[0])] if d else []
        self._check(fn(self.ctx, l, ityprk, _arr(u), _arr(v), *dd, _arr(ff), *self._tau9(tau),
                       equat or b"ns3d   ", snp, lg, *([None] * 10), _arr(ps)), name)

    def sch_roe_euler(self, l, u, v, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_euler(self.lib.cns_sch_roe_euler, "cns_sch_roe_euler", l, u, v, sn, ps,
                         ityprk, ff, equat)

    def sch_roe(self, l, u, v, tau, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_ns(self.lib.cns_sch_roe, "cns_sch_roe", l, u, v, tau, sn, ps, ityprk, ff,
                      equat)

    def sch_hllc_euler(self, l, u, v, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_euler(self.lib.cns_sch_hllc_euler, "cns_sch_hllc_euler", l, u, v, sn, ps,
                         ityprk, ff, equat)

    def sch_hllc(self, l, u, v, tau, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_ns(self.lib.cns_sch_hllc, "cns_sch_hllc", l, u, v, tau, sn, ps, ityprk, ff,
                      equat)

    def sch_weno5_3d(self, l, u, v, tau, sn, ps, ityprk=0, ff=None, equat=None):
        """the WENO5 residual of block l (sch_weno5_3d.f90; tau is read with
        either equations, zero for Euler)"""
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_sch_weno5_3d(self.ctx, l, ityprk, _arr(u), _arr(v), _arr(ff),
                                              *self._tau9(tau), equat or b"ns3d   ", snp, lg,
                                              *([None] * 9), _arr(ps)), "cns_sch_weno5_3d")

    def sch_rusanov(self, l, u, v, tau, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_ns(self.lib.cns_sch_rusanov, "cns_sch_rusanov", l, u, v, tau, sn, ps, ityprk,
                      ff, equat or self._equat())

    def sch_ausmp(self, l, u, v, tau, sn, ps, ityprk=0, ff=None, equat=None):
        self._flux_ns(self.lib.cns_sch_ausmp, "cns_sch_ausmp", l, u, v, tau, sn, ps, ityprk, ff,
                      equat, d=(None,))

    def chrono_global(self, dt):
        """chrono.f90:113-151: the global time step (kdtl = 0)"""
        self._check(self.lib.cns_chrono_global(self.ctx, _ptr(dt)), "cns_chrono_global")

    # discrete adjoint of the Euler Roe iteration (see codens_b200/adjoint.py)
    def adjoint_prepare(self):
        self._check(self.lib.cns_adjoint_prepare(self.ctx), "cns_adjoint_prepare")

    def adjoint_rt(self, lam, wbar, sbar=None):
        self._check(self.lib.cns_adjoint_rt(self.ctx, _ptr(lam), _ptr(wbar),
                                            None if sbar is None else _ptr(sbar)),
                    "cns_adjoint_rt")

    def adjoint_lt(self, y, out):
        self._check(self.lib.cns_adjoint_lt(self.ctx, _ptr(y), _ptr(out)), "cns_adjoint_lt")

    # Jameson scheme (dissip_jameson.f90, sch_jameson.f90, rfve.f90, rfvc.f90)
    def rfve(self, v, ps, ztemp, cson):
        self._check(self.lib.cns_rfve(self.ctx, _ptr(v), _ptr(ps), _ptr(ztemp), _ptr(cson)),
                    "cns_rfve")

    def rfvc(self, v, ps, ztemp, cson):
        self._check(self.lib.cns_rfvc(self.ctx, _ptr(v), _ptr(ps), _ptr(ztemp), _ptr(cson)),
                    "cns_rfvc")

    def dissip_jameson(self, l, v, d, sn, ps, cson):
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_dissip_jameson(self.ctx, l, _arr(v), _arr(d), self._equat(),
                                                snp, lg, None, _arr(ps), _arr(cson)),
                    "cns_dissip_jameson")

    def sch_jameson(self, l, u, v, d, tau, sn, ps, ityprk=0, ff=None):
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_sch_jameson(self.ctx, l, ityprk, _arr(u), _arr(v), _arr(d),
                                             _arr(ff), *self._tau9(tau), self._equat(), snp,
                                             lg, *([None] * 9), _arr(ps)), "cns_sch_jameson")

    # turbulence-transport terms (met_fludc, met_fludcsa, met_roe2o, met_roe2oh)
    def set_turbulence(self, alfak=1.0, alfae=1.3, sigma=2.0 / 3.0, epsroe=0.0):
        self._check(self.lib.cns_set_turbulence(self.ctx, alfak, alfae, sigma, epsroe),
                    "cns_set_turbulence")

    def met_fludc(self, l, mu, mut, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z):
        self._check(self.lib.cns_met_fludc(self.ctx, l, None, _arr(mu), _arr(mut), None, None,
                                           None, None, *(_arr(a) for a in (
                                               fd5x, fd5y, fd5z, fd6x, fd6y, fd6z))),
                    "cns_met_fludc")

    def met_fludcsa(self, l, s, mu, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z):
        self._check(self.lib.cns_met_fludcsa(self.ctx, l, *(_ptr(a) for a in (
            s, mu, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z))), "cns_met_fludcsa")

    def met_roe2o(self, l, t, d, sn, harten=False):
        f = self.lib.cns_met_roe2oh if harten else self.lib.cns_met_roe2o
        snp, lg = self._sn(l, sn)
        self._check(f(self.ctx, l, _arr(t), _arr(d), snp, lg, None, None, None),
                    "cns_met_roe2oh" if harten else "cns_met_roe2o")

    def met_samut(self, l, v, mu, mut):
        self._check(self.lib.cns_met_samut(self.ctx, l, _ptr(v), _ptr(mu), _ptr(mut)),
                    "cns_met_samut")

    def sch_turb(self, l, u, v, d, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z, ts6, ts7, sn, vol):
        self._check(self.lib.cns_sch_turb(self.ctx, l, *(_ptr(a) for a in (
            u, v, d, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z, ts6, ts7, sn, vol))), "cns_sch_turb")

    def teq_gradv(self, l, v, sn, vol, dv):
        self._check(self.lib.cns_teq_gradv(self.ctx, l, _ptr(v), _ptr(sn), _ptr(vol), _ptr(dv)),
                    "cns_teq_gradv")

    def met_smsa(self, l, v, mu, dist, sn, vol, dv, fd5x, fd5y, fd5z, ts6, ts7, cfke):
        self._check(self.lib.cns_met_smsa(self.ctx, l, *(_ptr(a) for a in (
            v, mu, dist, sn, vol, dv, fd5x, fd5y, fd5z, ts6, ts7, cfke))), "cns_met_smsa")

    def impli2_eqt_3d(self, l, u, dt, v, mu, mut, cfke, sn, vol, cmt=1.0):
        self._check(self.lib.cns_impli2_eqt_3d(self.ctx, l, *(_ptr(a) for a in (
            u, dt, v, mu, mut, cfke, sn, vol)), float(cmt)), "cns_impli2_eqt_3d")

    # --- the rest of the Spalart-Allmaras step (met_num.f90, 1SA) ---------
    def atcaldis3(self, dist=None):
        """wall distance of the real cells from this case's nodes"""
        if dist is None:
            dist = self.torch.zeros(self.ld, dtype=self.torch.float64, device=self.dev)
        self._check(self.lib.cns_atcaldis3(self.ctx, _ptr(self.x), _ptr(self.y), _ptr(self.z),
                                           _ptr(dist)), "cns_atcaldis3")
        return dist

    def met_bord(self, v, rokinf, roeinf):
        self._check(self.lib.cns_met_bord(self.ctx, _ptr(v), rokinf, roeinf), "cns_met_bord")

    def met_gradtr(self, l, s, sn, vol, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z):
        self._check(self.lib.cns_met_gradtr(self.ctx, l, *map(_ptr, (s, sn, vol, fd5x, fd5y, fd5z,
                                                                   fd6x, fd6y, fd6z))),
                    "cns_met_gradtr")

    def met_rbse(self, fd5x, fd5y, fd5z, fd6x, fd6y, fd6z):
        self._check(self.lib.cns_met_rbse(self.ctx, *map(_ptr, (fd5x, fd5y, fd5z, fd6x, fd6y,
                                                              fd6z))), "cns_met_rbse")

    def met_cutsa(self, l, v, epsk):
        self._check(self.lib.cns_met_cutsa(self.ctx, l, _ptr(v), epsk), "cns_met_cutsa")

    def set_sa(self, dist=None, rokinf=0.0, roeinf=0.0, epsk=1e-8, stilde_fix=0):
        """enable the Spalart-Allmaras step in the fused iteration (dist: the
        wall distance, device FP64; None disables it).  The state must have
        7 columns.  stilde_fix = 1: the non-reference source fix (modified
        vorticity, guarded derivative; see cns_sa_t)."""
        if dist is None:
            self._check(self.lib.cns_set_sa(self.ctx, None), "cns_set_sa")
            self._sa = None
            return
        if self.ncol != 7:
            raise ValueError("the Spalart-Allmaras step needs a (ld, 7) state")
        self._sa = (dist, abi.Sa_t(C.c_void_p(dist.data_ptr()), rokinf, roeinf, epsk,
                                   int(stilde_fix)))
        self._check(self.lib.cns_set_sa(self.ctx, C.byref(self._sa[1])), "cns_set_sa")

    def set_ke(self, rokinf=None, roeinf=0.0, epsk=1e-10, epse=1e-10):
        """enable the k-epsilon step of Jones & Launder ('2JL') in the fused
        iteration (rokinf None disables it); the state must have 7 columns"""
        if rokinf is None:
            self._check(self.lib.cns_set_ke(self.ctx, None), "cns_set_ke")
            return
        if self.ncol != 7:
            raise ValueError("the k-epsilon step needs a (ld, 7) state")
        ke = abi.Ke_t(rokinf, roeinf, epsk, epse)
        self._check(self.lib.cns_set_ke(self.ctx, C.byref(ke)), "cns_set_ke")

    def met_num(self):
        self._check(self.lib.cns_met_num(self.ctx), "cns_met_num")

    def met_prod(self, l, mut, s, dv, tprod, ncyc=1):
        self._check(self.lib.cns_met_prod(self.ctx, l, ncyc, _ptr(mut), _ptr(s), _ptr(dv),
                                          _ptr(tprod)), "cns_met_prod")

    def met_smke(self, l, sn, vol, v, mu, mut, tprod, cfke, dv, ts6, ts7):
        self._check(self.lib.cns_met_smke(self.ctx, l, _ptr(sn), _ptr(vol), _ptr(v), _ptr(mu),
                                          _ptr(mut), _ptr(tprod), _ptr(cfke), _ptr(dv),
                                          _ptr(ts6), _ptr(ts7)), "cns_met_smke")

    def met_kemut(self, l, v, mu, mut):
        self._check(self.lib.cns_met_kemut(self.ctx, l, _ptr(v), _ptr(mu), _ptr(mut)),
                    "cns_met_kemut")

    def met_cutke(self, l, v, epsk, epse):
        self._check(self.lib.cns_met_cutke(self.ctx, l, _ptr(v), epsk, epse), "cns_met_cutke")

    def met_inisa(self, l, v, mut, mu):
        self._check(self.lib.cns_met_inisa(self.ctx, l, _ptr(v), _ptr(mut), _ptr(mu)),
                    "cns_met_inisa")

    def met_inmut(self, l, mu, mut):
        self._check(self.lib.cns_met_inmut(self.ctx, l, _ptr(mu), _ptr(mut)), "cns_met_inmut")

    def met_ini(self, l, v, mut, mu, sn, vol, dv):
        self._check(self.lib.cns_met_ini(self.ctx, l, _ptr(v), _ptr(mut), _ptr(mu), _ptr(sn),
                                         _ptr(vol), _ptr(dv)), "cns_met_ini")

    def lpsa(self, l, v, mu, mut, dist, ztemp):
        """the wall law's rho nu~ and mut of block l's 'lp2' first cells
        (lpsa.f90; the floor is set_sa's epsk)"""
        self._check(self.lib.cns_lpsa(self.ctx, l, _ptr(v), _ptr(mu), _ptr(mut), _ptr(dist),
                                      _ptr(ztemp)), "cns_lpsa")

    def cllparoi1(self, v, dist, mu, mut, tau, ztemp):
        """the wall law's stresses and heat flux at every 'lp2' wall
        (cllparoi1.f90)"""
        self._check(self.lib.cns_cllparoi1(self.ctx, _ptr(v), _ptr(dist), _ptr(mu), _ptr(mut),
                                           _ptr(tau), _ptr(ztemp)), "cns_cllparoi1")

    # iteration counters and dual time stepping
    def set_cycle(self, ncyc: int, icyc: int):
        """the reference's ncyc, icyc of the last iteration done"""
        self._check(self.lib.cns_set_cycle(self.ctx, int(ncyc), int(icyc)), "cns_set_cycle")

    def sch_duin(self):
        self._check(self.lib.cns_sch_duin(self.ctx), "cns_sch_duin")

    def sch_duup(self):
        self._check(self.lib.cns_sch_duup(self.ctx), "cns_sch_duup")

    def set_dual_cycle(self, icycle: int):
        self._check(self.lib.cns_set_dual_cycle(self.ctx, int(icycle)), "cns_set_dual_cycle")

    def sch_dual(self, l, u, v, icycle, vol, ptdual):
        self._check(self.lib.cns_sch_dual(self.ctx, l, _ptr(u), _ptr(v), int(icycle), _ptr(vol),
                                          _ptr(ptdual)), "cns_sch_dual")

    def dual_time(self, ncycl: int, niter: int, tol: float, start: bool = True):
        """the physical time loop of smg_num.f90:130-470 for kfmg = 3: ncycl
        physical steps of at most niter pseudo-time iterations, each step
        ending when the density residual relative to the first iteration's
        falls to tol (dua_resro.f90; here from the fused step's L2 norm of
        (v - u0)/dt, which differs from dua_resro's by the constant factor
        1/sqrt(real cells), so only the last bits of the ratio can differ),
        then sch_duup.  start: run sch_duin first (a fresh physical time
        loop).  Returns the inner iteration count of each physical step."""
        if self.ptdual is None:
            raise ValueError("dual time stepping needs a case with scheme.kfmg = 3")
        if not self._metric_done:
            self.metric()
        if start:
            self.sch_duin()
            self._resno1 = None
        counts = []
        for icycle in range(1, ncycl + 1):
            self.set_dual_cycle(icycle)
            # smg_num.f90:130-147: icyc restarts with each physical step and
            # ncyc = icycle + iter - 1
            self.set_cycle(icycle - 1, 0)
            it = 0
            for it in range(1, niter + 1):
                norms = self.atsch_num(1)
                r = float(norms[1, 0])
                if self._resno1 is None:
                    self._resno1 = r if abs(r) >= np.finfo(np.float64).tiny else 1.0
                if r / self._resno1 <= tol:
                    break
            counts.append(it)
            self.sch_duup()
        return counts

    # reference grid and flow files (Fortran unformatted sequential)
    def set_subrecord_length(self, nbytes: int):
        self._check(self.lib.cns_set_subrecord_length(self.ctx, int(nbytes)),
                    "cns_set_subrecord_length")

    def readdg(self, path, x=None, y=None, z=None):
        """fgv: the real nodes of every block into x, y, z (default: this
        context's node arrays)"""
        x, y, z = (self.x if x is None else x, self.y if y is None else y,
                   self.z if z is None else z)
        self._check(self.lib.cns_readdg(self.ctx, os.fsencode(path), _ptr(x), _ptr(y), _ptr(z)),
                    "cns_readdg")

    def writdg(self, path, disc="cvcv", x=None, y=None, z=None):
        """svgr: disc cvcv (fgv, nodes), cvcc (fgc, cell centres), cvcf (fgcf,
        cell centres with the ghost layer)"""
        x, y, z = (self.x if x is None else x, self.y if y is None else y,
                   self.z if z is None else z)
        self._check(self.lib.cns_writdg(self.ctx, os.fsencode(path), disc.encode(), _ptr(x),
                                        _ptr(y), _ptr(z)), "cns_writdg")

    def readda(self, path, equat, v=None, mut=None, keinit=0):
        """fac: the real cells of v (and mut for 'ns', v(:,6:7) for 'ke')"""
        v = self.v if v is None else v
        mut = self.mut if mut is None else mut
        _check_ke(equat, v, self.ld)
        self._check(self.lib.cns_readda(self.ctx, os.fsencode(path), equat.encode(),
                                        int(keinit), _ptr(v), _ptr(mut)), "cns_readda")

    def writda(self, path, equat, disc="cccc", v=None, mut=None):
        """svfw: disc cccc (fac, real cells) or cccf (facf, with the ghost layer)"""
        v = self.v if v is None else v
        mut = self.mut if mut is None else mut
        _check_ke(equat, v, self.ld)
        self._check(self.lib.cns_writda(self.ctx, os.fsencode(path), disc.encode(),
                                        equat.encode(), _ptr(v), _ptr(mut)), "cns_writda")

    def zvisqc(self, v, mu, mut, tau, sn, vol, ztemp):
        self._check(self.lib.cns_zvisqc(self.ctx, _arr(v), _arr(mu), _arr(mut), _arr(tau),
                                        _arr(sn), _arr(vol), _arr(ztemp)), "cns_zvisqc")

    def _dtpas(self, dtpas):
        return float(self.case.scheme.dt1min if dtpas is None else dtpas)

    def implimf_eu(self, l, u, dt, v, d, sn, vol, ps, cson, lmx, ityprk=0, ff=None,
                   dtpas=None):
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_implimf_eu(self.ctx, l, _arr(u), _arr(dt), _arr(v), _arr(d),
                                            _arr(ff), b"eu3d   ", lmx, snp, lg, _arr(vol),
                                            self._dtpas(dtpas), ityprk, *([None] * 10),
                                            _arr(ps), _arr(cson)), "cns_implimf_eu")

    def implimf_3d(self, l, u, dt, v, d, mu, mut, sn, vol, ps, cson, lmx, ityprk=0, ff=None,
                   dtpas=None):
        snp, lg = self._sn(l, sn)
        self._check(self.lib.cns_implimf_3d(self.ctx, l, _arr(u), _arr(dt), _arr(v), _arr(d),
                                            _arr(ff), _arr(mu), _arr(mut), b"ns3d   ", lmx, snp,
                                            lg, _arr(vol), self._dtpas(dtpas), ityprk,
                                            *([None] * 10), _arr(ps), _arr(cson)),
                    "cns_implimf_3d")

    def rscpsv(self, u0, v, dt) -> np.ndarray:
        out = (C.c_double * 15)()
        self._check(self.lib.cns_rscpsv(self.ctx, _arr(u0), _arr(v), _arr(dt), out),
                    "cns_rscpsv")
        return np.array(out).reshape(3, 5)

    # ---- fused fast path ------------------------------------------------
    def atsch_num(self, nsteps: int = 1) -> np.ndarray:
        """nsteps pseudo-time iterations on the device-resident state (one
        CUDA graph per iteration); returns the L1/L2/Linf of the last one."""
        if not self._metric_done:
            self.metric()
        out = (C.c_double * 15)()
        self._check(self.lib.cns_atsch_num_step(self.ctx, int(nsteps), out),
                    "cns_atsch_num_step")
        return np.array(out).reshape(3, 5)

    def atsch_num_launch(self, nsteps: int = 1):
        """enqueue nsteps iterations on self.stream without waiting"""
        if not self._metric_done:
            self.metric()
        self._check(self.lib.cns_atsch_num_launch(self.ctx, int(nsteps)), "cns_atsch_num_launch")

    def last_norms(self) -> np.ndarray:
        out = (C.c_double * 15)()
        self._check(self.lib.cns_last_norms(self.ctx, out), "cns_last_norms")
        return np.array(out).reshape(3, 5)

    def atsch_num_host(self, v_host, nsteps: int = 1) -> np.ndarray:
        """Same through the host-array entry point: v_host (a pinned CPU
        float64 tensor of 5*ld) is copied in, advanced and copied back."""
        if not self._metric_done:
            self.metric()
        if v_host.is_cuda or v_host.dtype != self.torch.float64 or not v_host.is_contiguous():
            raise ValueError("v_host must be a contiguous float64 CPU tensor")
        out = (C.c_double * 15)()
        self._check(self.lib.cns_atsch_num_step_host(self.ctx, C.c_void_p(v_host.data_ptr()),
                                                     int(nsteps), out),
                    "cns_atsch_num_step_host")
        return np.array(out).reshape(3, 5)
