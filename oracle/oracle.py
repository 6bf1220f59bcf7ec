"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker of the CUDA product.  Parity status: UNPINNED (see
cns_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libcns_oracle.so")
_lib = None

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.orc_setup.argtypes = [C.c_int, _i32, C.c_int64]
        L.orc_pow.argtypes = [C.c_double, C.c_double]
        L.orc_pow.restype = C.c_double
        L.orc_exp.argtypes = [C.c_double]
        L.orc_exp.restype = C.c_double
        L.orc_setup.restype = C.c_int
        L.orc_set_phys.argtypes = [C.c_double] * 9
        L.orc_set_scheme.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int,
                                     C.c_double, C.c_int, C.c_double, C.c_int, C.c_int]
        L.orc_set_boundaries.argtypes = [C.c_int, _i32, _i32, _i32, _i64, _i32,
                                         _i32, _d, _d, C.c_int64, _i64, _i64, _d]
        L.orc_metric.argtypes = [_d] * 5
        L.orc_boundary_geom.argtypes = [_d] * 5
        L.orc_zpres.argtypes = [C.c_int, _d, _d, _d, _d]
        L.orc_zvismo.argtypes = [C.c_int, _d, _d]
        L.orc_chronos.argtypes = [C.c_int, _d, _d, _d, _d, _d, _d, _d]
        L.orc_chrono_global.argtypes = [_d]
        L.orc_rbord.argtypes = [_d, _d, _d, _d]
        L.orc_sch_roe_euler.argtypes = [C.c_int, _d, _d, _d, _d]
        L.orc_zvisqc.argtypes = [_d, _d, _d, _d, _d, _d, _d]
        L.orc_sch_roe.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.orc_implimf_eu.argtypes = [C.c_int, _d, _d, _d, _d, _d, _d, _d, _d, C.c_int]
        L.orc_implimf_3d.argtypes = [C.c_int, _d, _d, _d, _d, _d, _d, _d, _d, _d,
                                     _d, C.c_int]
        L.orc_rscpsv.argtypes = [_d, _d, _d, _d]
        L.orc_step.argtypes = [_d] * 12 + [C.c_int]
        L.orc_step.restype = C.c_int
        L.orc_set_dissipation.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_rfve.argtypes = [_d] * 4
        L.orc_rfvc.argtypes = [_d] * 4
        L.orc_dissip_jameson.argtypes = [C.c_int] + [_d] * 5
        L.orc_sch_jameson.argtypes = [C.c_int] + [_d] * 6
        L.orc_step_jameson.argtypes = [_d] * 13 + [C.c_int]
        L.orc_step_jameson.restype = C.c_int
        L.orc_met_fludc.argtypes = [C.c_int] + [_d] * 8 + [C.c_double] * 2
        L.orc_met_fludcsa.argtypes = [C.c_int] + [_d] * 8 + [C.c_double]
        L.orc_met_roe2o.argtypes = [C.c_int, _d, _d, _d, C.c_int, C.c_double]
        L.orc_met_samut.argtypes = [C.c_int, _d, _d, _d]
        L.orc_sch_turb.argtypes = [C.c_int] + [_d] * 13
        L.orc_teq_gradv.argtypes = [C.c_int] + [_d] * 4
        L.orc_met_smsa.argtypes = [C.c_int] + [_d] * 12
        L.orc_impli2_eqt_3d.argtypes = [C.c_int] + [_d] * 8 + [C.c_double]
        L.orc_atcaldis3.argtypes = [_d] * 4
        L.orc_atcaldis3.restype = C.c_int
        L.orc_met_bord.argtypes = [_d, C.c_double, C.c_double]
        L.orc_met_gradtr.argtypes = [C.c_int] + [_d] * 9
        L.orc_met_rbse.argtypes = [_d] * 6
        L.orc_met_cutsa.argtypes = [C.c_int, _d, C.c_double]
        L.orc_set_sa.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                 C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                 C.c_void_p]
        L.orc_met_num.argtypes = [_d] * 9
        L.orc_met_prod.argtypes = [C.c_int] + [_d] * 4
        L.orc_met_smke.argtypes = [C.c_int] + [_d] * 10
        L.orc_met_kemut.argtypes = [C.c_int, _d, _d, _d]
        L.orc_met_cutke.argtypes = [C.c_int, _d, C.c_double, C.c_double]
        L.orc_set_ke.argtypes = ([C.c_int] + [C.c_double] * 6 + [C.c_int, C.c_double] +
                                 [C.c_void_p] * 3)
        L.orc_met_num_ke.argtypes = [_d] * 8
        L.orc_met_inisa.argtypes = [C.c_int, _d, _d]
        L.orc_met_inmut.argtypes = [C.c_int, _d, _d]
        L.orc_met_ini.argtypes = [C.c_int] + [_d] * 5
        L.orc_lpsa.argtypes = [C.c_int] + [_d] * 5 + [C.c_double]
        L.orc_cllparoi1.argtypes = [_d] * 6
        L.orc_asin.argtypes = [C.c_double]
        L.orc_asin.restype = C.c_double
        L.orc_set_sa_fix.argtypes = [C.c_int]
        L.orc_set_block_scheme.argtypes = [C.c_void_p] * 3
        L.orc_sch_hllc_euler.argtypes = [C.c_int, _d, _d, _d, _d]
        L.orc_sch_hllc.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.orc_sch_rusanov.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.orc_sch_weno5_3d.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.orc_set_weno_fix.argtypes = [C.c_int]
        L.orc_sch_ausmp.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.orc_set_dual.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_sch_dual.argtypes = [C.c_int, _d, _d, C.c_int, _d, _d]
        L.orc_sch_duin.argtypes = [_d] * 5
        L.orc_sch_duup.argtypes = [_d] * 5
        cs = C.c_char_p
        L.orc_writdg.argtypes = [cs, cs, _d, _d, _d, C.c_int64]
        L.orc_readdg.argtypes = [cs, _d, _d, _d]
        L.orc_writda.argtypes = [cs, cs, cs, _d, _d, C.c_int64]
        L.orc_readda.argtypes = [cs, cs, C.c_int, _d, _d]
        _lib = L
    return _lib


class OracleState:
    """Host arrays of one case, in the reference's flat layout."""

    def __init__(self, case):
        ld = case.layout.ld
        self.ld = ld
        self.x = case.x.copy()
        self.y = case.y.copy()
        self.z = case.z.copy()
        self.sn = np.zeros(9 * ld)
        self.vol = np.zeros(ld)
        self.v = np.ascontiguousarray(case.v0.reshape(-1)).copy()
        ncol = int(case.v0.shape[0])   # 5, or 7 with the transport variables
        self.u = np.zeros(ncol * ld)
        self.d = np.zeros(ncol * ld)
        self.dis = np.zeros(5 * ld)   # Jameson dissipation
        self.dt = np.zeros(ld)
        self.ps = np.zeros(ld)
        self.temp = np.zeros(ld)
        self.cson = np.zeros(ld)
        self.mu = np.zeros(ld)
        self.mut = np.zeros(ld)
        self.tau = np.zeros(9 * ld)


class Oracle:
    """The reference hot path on the CPU, one case at a time (the library keeps
    module-global state like the Fortran reference, so only one Oracle is
    active at a time)."""

    def __init__(self, case):
        self.case = case
        L = lib()
        lay = case.layout
        rc = L.orc_setup(lay.nblk, lay.dims_array(), lay.ld)
        if rc:
            raise ValueError(f"orc_setup failed ({rc})")
        p = case.phys
        L.orc_set_phys(p.gam, p.pinfl, p.pr, p.prt, p.reynz, p.suth_a, p.pa1,
                       p.aa1, p.omg)
        self.set_scheme(case.scheme)
        self.clear_sa()
        L.orc_set_dual(0, 0, 0, None)
        self._dual = None
        ba = case.boundary_arrays()
        self._ba = ba
        L.orc_set_boundaries(len(ba["type"]), ba["type"], ba["blk"], ba["face"],
                             ba["mpb"], ba["mmb"], ba["partner"], ba["cosr"],
                             ba["sinr"], len(ba["ncbd"]), ba["ncbd"], ba["ncin"],
                             np.ascontiguousarray(ba["bceqt"].reshape(-1)))

    def set_scheme(self, s):
        lib().orc_set_scheme(s.ns, s.muscl, s.xk, s.ilim, s.eta, s.kdtl,
                             s.dt1min, s.lmax, int(getattr(s, "qfix_dfez", 0)))
        lib().orc_set_dissipation(int(getattr(s, "ischema", 7)), float(getattr(s, "ki2", 0.5)),
                                  float(getattr(s, "ki4", 1.0 / 32.0)))
        lib().orc_set_weno_fix(int(getattr(s, "weno_fix", 0)))
        self.jameson = int(getattr(s, "ischema", 7)) <= 4
        self._block = [None if getattr(s, n, None) is None
                       else np.ascontiguousarray(getattr(s, n), dtype=np.float64)
                       for n in ("eta_l", "ki2_l", "ki4_l")]
        lib().orc_set_block_scheme(*[None if a is None else a.ctypes.data for a in self._block])
        self.ncyc = 0

    def set_sa(self, st: OracleState, dist, rokinf: float, roeinf: float, epsk: float = 1e-8,
               epsroe: float = 0.0, sigma: float = 2.0 / 3.0, stilde_fix: int = 0):
        """run the Spalart-Allmaras step (met_num, 1SA) in every iteration
        from now on; dist: the wall distance (kept referenced here)"""
        ld = self.case.layout.ld
        self._sa = dict(dist=np.ascontiguousarray(dist, dtype=np.float64),
                        fd=np.zeros(6 * ld), ts=np.zeros(2 * ld), cfke=np.zeros(ld))
        harten = int(abs(epsroe) > 1.17549435082228751e-38)
        a = self._sa
        lib().orc_set_sa(1, a["dist"].ctypes.data, rokinf, roeinf, epsk, harten, epsroe, sigma,
                         a["fd"].ctypes.data, a["ts"].ctypes.data, a["cfke"].ctypes.data)
        lib().orc_set_sa_fix(int(stilde_fix))

    def set_ke(self, st: OracleState, rokinf: float, roeinf: float, epsk: float = 1e-10,
               epse: float = 1e-10, epsroe: float = 0.0, alfak: float = 1.0,
               alfae: float = 1.3):
        """run the k-epsilon step of Jones & Launder (met_num, '2JL') in every
        iteration from now on"""
        ld = self.case.layout.ld
        self._ke = dict(fd=np.zeros(6 * ld), ts=np.zeros(2 * ld), cfke=np.zeros(ld))
        harten = int(abs(epsroe) > 1.17549435082228751e-38)
        a = self._ke
        lib().orc_set_ke(1, rokinf, roeinf, epsk, epse, alfak, alfae, harten, epsroe,
                         a["fd"].ctypes.data, a["ts"].ctypes.data, a["cfke"].ctypes.data)

    def set_dual(self, st: OracleState, kdualns: int = 0):
        """dual time stepping (kfmg = 3; the scheme's dt1min is the physical
        time step): allocates ptdual, vdual, vdual1, vdual2 on the state and
        runs sch_duin on its v"""
        ld = st.ld
        st.ptdual, st.vdual, st.vdual1, st.vdual2 = (np.zeros(5 * ld) for _ in range(4))
        self._dual = (kdualns, st.ptdual)
        lib().orc_set_dual(3, kdualns, 1, st.ptdual.ctypes.data)
        lib().orc_sch_duin(st.v[:5 * ld], st.ptdual, st.vdual, st.vdual1, st.vdual2)

    def set_dual_cycle(self, icycle: int):
        kdualns, pt = self._dual
        lib().orc_set_dual(3, kdualns, int(icycle), pt.ctypes.data)

    def sch_duup(self, st: OracleState):
        lib().orc_sch_duup(st.v[:5 * st.ld], st.ptdual, st.vdual, st.vdual1, st.vdual2)

    def clear_sa(self):
        lib().orc_set_sa(0, None, 0.0, 0.0, 0.0, 0, 0.0, 1.0, None, None, None)
        lib().orc_set_sa_fix(0)
        lib().orc_set_ke(0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0, 0.0, None, None, None)
        self._sa = None
        self._ke = None

    def metric(self, st: OracleState):
        lib().orc_metric(st.x, st.y, st.z, st.sn, st.vol)

    # reference grid and flow files; each returns the routine's code
    # (0, 1 bad disc, 8 file error, 9 records do not match the layout)
    @staticmethod
    def writdg(path, disc, x, y, z, maxsub=2147483639) -> int:
        return lib().orc_writdg(os.fsencode(path), disc.encode(), x, y, z, maxsub)

    @staticmethod
    def readdg(path, x, y, z) -> int:
        return lib().orc_readdg(os.fsencode(path), x, y, z)

    @staticmethod
    def writda(path, disc, equat, v, mut, maxsub=2147483639) -> int:
        return lib().orc_writda(os.fsencode(path), disc.encode(), equat.encode(), v, mut, maxsub)

    @staticmethod
    def readda(path, equat, v, mut, keinit=0) -> int:
        return lib().orc_readda(os.fsencode(path), equat.encode(), int(keinit), v, mut)

    def boundary_geom(self):
        n = len(self._ba["ncbd"])
        out = [np.zeros(max(n, 1)) for _ in range(5)]
        lib().orc_boundary_geom(*out)
        return [o[:n] for o in out]

    def step(self, st: OracleState, compute_dt: bool = True):
        """one iteration: atsch_num's Roe or Jameson sequence by ischema
        (the Jameson one extrapolates the physical ghosts on the first cycle)"""
        self.ncyc += 1
        if self.jameson:
            return lib().orc_step_jameson(st.v, st.u, st.d, st.dis, st.dt, st.sn, st.vol,
                                          st.ps, st.temp, st.cson, st.mu, st.mut, st.tau,
                                          int(self.ncyc == 1))
        return lib().orc_step(st.v, st.u, st.d, st.dt, st.sn, st.vol, st.ps,
                              st.temp, st.cson, st.mu, st.mut, st.tau,
                              int(compute_dt))

    def norms(self, u0, st: OracleState):
        out = np.zeros(15)
        lib().orc_rscpsv(u0, st.v, st.dt, out)
        return out.reshape(3, 5)
