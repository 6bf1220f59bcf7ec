"""ctypes bindings of libcodens_b200.so (include/cns_abi.h).

The product path has no CPU fallback: if the CUDA library is missing or no
GPU is visible, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

c_i32, c_i64, c_f64 = C.c_int32, C.c_int64, C.c_double
P = C.POINTER

ERRORS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-positive temperature",
    4: "time step below dt1min", 5: "unknown boundary condition",
    6: "not ready", 7: "non-finite residual norm", 8: "file error",
    9: "file does not match the layout",
}
(CNS_OK, CNS_EINVAL, CNS_ECUDA, CNS_ETEMP, CNS_EDT, CNS_EBC, CNS_ENOTREADY,
 CNS_ENONFINITE, CNS_EIO, CNS_EFORMAT) = range(10)


class Layout_t(C.Structure):
    _fields_ = [("nblk", c_i32), ("dims", P(c_i32)), ("ld", c_i64)]


class Phys_t(C.Structure):
    _fields_ = [(n, c_f64) for n in
                ("gam", "pinfl", "pr", "prt", "reynz", "suth_a", "pa1", "aa1", "omg")]


class Scheme_t(C.Structure):
    _fields_ = [("ns", c_i32), ("muscl", c_i32), ("xk", c_f64), ("ilim", c_i32),
                ("eta", c_f64), ("kdtl", c_i32), ("dt1min", c_f64), ("lmax", c_i32),
                ("qfix_dfez", c_i32), ("precision", c_i32), ("kdefect", c_i32),
                ("ischema", c_i32), ("ki2", c_f64), ("ki4", c_f64), ("ncychro", c_i32),
                ("icychr0", c_i32), ("kfmg", c_i32), ("kdualns", c_i32),
                ("eta_l", P(c_f64)), ("ki2_l", P(c_f64)), ("ki4_l", P(c_f64)),
                ("weno_fix", c_i32)]


class Ke_t(C.Structure):
    _fields_ = [("rokinf", c_f64), ("roeinf", c_f64), ("epsk", c_f64), ("epse", c_f64)]


class Bnd_t(C.Structure):
    _fields_ = [("nbnd", c_i32), ("type", P(c_i32)), ("blk", P(c_i32)),
                ("face", P(c_i32)), ("mpb", P(c_i64)), ("mmb", P(c_i32)),
                ("partner", P(c_i32)), ("cosr", P(c_f64)), ("sinr", P(c_f64)),
                ("nlist", c_i64), ("ncbd", P(c_i64)), ("ncin", P(c_i64)),
                ("bceqt", P(c_f64))]


class Sa_t(C.Structure):
    _fields_ = [("dist", C.c_void_p), ("rokinf", c_f64), ("roeinf", c_f64), ("epsk", c_f64),
                ("stilde_fix", c_i32)]


class State_t(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in
                ("v", "u", "d", "dt", "sn", "vol", "pression", "ztemp", "cson",
                 "mu", "mut", "tau", "ptdual", "vdual", "vdual1", "vdual2")]


EXPORTS = [
    "cns_create", "cns_destroy", "cns_set_stream", "cns_set_scheme",
    "cns_last_error", "cns_scratch_bytes", "cns_kernels_launched", "cns_metric", "cns_boundary_geom",
    "cns_zpres", "cns_zvismo", "cns_chronos", "cns_rbord", "cns_sch_roe_euler",
    "cns_sch_roe", "cns_zvisqc", "cns_implimf_eu", "cns_implimf_3d",
    "cns_rscpsv", "cns_bind_state", "cns_atsch_num_step",
    "cns_atsch_num_launch", "cns_last_norms", "cns_atsch_num_step_host",
    "cns_sch_roe_euler_noalloc", "cns_sweep_tiles", "cns_set_sweep_tiles",
    "cns_set_residual_tiles", "cns_residual_tiles", "cns_set_tune_cache",
    "cns_set_sweep_staging", "cns_sweep_staging",
    "cns_rfve", "cns_rfvc", "cns_dissip_jameson", "cns_sch_jameson",
    "cns_chrono_global", "cns_adjoint_prepare", "cns_adjoint_rt", "cns_adjoint_lt",
    "cns_set_turbulence", "cns_met_fludc", "cns_met_fludcsa", "cns_met_roe2o", "cns_met_roe2oh",
    "cns_met_samut", "cns_sch_turb", "cns_teq_gradv", "cns_met_smsa", "cns_impli2_eqt_3d",
    "cns_atcaldis3", "cns_met_bord", "cns_met_gradtr", "cns_met_rbse", "cns_met_cutsa",
    "cns_set_sa", "cns_met_num", "cns_lpsa", "cns_cllparoi1", "cns_set_ke", "cns_met_prod",
    "cns_met_smke", "cns_met_kemut", "cns_met_cutke", "cns_met_inisa", "cns_met_inmut",
    "cns_met_ini",
    "cns_set_subrecord_length", "cns_readdg", "cns_writdg", "cns_readda", "cns_writda",
    "cns_set_cycle", "cns_sch_duin", "cns_sch_duup", "cns_set_dual_cycle", "cns_sch_dual",
    "cns_sch_hllc_euler", "cns_sch_hllc", "cns_sch_rusanov", "cns_sch_ausmp",
    "cns_sch_weno5_3d",
]

_lib = None


def load(build_if_missing: bool = True):
    """Load the CUDA library (building it in-tree if needed)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"{path} is missing; build it with codens_b200/build.py")
        _build.build()
    L = C.CDLL(path)
    vp = C.c_void_p
    L.cns_create.argtypes = [P(Layout_t), P(Phys_t), P(Scheme_t), P(Bnd_t), P(vp)]
    L.cns_destroy.argtypes = [vp]
    L.cns_set_stream.argtypes = [vp, vp]
    L.cns_set_scheme.argtypes = [vp, P(Scheme_t)]
    L.cns_last_error.argtypes = [vp]
    L.cns_last_error.restype = C.c_char_p
    L.cns_scratch_bytes.argtypes = [vp]
    L.cns_scratch_bytes.restype = c_i64
    L.cns_kernels_launched.argtypes = [vp]
    L.cns_kernels_launched.restype = c_i64
    L.cns_metric.argtypes = [vp] * 6
    L.cns_boundary_geom.argtypes = [vp] + [P(c_f64)] * 5
    L.cns_zpres.argtypes = [vp, C.c_int] + [vp] * 4
    L.cns_zvismo.argtypes = [vp, C.c_int] + [vp] * 3
    cs, i64 = C.c_char_p, c_i64
    # the reference's argument lists (include/cns_abi.h); work arrays as vp
    L.cns_chronos.argtypes = ([vp, C.c_int, c_f64] + [vp] * 3 + [vp, cs, vp, i64, vp] + [vp] * 4
                              + [vp])
    L.cns_rbord.argtypes = [vp] * 5
    L.cns_sch_roe_euler.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, cs, vp, i64] + [vp] * 11
    L.cns_sch_roe.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp] + [vp] * 9 + [cs, vp, i64] + \
        [vp] * 11
    L.cns_zvisqc.argtypes = [vp] * 8
    L.cns_implimf_eu.argtypes = ([vp, C.c_int] + [vp] * 5 + [cs, C.c_int, vp, i64, vp, c_f64,
                                                             C.c_int] + [vp] * 10 + [vp] * 2)
    L.cns_implimf_3d.argtypes = ([vp, C.c_int] + [vp] * 7 + [cs, C.c_int, vp, i64, vp, c_f64,
                                                             C.c_int] + [vp] * 10 + [vp] * 2)
    L.cns_rscpsv.argtypes = [vp] * 4 + [P(c_f64)]
    L.cns_bind_state.argtypes = [vp, P(State_t)]
    L.cns_atsch_num_step.argtypes = [vp, C.c_int, P(c_f64)]
    L.cns_atsch_num_launch.argtypes = [vp, C.c_int]
    L.cns_last_norms.argtypes = [vp, P(c_f64)]
    L.cns_sweep_tiles.argtypes = [vp, C.c_int, P(c_i32)]
    L.cns_rfve.argtypes = [vp] * 5
    L.cns_rfvc.argtypes = [vp] * 5
    L.cns_dissip_jameson.argtypes = [vp, C.c_int, vp, vp, cs, vp, i64, vp, vp, vp]
    L.cns_sch_jameson.argtypes = ([vp, C.c_int, C.c_int] + [vp] * 4 + [vp] * 9 + [cs, vp, i64]
                                  + [vp] * 9 + [vp])
    L.cns_set_turbulence.argtypes = [vp] + [c_f64] * 4
    L.cns_chrono_global.argtypes = [vp, vp]
    L.cns_adjoint_prepare.argtypes = [vp]
    L.cns_adjoint_rt.argtypes = [vp] * 4
    L.cns_adjoint_lt.argtypes = [vp] * 3
    L.cns_met_fludc.argtypes = [vp, C.c_int] + [vp] * 13
    L.cns_met_fludcsa.argtypes = [vp, C.c_int] + [vp] * 8
    L.cns_met_roe2o.argtypes = [vp, C.c_int, vp, vp, vp, i64, vp, vp, vp]
    L.cns_met_roe2oh.argtypes = [vp, C.c_int, vp, vp, vp, i64, vp, vp, vp]
    L.cns_met_samut.argtypes = [vp, C.c_int] + [vp] * 3
    L.cns_sch_turb.argtypes = [vp, C.c_int] + [vp] * 13
    L.cns_teq_gradv.argtypes = [vp, C.c_int] + [vp] * 4
    L.cns_met_smsa.argtypes = [vp, C.c_int] + [vp] * 12
    L.cns_impli2_eqt_3d.argtypes = [vp, C.c_int] + [vp] * 8 + [c_f64]
    L.cns_atcaldis3.argtypes = [vp] * 5
    L.cns_met_bord.argtypes = [vp, vp, c_f64, c_f64]
    L.cns_met_gradtr.argtypes = [vp, C.c_int] + [vp] * 9
    L.cns_met_rbse.argtypes = [vp] * 7
    L.cns_met_cutsa.argtypes = [vp, C.c_int, vp, c_f64]
    L.cns_set_sa.argtypes = [vp, P(Sa_t)]
    L.cns_met_num.argtypes = [vp]
    L.cns_lpsa.argtypes = [vp, C.c_int] + [vp] * 5
    L.cns_set_ke.argtypes = [vp, C.POINTER(Ke_t)]
    L.cns_met_prod.argtypes = [vp, C.c_int, C.c_int] + [vp] * 4
    L.cns_met_smke.argtypes = [vp, C.c_int] + [vp] * 10
    L.cns_met_kemut.argtypes = [vp, C.c_int] + [vp] * 3
    L.cns_met_cutke.argtypes = [vp, C.c_int, vp, c_f64, c_f64]
    L.cns_met_inisa.argtypes = [vp, C.c_int, vp, vp, vp]
    L.cns_met_inmut.argtypes = [vp, C.c_int, vp, vp]
    L.cns_met_ini.argtypes = [vp, C.c_int] + [vp] * 6
    L.cns_cllparoi1.argtypes = [vp] * 7
    L.cns_set_sweep_tiles.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.cns_set_residual_tiles.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.cns_set_tune_cache.argtypes = [vp, C.c_char_p]
    L.cns_residual_tiles.argtypes = [vp, P(c_i32)]
    L.cns_set_sweep_staging.argtypes = [vp, C.c_int]
    L.cns_sweep_staging.argtypes = [vp, P(c_i32)]
    L.cns_atsch_num_step_host.argtypes = [vp, vp, C.c_int, P(c_f64)]
    L.cns_sch_roe_euler_noalloc.argtypes = [c_i32, c_i32, c_i32, c_i64, c_f64, c_f64, c_i32,
                                            c_f64, vp, vp, vp, vp, vp]
    L.cns_set_subrecord_length.argtypes = [vp, c_i64]
    L.cns_readdg.argtypes = [vp, cs, vp, vp, vp]
    L.cns_writdg.argtypes = [vp, cs, cs, vp, vp, vp]
    L.cns_readda.argtypes = [vp, cs, cs, C.c_int, vp, vp]
    L.cns_writda.argtypes = [vp, cs, cs, cs, vp, vp]
    L.cns_sch_hllc_euler.argtypes = L.cns_sch_roe_euler.argtypes
    L.cns_sch_hllc.argtypes = L.cns_sch_roe.argtypes
    L.cns_sch_rusanov.argtypes = L.cns_sch_roe.argtypes
    L.cns_sch_weno5_3d.argtypes = L.cns_sch_roe.argtypes[:-2] + [vp]
    L.cns_sch_ausmp.argtypes = ([vp, C.c_int, C.c_int, vp, vp, vp, vp] + [vp] * 9 +
                                [cs, vp, i64] + [vp] * 11)
    L.cns_set_cycle.argtypes = [vp, c_i64, c_i64]
    L.cns_sch_duin.argtypes = [vp]
    L.cns_sch_duup.argtypes = [vp]
    L.cns_set_dual_cycle.argtypes = [vp, C.c_int]
    L.cns_sch_dual.argtypes = [vp, C.c_int, vp, vp, C.c_int, vp, vp]
    for f in EXPORTS:
        getattr(L, f).restype = getattr(L, f).restype or C.c_int
    L.cns_last_error.restype = C.c_char_p
    L.cns_scratch_bytes.restype = c_i64
    L.cns_kernels_launched.restype = c_i64
    _lib = L
    return L


class CnsError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str = ""):
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code}) {detail}".strip())
        self.code = code
