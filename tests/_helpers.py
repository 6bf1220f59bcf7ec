"""Shared helpers of the parity tests: run the oracle and the CUDA product on
the same seeded case and compare."""
from __future__ import annotations

import numpy as np

from codens_b200 import cases
from oracle.oracle import Oracle, OracleState, lib as orc_lib

# small seeded cases covering the paths of the configs (sizes are cells)
SMALL = {
    # config-1a form: Euler, unlimited kappa=-1 MUSCL, extr + self-periodic
    "box_eu": lambda: cases.box_case((12, 7, 6), seed=11, skew=0.02, alpha=2.0),
    # config-1c form: NS equations (Re 1e12) with the minmod limiter
    "box_ns": lambda: cases.box_case((10, 8, 5), seed=12, ns=True, ilim=1, skew=0.02,
                                     alpha=-3.0),
    # config-2 form: laminar bump channel, 3 blocks, idd/prd/para/rc
    "channel": lambda: cases.channel_case([9, 6, 7], 8, 5, seed=13, reynz=1.0e3),
    # config-4 form: independent boxes in one layout
    "batch": lambda: cases.batch_case(ncase=4, side=(3, 9), seed=14, qfix_dfez=1),
    # Euler with the flagged non-reference fix of implimf_eu.f90:312
    "box_eu_qfix": lambda: cases.box_case((12, 7, 6), seed=16, skew=0.02, alpha=2.0,
                                          qfix_dfez=1),
    # stiffened gas (pinfl != 0) exercises every pinfl term
    "box_pinfl": lambda: cases.box_case((8, 6, 5), seed=15, ns=True, ilim=1, pinfl=0.3,
                                        reynz=500.0, skew=0.01),
}


def oracle_prepared(case):
    orc = Oracle(case)
    st = OracleState(case)
    orc.metric(st)
    return orc, st


def real(case):
    return case.layout.real_cells()


def cols(a, ncol, ld):
    return a.reshape(ncol, ld)


def max_rel(a, b):
    den = np.maximum(np.abs(a), np.abs(b))
    den[den == 0] = 1.0
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


def max_rel_cols(a, b):
    """largest difference of each component relative to that component's
    largest magnitude (a state comparison insensitive to near-zero entries)"""
    a = np.asarray(a).reshape(a.shape[0], -1)
    b = np.asarray(b).reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1, keepdims=True), 1e-300)
    return float((np.abs(a - b) / scale).max())


def state_err(a, b):
    """largest state difference relative to the reference state's scale:
    density and energy by their largest magnitude, every momentum component
    by the largest momentum magnitude (a flow along x leaves the y and z
    momenta at rounding level, where a per-component scale means nothing)"""
    a = np.asarray(a).reshape(5, -1)
    b = np.asarray(b).reshape(5, -1)
    mom = float(np.sqrt((b[1:4] ** 2).sum(axis=0)).max())
    scale = np.array([np.abs(b[0]).max(), mom, mom, mom, np.abs(b[4]).max()])
    scale = np.maximum(scale, 1e-300)[:, None]
    return float((np.abs(a - b) / scale).max())


def assert_equal_bits(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, what
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if bad.any():
        i = np.flatnonzero(bad)[:5]
        raise AssertionError(f"{what}: {bad.sum()} of {a.size} differ, e.g. at {i}: "
                             f"{a.reshape(-1)[i]} vs {b.reshape(-1)[i]} "
                             f"(max rel {max_rel(a.reshape(-1), b.reshape(-1)):.3e})")
