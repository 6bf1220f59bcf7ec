"""The 2.5D Jacobi sweep tiling: every patch shape and plane count gives the
same FP64 iteration bit for bit (each cell's arithmetic does not depend on
the tiling), the autotuner runs on the first fused iteration, and the
reduced-precision forms are tiling-independent bit for bit too, with the
planes staged as tensor boxes (the default) or by cp.async element copies."""
from __future__ import annotations

import numpy as np
import pytest

from ._helpers import SMALL, assert_equal_bits, real

pytestmark = pytest.mark.gpu

SHAPES = [(32, 4), (32, 8), (16, 8), (16, 16)]


def _run(name, precision, tiles, nsteps=3, staging=0):
    from codens_b200.solver import CodeNS
    case = SMALL[name]()
    case.scheme.precision = precision
    s = CodeNS(case)
    s.metric()
    if staging:
        s.set_sweep_staging(staging)
        assert s.sweep_staging == staging
    if tiles is not None:
        s.set_sweep_tiles(0 if precision == 0 else 1, *tiles)
    s.atsch_num(nsteps)
    v = s.v.cpu().numpy().reshape(5, case.layout.ld)[:, real(case)]
    cfg = s.sweep_tiles(0 if precision == 0 else 1)
    s.close()
    return v, cfg


@pytest.mark.parametrize("name", ["box_ns", "channel"])
def test_fp64_iteration_independent_of_tiling(cuda, name):
    ref, cfg = _run(name, 0, None)
    assert cfg[3] == 1, "the first fused iteration tunes the sweep tiling"
    for ti, tj in SHAPES:
        for kc in (1, 3, 8):
            v, cfg = _run(name, 0, (ti, tj, kc))
            assert cfg[:3] == (ti, tj, kc)
            assert_equal_bits(v, ref, f"tiles {ti}x{tj}x{kc}")


@pytest.mark.parametrize("name,precision", [("channel", 1), ("box_ns", 1), ("box_eu_qfix", 1),
                                            ("channel", 2)])
def test_reduced_precision_iteration_independent_of_tiling(cuda, name, precision):
    """the FP32 sweeps evaluate every increment with explicit roundings, so
    the mixed and defect iterations give the same bits under every patch
    shape and plane count (the autotuner's pick cannot change a result)"""
    ref, cfg = _run(name, precision, None)
    assert cfg[3] == 1
    for ti, tj in SHAPES:
        for kc in (1, 2, 3, 8):
            v, _ = _run(name, precision, (ti, tj, kc))
            assert_equal_bits(v, ref, f"precision {precision} tiles {ti}x{tj}x{kc}")
        for kc in (2, 3):
            v, _ = _run(name, precision, (ti, tj, kc), staging=1)
            assert_equal_bits(v, ref, f"cp.async staging, tiles {ti}x{tj}x{kc}")


def test_rejects_unknown_shape(cuda):
    from codens_b200 import abi
    from codens_b200.solver import CodeNS
    s = CodeNS(SMALL["box_ns"]())
    with pytest.raises(abi.CnsError) as ei:
        s.set_sweep_tiles(0, 8, 8, 4)
    assert ei.value.code == abi.CNS_EINVAL
    with pytest.raises(abi.CnsError):
        s.set_sweep_tiles(0, 32, 8, 0)
    s.close()


@pytest.mark.parametrize("name", ["box_ns", "channel", "box_eu_qfix", "box_pinfl"])
def test_fused_residual_variant_gives_the_same_bits(cuda, name):
    """the fused residual kernel (three face directions and the accumulation
    in one 2.5D launch) against the face kernels + accumulation: the same
    FP64 iteration bit for bit, for both patch shapes and several plane
    counts"""
    from codens_b200.solver import CodeNS
    ref, _ = _run(name, 0, (32, 8, 8))
    for ti, tj in ((32, 4), (16, 8)):
        for kc in (1, 3, 16):
            case = SMALL[name]()
            s = CodeNS(case)
            s.metric()
            s.set_residual_tiles(ti, tj, kc)
            assert s.residual_tiles() == (ti, tj, kc)
            s.set_sweep_tiles(0, 32, 8, 8)
            s.atsch_num(3)
            v = s.v.cpu().numpy().reshape(5, case.layout.ld)[:, real(case)]
            s.close()
            assert_equal_bits(v, ref, f"fused residual {ti}x{tj}x{kc}")


def test_tuning_cache(cuda, tmp_path):
    """the first context times the sweep tilings and appends its pick to the
    cache file; a second context of the same configuration reads it (no
    timing) and runs the same tiling; an entry this build has no kernel for
    is ignored"""
    from codens_b200.solver import CodeNS
    path = tmp_path / "tune.txt"
    picks = []
    for run in range(2):
        case = SMALL["channel"]()
        case.scheme.precision = 1
        s = CodeNS(case)
        s.metric()
        s.set_tune_cache(path)
        s.atsch_num(2)
        cfg32 = s.sweep_tiles(1)
        assert cfg32[3] == (1 if run == 0 else 2), (run, cfg32)
        picks.append(cfg32[:3])
        s.close()
    assert picks[0] == picks[1]
    lines = path.read_text().split()
    assert len(lines) == 4 and lines[0].count("|") == 6 and "f32" in lines[0]
    # an unusable entry (shape without a kernel) for the same key: timed again
    path.write_text(f"{lines[0]} 8 8 4\n")
    case = SMALL["channel"]()
    case.scheme.precision = 1
    s = CodeNS(case)
    s.metric()
    s.set_tune_cache(path)
    s.atsch_num(1)
    assert s.sweep_tiles(1)[3] == 1
    s.close()


def test_staging_mode_is_checked(cuda):
    from codens_b200 import abi
    from codens_b200.solver import CodeNS
    s = CodeNS(SMALL["box_ns"]())
    assert s.sweep_staging == 0
    with pytest.raises(abi.CnsError) as e:
        s.set_sweep_staging(2)
    assert e.value.code == abi.CNS_EINVAL
    s.close()
