"""The discrete adjoint of the steady Euler Roe solution (bump channel,
first-order reconstruction): gradients of the wall pressure force with
respect to the inflow Mach number, the inflow angle and lower-wall node
heights against central finite differences of the converged primal, and the
transposed residual product against a finite-difference directional
derivative of the library's residual."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# gradients: finite differences with step 1e-6 of primal solves converged to
# L2 < 1e-14 agree with the adjoint to ~1e-9 relative; the bound leaves room
# for the finite-difference truncation on small components
GRAD_TOL = 1e-6


def _design():
    from codens_b200 import adjoint
    return adjoint.Design(ni=16, nj=8, nk=2, mach=0.5, alpha=1.0, bump=0.1)


def test_transposed_residual_product(cuda):
    """<A^T lam, dW> = <lam, (u(W + e dW) - u(W - e dW)) / 2e> on random
    vectors, u the library's residual with its boundary conditions"""
    torch = cuda
    from codens_b200 import adjoint
    d = _design()
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-10, adj_max=0)
    s, M = g.s, g.maps
    ld = M.ld
    gen = torch.Generator(device="cuda").manual_seed(3)
    lam = torch.zeros(5, ld, dtype=torch.float64, device="cuda")
    dW = torch.zeros(5, ld, dtype=torch.float64, device="cuda")
    lam[:, M.real] = torch.rand(5, len(M.real), generator=gen, device="cuda",
                                dtype=torch.float64) - 0.5
    dW[:, M.real] = (torch.rand(5, len(M.real), generator=gen, device="cuda",
                                dtype=torch.float64) - 0.5) * g.W[:, M.real].abs()
    wbar = torch.zeros(6 * ld, dtype=torch.float64, device="cuda")
    s.adjoint_rt(lam.reshape(-1), wbar)
    s.sync()
    lhs = float((g._chain(wbar) * dW).sum())

    def residual(W):
        s.v.copy_(W.reshape(-1))
        s.zpres(0, s.v, s.pression, s.ztemp, s.cson)
        s.rbord(s.v, s.pression, s.ztemp, s.cson)
        s.sch_roe_euler(0, s.u, s.v, s.sn, s.pression)
        s.sync()
        return s.u.reshape(5, ld).clone()

    eps = 1e-6
    up = residual(g.W + eps * dW)
    um = residual(g.W - eps * dW)
    rhs = float((lam * (up - um)).sum()) / (2 * eps)
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs), (lhs, rhs)
    g.close()


def test_wall_force_gradient_matches_finite_differences(cuda):
    from codens_b200 import adjoint
    d = _design()
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-14, adj_tol=1e-12)
    J, gm, ga, gw = g.gradient()
    gw = gw.cpu().numpy()
    g.close()

    def Jat(mach=d.mach, alpha=d.alpha, wall=None):
        return adjoint.wall_force(d, mach, alpha, d.wall() if wall is None else wall,
                                  tol=1e-14)

    eps = 1e-6
    fd_m = (Jat(mach=d.mach + eps) - Jat(mach=d.mach - eps)) / (2 * eps)
    assert abs(gm - fd_m) <= GRAD_TOL * abs(fd_m), (gm, fd_m)
    fd_a = (Jat(alpha=d.alpha + eps) - Jat(alpha=d.alpha - eps)) / (2 * eps)
    assert abs(ga - fd_a) <= 1e-3 * abs(fd_a) + 1e-9, (ga, fd_a)
    w0 = d.wall()
    for i in (7, 8, 9):
        wp, wm = w0.copy(), w0.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (Jat(wall=wp) - Jat(wall=wm)) / (2 * eps)
        assert abs(gw[i] - fd) <= GRAD_TOL * max(abs(fd), 1e-3), (i, gw[i], fd)


def test_autograd_function(cuda):
    torch = cuda
    from codens_b200 import adjoint
    d = _design()
    WallForce = adjoint.make_function()
    mach = torch.tensor(d.mach, dtype=torch.float64, requires_grad=True)
    alpha = torch.tensor(d.alpha, dtype=torch.float64, requires_grad=True)
    wall = torch.tensor(d.wall(), dtype=torch.float64, requires_grad=True)
    J = WallForce.apply(mach, alpha, wall, d)
    J.backward()
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-13, adj_tol=1e-12)
    J2, gm, ga, gw = g.gradient()
    g.close()
    assert abs(float(J) - J2) <= 1e-12 * abs(J2)
    assert abs(float(mach.grad) - gm) <= 1e-8 * abs(gm)
    np.testing.assert_allclose(wall.grad.numpy(), gw.cpu().numpy(), rtol=1e-8, atol=1e-12)


def test_mixed_form_gradient_matches_fp64(cuda):
    """the mixed form (FP32 primal sweeps, FP32 transposed sweeps; FP64
    residual and A^T lambda) converges to the same steady state and adjoint,
    so its gradient equals the FP64 one to the convergence tolerances"""
    from codens_b200 import adjoint
    import dataclasses
    d = _design()
    dm = dataclasses.replace(d, precision=1)
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-14, adj_tol=1e-12)
    J, gm, ga, gw = g.gradient()
    g.close()
    h = adjoint.WallForceGradient(dm, dm.mach, dm.alpha, dm.wall(), tol=1e-14, adj_tol=1e-12)
    J2, gm2, ga2, gw2 = h.gradient()
    h.close()
    assert abs(J2 - J) <= 1e-12 * abs(J)
    assert abs(gm2 - gm) <= 1e-8 * abs(gm), (gm2, gm)
    assert abs(ga2 - ga) <= 1e-8 * abs(ga) + 1e-12, (ga2, ga)
    np.testing.assert_allclose(gw2.cpu().numpy(), gw.cpu().numpy(), rtol=1e-7,
                               atol=1e-9 * float(gw.abs().max()))


def _oracle_state(d, mach, tol=1e-14, cap=200000):
    """the converged primal of the CPU restatement of the reference"""
    from oracle.oracle import Oracle, OracleState
    case = d.case(mach, d.alpha, d.wall())
    orc = Oracle(case)
    st = OracleState(case)
    orc.metric(st)
    for it in range(cap):
        v0 = st.v.copy()
        orc.step(st)
        if it % 50 == 49 and orc.norms(v0, st)[1, 0] < tol:
            break
    return st.v.copy()


def test_gradient_matches_finite_differences_of_the_oracle(cuda):
    """dJ/dMach of the adjoint against central differences of J evaluated on
    primal states converged by the CPU restatement of the reference"""
    from codens_b200 import adjoint
    d = _design()
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-14, adj_tol=1e-12)
    J, gm, _, _ = g.gradient()
    g.close()
    eps = 1e-6
    Jp = adjoint.wall_force(d, d.mach + eps, d.alpha, d.wall(),
                            state=_oracle_state(d, d.mach + eps))
    Jm = adjoint.wall_force(d, d.mach - eps, d.alpha, d.wall(),
                            state=_oracle_state(d, d.mach - eps))
    fd = (Jp - Jm) / (2 * eps)
    assert abs(gm - fd) <= GRAD_TOL * abs(fd), (gm, fd)


def test_checkpointed_reverse_accumulation_independent_of_interval(cuda):
    """pseudo-time checkpointing: the reverse sweep over 12 iterations from
    the initial state gives the same adjoint states bit for bit whether every
    state, every fifth or only the first is kept (the recomputed states are
    the forward run's), with at most N/every + every states held"""
    from codens_b200 import adjoint
    d = _design()
    out = []
    for every in (1, 5, 12):
        g = adjoint.CheckpointedGradient(d, d.mach, d.alpha, d.wall(), n_iter=12, every=every)
        J, gm, ga, gw = g.gradient()
        out.append((J, gm, ga, gw.cpu().numpy(), g.mu_sum.cpu().numpy()))
        assert g.max_states <= (12 + every - 1) // every + every, (every, g.max_states)
        g.close()
    for J, gm, ga, gw, mu in out[1:]:
        # the state part of the reverse sweep (library kernels and the
        # boundary chain) is the same bits; the parameter parts go through
        # torch autograd, whose scatter-adds into the wall nodes sum in a
        # varying order, so they agree to rounding
        assert J == out[0][0]
        assert np.array_equal(mu, out[0][4])
        assert abs(gm - out[0][1]) <= 1e-13 * abs(out[0][1])
        assert abs(ga - out[0][2]) <= 1e-12 * max(abs(out[0][2]), 1e-3 * abs(out[0][1]))
        assert np.abs(gw - out[0][3]).max() <= 1e-13 * np.abs(out[0][3]).max()
    assert np.isfinite(out[0][1]) and np.isfinite(out[0][3]).all()


def test_checkpointed_gradient_equals_the_steady_adjoint_truncation(cuda):
    """over a converged history, N reverse steps sum the series the steady
    adjoint iteration sums in N iterations: both gradients agree to rounding
    (the reverse sweep re-linearises at every recomputed state)"""
    import torch
    from codens_b200 import adjoint
    d = _design()
    n = 30
    steady = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-13,
                                       adj_tol=0.0, adj_max=n, check=10 ** 9)
    Js, gms, gas, gws = steady.gradient()
    assert steady.adj_iters == n
    Wstar = steady.s.v.detach().cpu().numpy().copy()
    steady.close()
    g = adjoint.CheckpointedGradient(d, d.mach, d.alpha, d.wall(), n_iter=n, every=10,
                                     start=Wstar)
    Jc, gmc, gac, gwc = g.gradient()
    g.close()
    # the history starts at the converged state and moves at the 1e-13 level
    assert abs(Jc - Js) <= 1e-9 * abs(Js)
    assert abs(gmc - gms) <= 1e-8 * abs(gms), (gmc, gms)
    assert abs(gac - gas) <= 1e-8 * max(abs(gas), 1e-3 * abs(gms)), (gac, gas)
    scale = float(torch.as_tensor(gws).abs().max())
    assert float((gwc - gws).abs().max()) <= 1e-8 * scale


def test_muscl_gradient_matches_finite_differences(cuda):
    """the configuration-5 scheme, kappa = -1 MUSCL (sch_roe_euler.f90:137-174),
    on a channel small enough for its primal to converge (on 128x64x4 and
    larger the MUSCL iteration settles into a limit cycle at CFL 5): the
    adjoint linearises the four-cell stencil of every face"""
    from codens_b200 import adjoint
    d = adjoint.Design(ni=16, nj=8, nk=2, mach=0.5, alpha=1.0, bump=0.1, muscl=1)
    g = adjoint.WallForceGradient(d, d.mach, d.alpha, d.wall(), tol=1e-14, max_iter=80000,
                                  adj_tol=1e-12, adj_max=80000)
    assert g.l2 < 1e-13, g.l2
    J, gm, ga, gw = g.gradient()
    gw = gw.cpu().numpy()
    g.close()

    def Jat(mach=d.mach, alpha=d.alpha, wall=None):
        return adjoint.wall_force(d, mach, alpha, d.wall() if wall is None else wall,
                                  tol=1e-14, max_iter=80000)

    eps = 1e-6
    fd_m = (Jat(mach=d.mach + eps) - Jat(mach=d.mach - eps)) / (2 * eps)
    assert abs(gm - fd_m) <= GRAD_TOL * abs(fd_m), (gm, fd_m)
    w0 = d.wall()
    for i in (7, 9):
        wp, wm = w0.copy(), w0.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (Jat(wall=wp) - Jat(wall=wm)) / (2 * eps)
        assert abs(gw[i] - fd) <= GRAD_TOL * max(abs(fd), 1e-3), (i, gw[i], fd)
