"""OS-PWLS (statsrecon/pwls/reconPwlsSeSqs.m) and its penalties on the device,
against the oracle's single-precision numpy restatement."""
import numpy as np
import pytest

from ctsim_b200 import CTGeometry, circular_betas
from oracle import pwls_oracle


def test_oracle_penalty_gradient_is_derivative_of_value():
    """The restated 3-D neighbourhood (5 directions, 1/sqrt(2) diagonals, 1/2 in z):
    the gradient is the derivative of the value (quadratic exactly, Huber away from kinks)."""
    rng = np.random.default_rng(0)
    x = rng.random((5, 6, 7)).astype(np.float32)
    for f, kw in ((pwls_oracle.quad_penalty, {}), (pwls_oracle.huber_penalty, {"delta": 0.05})):
        g = f(x, 1, **kw).astype(np.float64)
        for idx in [(0, 0, 0), (2, 3, 4), (4, 5, 6), (1, 0, 3)]:
            e = np.zeros_like(x, dtype=np.float64)
            e[idx] = 1e-3
            num = (f((x + e).astype(np.float32), 0, **kw) - f((x - e).astype(np.float32), 0, **kw)) / 2e-3
            assert abs(num - g[idx]) < 2e-3 * max(1.0, abs(g[idx])), (f.__name__, idx, num, g[idx])


def test_oracle_weights():
    s = np.array([0.0, -1.0, 2.0, 5.0], np.float32)
    assert np.array_equal(pwls_oracle.compute_weights_pwls(s), np.array([0, 0, 2, 5], np.float32))
    w = pwls_oracle.compute_weights_pwls(s, 1.0, 3.0)
    assert w[2] == np.float32(1.0 / 5.0) and w[1] == 0


def pwls_case():
    g = CTGeometry((28, 26, 10), (1.0, 1.0, 1.0), (0, 0, 0), (56, 18), (1.6, 1.6), (0, 0), 1000.0, 500.0, 1500.0,
                   circular_betas(24))
    rng = np.random.default_rng(5)
    xt = np.zeros(g.image_shape, np.float32)
    xt[:, 6:20, 5:22] = 0.2
    xt[3:7, 10:14, 9:15] = 0.35
    from oracle.bindings import oracle_cbct
    p = oracle_cbct("proj,tf", g, xt)
    counts = rng.poisson(1e4 * np.exp(-p)).astype(np.float32)
    y = np.log(1e4 / np.maximum(counts, 10)).astype(np.float32)
    w = pwls_oracle.compute_weights_pwls(counts)
    x0 = np.full(g.image_shape, 0.1, np.float32)
    return g, y, w, counts, x0


@pytest.mark.gpu
def test_device_penalties_match_oracle():
    import torch
    from ctsim_b200.pwls import huberPenalty, quadPenalty
    rng = np.random.default_rng(1)
    x = (rng.random((9, 11, 13)) * 0.01).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    for mode in (1, 2):
        got = huberPenalty(xd, mode, 0.003).cpu().numpy()
        want = pwls_oracle.huber_penalty(x, mode, 0.003)
        assert np.max(np.abs(got - want)) <= 1e-6 * max(1.0, np.max(np.abs(want)))
        got = quadPenalty(xd, mode).cpu().numpy()
        want = pwls_oracle.quad_penalty(x, mode)
        assert np.max(np.abs(got - want)) <= 1e-6 * max(1.0, np.max(np.abs(want)))
    v = float(huberPenalty(xd, 0, 0.003).item())  # delta is single precision on the device
    assert abs(v - pwls_oracle.huber_penalty(x, 0, 0.003)) <= 1e-6 * abs(v)
    v = float(quadPenalty(xd, 0).item())
    assert abs(v - pwls_oracle.quad_penalty(x, 0)) <= 1e-9 * abs(v)


@pytest.mark.gpu
@pytest.mark.parametrize("pfun", ["huber", "quad"])
def test_device_os_sqs_matches_oracle(pfun):
    import torch
    from ctsim_b200.pwls import computeWeightsPwls, reconPwlsSeSqs
    g, y, w, counts, x0 = pwls_case()
    wd = computeWeightsPwls(torch.from_numpy(counts).cuda())
    assert np.array_equal(wd.cpu().numpy(), w)
    beta, delta, M, its = 2.0, 0.01, 3, 3
    x, phis, rmsds = reconPwlsSeSqs(torch.from_numpy(y).cuda(), wd, g, beta, pfun, its, delta, M,
                                    torch.from_numpy(x0).cuda())
    xo, phio, rmsdo = pwls_oracle.recon_pwls_se_sqs(y, w, g, beta, pfun, its, delta, M, x0)
    got = x.cpu().numpy()
    err = np.linalg.norm(got - xo) / np.linalg.norm(xo)
    assert err <= 1e-4, err
    assert np.allclose(phis, phio, rtol=1e-4)
    assert np.allclose(rmsds, rmsdo, rtol=1e-3)
    assert phis[-1] < phis[0]  # the cost decreases


def test_oracle_nesterov_first_step_is_the_sqs_step():
    """With t = 1 the first Nesterov step from z = x is the plain SQS step, so one
    iteration with one subset gives the reconPwlsSeSqs image exactly."""
    g, y, w, counts, x0 = pwls_case()
    xs, ps, _ = pwls_oracle.recon_pwls_se_sqs(y, w, g, 2.0, "huber", 1, 0.01, 1, x0)
    xn, pn, _ = pwls_oracle.recon_pwls_nesterov_sqs(y, w, g, 2.0, "huber", 1, 0.01, 1, x0)
    assert np.array_equal(xs, xn) and np.allclose(ps, pn, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("pfun", ["huber", "quad"])
def test_device_nesterov_sqs_matches_oracle(pfun):
    import torch
    from ctsim_b200.pwls import reconPwlsSeNesterovSqs
    g, y, w, counts, x0 = pwls_case()
    beta, delta, M, its = 2.0, 0.01, 3, 4
    x, phis, rmsds = reconPwlsSeNesterovSqs(torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), g, beta, pfun,
                                            its, delta, M, torch.from_numpy(x0).cuda())
    xo, phio, rmsdo = pwls_oracle.recon_pwls_nesterov_sqs(y, w, g, beta, pfun, its, delta, M, x0)
    got = x.cpu().numpy()
    err = np.linalg.norm(got - xo) / np.linalg.norm(xo)
    assert err <= 1e-4, err
    assert np.allclose(phis, phio, rtol=1e-4)
    assert np.allclose(rmsds, rmsdo, rtol=1e-3)


@pytest.mark.gpu
def test_device_nesterov_rmsd_against_converged_image():
    """imgOpt switches the rmsd to the middle slice's distance from the converged image."""
    import torch
    from ctsim_b200.pwls import reconPwlsSeNesterovSqs
    g, y, w, counts, x0 = pwls_case()
    x_opt, _, _ = pwls_oracle.recon_pwls_se_sqs(y, w, g, 2.0, "huber", 8, 0.01, 3, x0)
    x, phis, rmsds = reconPwlsSeNesterovSqs(torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), g, 2.0, "huber",
                                            4, 0.01, 3, torch.from_numpy(x0).cuda(), torch.from_numpy(x_opt).cuda())
    xo, _, rmsdo = pwls_oracle.recon_pwls_nesterov_sqs(y, w, g, 2.0, "huber", 4, 0.01, 3, x0, img_opt=x_opt)
    assert np.allclose(rmsds, rmsdo, rtol=1e-3)
    assert rmsds[-1] < rmsds[0]  # approaching the converged image


def config1_pwls_case(views=60):
    """Config-1 shapes (128^2 x 64 at 1 mm, flat 256 x 96 detector at 1.6 mm, SAD 1000, SDD
    1500) with ``views`` views over the turn: the seeded 12-ellipsoid phantom, Poisson counts
    at I0 = 1e5 (counts clamped at 10 in the log) and w = counts; a uniform start image."""
    from ctsim_b200.phantom import config1, to_projector_units
    from oracle.bindings import oracle_cbct
    g, x_mm = config1(n_views=views, seed=1)
    p = oracle_cbct("proj,tf", g, to_projector_units(x_mm))
    rng = np.random.default_rng(21)
    counts = rng.poisson(1e5 * np.exp(-p.astype(np.float64))).astype(np.float32)
    y = np.log(1e5 / np.maximum(counts, 10)).astype(np.float32)
    w = pwls_oracle.compute_weights_pwls(counts)
    x0 = np.full(g.image_shape, 0.15, np.float32)
    return g, y, w, x0


# relative L2 of the image after each outer iteration, device against the restatement: the
# FP32 projectors of the two sides differ in summation order (about 1e-6 per projection),
# and each SQS step divides two such sums
PER_ITERATION_REL_L2 = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("pfun", ["huber", "quad"])
@pytest.mark.parametrize("nesterov", [False, True], ids=["sqs", "nesterov"])
def test_config1_os_pwls_each_iteration_matches_oracle(pfun, nesterov):
    """reconPwlsSeSqs / reconPwlsSeNesterovSqs at config-1 shapes, 60 views, 4 ordered
    subsets, 2 outer iterations (statsrecon/pwls/reconPwlsSeSqs.m:51-78,
    reconPwlsSeNesterovSqs.m:60-113): the image after every iteration, phi and rmsd."""
    import torch
    from ctsim_b200.pwls import PwlsNesterovSolver, PwlsSolver
    g, y, w, x0 = config1_pwls_case()
    beta, delta, M, its = 1e3, 0.01, 4, 2
    cls = PwlsNesterovSolver if nesterov else PwlsSolver
    s = cls(torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), g, beta, pfun, delta, M,
            torch.from_numpy(x0).cuda())
    got, phis, rmsds = [], [], []
    for _ in range(its):
        phi, rmsd = s.step()
        got.append(s.x.cpu().numpy())
        phis.append(phi)
        rmsds.append(rmsd)
    hist = []
    run = pwls_oracle.recon_pwls_nesterov_sqs if nesterov else pwls_oracle.recon_pwls_se_sqs
    _, phio, rmsdo = run(y, w, g, beta, pfun, its, delta, M, x0, history=hist)
    errs = [float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b)) for a, b in zip(got, hist)]
    assert max(errs) <= PER_ITERATION_REL_L2, errs
    assert np.allclose(phis, phio, rtol=1e-5), (phis, phio)
    assert np.allclose(rmsds, rmsdo, rtol=1e-3), (rmsds, rmsdo)
