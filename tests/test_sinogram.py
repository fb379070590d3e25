"""Sinogram pre-processing: Poisson counts (simulateSimplePoissonData.m) and the log
transform with the max(I, 10) clamp (computeSimplePoissonSinogramAttunation.m)."""
import math

import numpy as np
import pytest

from oracle import sino_oracle as so


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of its authors' reference implementation."""
    assert so.philox4x32_10((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert so.philox4x32_10((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF)) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                               0x6D5451FD)
    assert so.philox4x32_10((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


@pytest.mark.parametrize("lam", [0.7, 4.0, 12.0, 250.0, 1e5])
def test_oracle_poisson_moments(lam):
    n = 6000
    k = np.array([so.poisson_ptrs(lam, so._Stream(i, 99))[0] for i in range(n)], dtype=np.float64)
    se = math.sqrt(lam / n)
    assert abs(k.mean() - lam) < 5 * se, (k.mean(), lam)
    assert abs(k.var() / lam - 1.0) < 0.12
    assert (k >= 0).all() and np.array_equal(k, np.floor(k))


def test_oracle_log_transform_clamps_low_counts():
    I = np.array([[[0.0, 5.0, 10.0, 1e4]]], np.float32)
    y = so.log_attenuation(I, 1e5)
    assert y[0, 0, 0] == y[0, 0, 1] == y[0, 0, 2] == np.float32(-np.log(np.float32(10 / np.float32(1e5))))
    assert abs(y[0, 0, 3] - np.log(10.0)) < 1e-6


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


@pytest.mark.gpu
def test_device_counts_match_oracle_stream():
    """The device draws the oracle's draws (same Philox streams, same PTRS steps); a
    last-ulp difference of exp/log between the two math libraries may flip a rare
    borderline acceptance, so at least 99.5% must be identical and the rest close."""
    import torch
    from ctsim_b200.sinogram import simulateSimplePoissonData
    rng = np.random.default_rng(4)
    line = rng.uniform(0.0, 12.0, 3000).astype(np.float32)   # lambda from 1e5 down to ~0.6
    d, fb = simulateSimplePoissonData(torch.from_numpy(line).cuda(), 1e5, seed=1234, return_fallbacks=True)
    got = d.cpu().numpy()
    want = so.simulate_counts(line, 1e5, seed=1234)
    same = np.mean(got == want)
    assert same >= 0.995, same
    assert int(fb.item()) == 0
    lam = 1e5 * np.exp(-line.astype(np.float64))
    assert np.all(np.abs(got - want) <= 6 * np.sqrt(lam) + 2)
    # without counting noise: round(photons * exp(-line))
    d0 = simulateSimplePoissonData(torch.from_numpy(line).cuda(), 1e5, addCountingNoise=False).cpu().numpy()
    assert np.mean(d0 == so.simulate_counts(line, 1e5, add_noise=False)) >= 0.999
    # electronic noise: Box-Muller on its own stream
    dn = simulateSimplePoissonData(torch.from_numpy(line[:500]).cuda(), 1e5, electronicNoise=4.0, seed=1234)
    wn = so.simulate_counts(line[:500], 1e5, electronic_noise=4.0, seed=1234)
    ok = np.abs(dn.cpu().numpy() - wn) <= 1e-3 * np.maximum(1.0, np.abs(wn))
    assert np.mean(ok) >= 0.99


@pytest.mark.gpu
def test_device_counts_deterministic_and_launch_independent():
    import torch
    from ctsim_b200.sinogram import simulateSimplePoissonData
    line = torch.rand(2_000_003, device="cuda") * 8
    a = simulateSimplePoissonData(line, 2e4, seed=7)
    b = simulateSimplePoissonData(line, 2e4, seed=7)
    c = simulateSimplePoissonData(line[:1000].clone(), 2e4, seed=7)
    d = simulateSimplePoissonData(line, 2e4, seed=8)
    assert torch.equal(a, b) and torch.equal(a[:1000], c)
    assert not torch.equal(a, d)


@pytest.mark.gpu
@pytest.mark.parametrize("lam", [2.5, 9.9, 10.0, 64.0, 1e5])
def test_device_poisson_moments(lam):
    import torch
    from ctsim_b200.sinogram import simulateSimplePoissonData
    n = 4_000_000
    line = torch.full((n,), -math.log(lam / 1e5), device="cuda")
    k = simulateSimplePoissonData(line, 1e5, seed=21).double()
    lam32 = float(np.float32(np.float32(1e5) * np.exp(np.float32(-line[0].item()))))
    mean, var = k.mean().item(), k.var().item()
    assert abs(mean - lam32) < 5 * math.sqrt(lam32 / n), (mean, lam32)
    assert abs(var / lam32 - 1) < 0.01, (var, lam32)
    # P(K = 0) = exp(-lambda)
    p0 = (k == 0).double().mean().item()
    assert abs(p0 - math.exp(-lam32)) < 5 * math.sqrt(max(math.exp(-lam32), 1e-9) / n) + 1e-6


@pytest.mark.gpu
def test_device_log_transform_matches_oracle():
    import torch
    from ctsim_b200.sinogram import computeSimplePoissonSinogramAttunation
    rng = np.random.default_rng(2)
    I = rng.uniform(-5.0, 2e5, (6, 16, 8)).astype(np.float32)
    I[0, 0, :4] = [0, 9.99, 10, 10.01]
    flat = rng.uniform(0.5, 1.0, (16, 8)).astype(np.float32)
    for f in (None, flat):
        got = computeSimplePoissonSinogramAttunation(torch.from_numpy(I).cuda(), 1e5,
                                                     None if f is None else torch.from_numpy(f)).cpu().numpy()
        want = so.log_attenuation(I, 1e5, f)
        assert _ulps(got, want).max() <= 2  # logf and numpy's float32 log: each within 1 ulp


@pytest.mark.gpu
def test_device_data_step_feeds_pwls_weights():
    """counts -> y = -log(max(I,10)/I0) and w = counts (computeWeightsPwls(counts, 0, 0))."""
    import torch
    from ctsim_b200.pwls import computeWeightsPwls
    from ctsim_b200.sinogram import computeSimplePoissonSinogramAttunation, simulateSimplePoissonData
    line = torch.rand(4, 32, 8, device="cuda") * 5
    counts = simulateSimplePoissonData(line, 1e5, seed=3)
    y = computeSimplePoissonSinogramAttunation(counts, 1e5)
    w = computeWeightsPwls(counts)
    assert torch.allclose(w, counts.clamp(min=0), rtol=1e-6, atol=0)  # (s - 0)^2 / (s + 0), 0 where s <= 0
    assert (y - line).abs().max().item() < 0.2  # noisy estimate of the line integrals
