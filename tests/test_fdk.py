"""FDK (fbp/reconFDK.m) on the device against the oracle restatement.

CPU: the library's filter design (designFilter2.m / designEquiangularFilter2.m)
matches the oracle's for every window.  GPU: the weighted, filtered sinogram
and the full reconstruction match the oracle to 1e-5 relative L2 (FP32 FFT
against a float64 restatement; the backprojection itself is bit-identical)."""
import numpy as np
import pytest

from ctsim_b200 import CTGeometry, circular_betas
from ctsim_b200.fdk import WINDOWS, design_filter
from oracle import fdk_oracle

REL_L2 = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("flat", [1, 0])
@pytest.mark.parametrize("window", WINDOWS)
def test_filter_design_matches_oracle(window, flat):
    # spacings exact in float32: the C ABI takes du as single (MATLAB designs with the double)
    for nu, du, crop in ((256, 1.5, 1.0), (1024, 0.75, 1.0), (37, 0.5, 0.75)):
        got = design_filter(nu, du, 1500.0, bool(flat), window, crop)
        if flat:
            want = fdk_oracle.design_filter2(du, window, nu, crop)
        else:
            want = fdk_oracle.design_equiangular(du, 1500.0, window, nu, crop)
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) <= 1e-9 * np.max(np.abs(want))


def test_unknown_window_is_rejected():
    from ctsim_b200._lib import CtsimError
    with pytest.raises(CtsimError, match="Invalid window"):
        design_filter(64, 1.0, 1500.0, True, "gauss")


def fdk_cases():
    full = CTGeometry((48, 44, 20), (1.0, 1.0, 1.0), (0, 0, 0), (96, 32), (1.6, 1.6), (0, 0), 1000.0, 500.0,
                      1500.0, circular_betas(60))
    curved = CTGeometry((40, 40, 16), (1.0, 1.0, 1.0), (0.5, 0, 0), (80, 28), (1.6, 1.6), (1.5, -0.5), 1000.0,
                        500.0, 1500.0, circular_betas(50), flatPanel=0)
    ss = np.linspace(-0.5 * (np.pi + 0.6), 0.5 * (np.pi + 0.6), 64)  # pi + fan, centred (loadProjectionGeometryShortScan.m:47)
    short = CTGeometry((40, 40, 12), (1.0, 1.0, 1.0), (0, 0, 0), (96, 24), (1.6, 1.6), (0, 0), 1000.0, 500.0,
                       1500.0, ss, shortScan=True)
    return {"flat_full_hann": (full, "hann"), "curved_full_hamming": (curved, "hamming"),
            "flat_short_hamming": (short, "hamming")}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(fdk_cases()))
def test_fdk_matches_oracle(name):
    import torch
    from ctsim_b200.fdk import FDK
    g, window = fdk_cases()[name]
    rng = np.random.default_rng(3)
    y = rng.random(g.sino_shape, dtype=np.float32)
    f = FDK(g, window)
    yd = torch.from_numpy(y).cuda()
    filt = f.filter(yd).cpu().numpy()
    assert rel_l2(filt, fdk_oracle.filtered_sinogram(y, g, window)) <= REL_L2
    img = f(yd).cpu().numpy()
    want = fdk_oracle.recon_fdk(y, g, window)
    assert rel_l2(img, want) <= REL_L2, rel_l2(img, want)


@pytest.mark.gpu
def test_fdk_reconstructs_a_projected_phantom():
    """End to end on config-1 shapes: A x with the device projector, then reconFDK;
    the central slices recover the phantom (cone-beam FDK error only)."""
    import torch
    from ctsim_b200.fdk import reconFDK
    from ctsim_b200.phantom import config1, to_projector_units
    from ctsim_b200.projector import Plan
    g, x_mm = config1(n_views=180)
    x = to_projector_units(x_mm)
    p = Plan(g)
    y = p.project(torch.from_numpy(x).cuda(), "dd")
    img = reconFDK(y, g, "hann").cpu().numpy()
    mid = slice(g.nz // 2 - 4, g.nz // 2 + 4)
    err = np.sqrt(np.mean((img[mid] - x[mid]) ** 2)) / np.sqrt(np.mean(x[mid] ** 2))
    assert err < 0.15, err
