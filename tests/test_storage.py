"""Sinograms stored in BF16/FP16 are read as they are: no FP32 sinogram-sized scratch.

The A^T (DD, SF) reads 16-bit sinograms with the axial amplitude applied in its rows
pass, FDK and back,var read them in the bilinear sample, and the PWLS residual is written
already multiplied by the amplitudes (CTSIM_INPUT_SCALED).  Widening BF16/FP16 to FP32 is
exact and the product with the amplitude is the same FP32 operation as in the scratch
copy, so each result equals the backprojection of an FP32 copy bit for bit, while the
plan's device memory does not grow.  Only an A^T of an unscaled FP32 sinogram allocates
the plan's scratch, once, at its first call.
"""
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _config2_views(n):
    """The benchmark geometry (512^2 x 256 at 0.5 mm, flat 1024 x 384 at 0.8 mm) with n of
    its 720 views, evenly spaced."""
    from ctsim_b200.phantom import config2
    g, _ = config2(seed=2)
    k = g.noViews // n
    return replace(g, betas=g.betas[::k][:n].copy(), couchZ=g.couchZ[::k][:n].copy())


def test_low_precision_and_scaled_backprojections_allocate_no_scratch():
    import torch
    from ctsim_b200.projector import Plan
    g = _config2_views(90)
    plan = Plan(g)
    base = plan.device_bytes
    gen = torch.Generator(device="cuda").manual_seed(3)
    y32 = torch.rand(g.sino_shape, device="cuda", generator=gen)
    got = {}
    for dt in (torch.bfloat16, torch.float16):
        for m in ("dd", "tf", "hpd", "var"):
            got[dt, m] = plan.backproject(y32.to(dt), m, out_dtype=torch.float32)
    torch.cuda.synchronize()
    plan.check()
    assert plan.device_bytes == base
    # the same values through FP32 copies (these A^T calls allocate the scratch)
    for (dt, m), a in got.items():
        assert torch.equal(a, plan.backproject(y32.to(dt).float(), m)), (dt, m)
    # the scratch is 4 bytes per sinogram pixel, allocated once
    p2 = Plan(g)
    b2 = p2.device_bytes
    p2.backproject(y32, "dd", scaled=True)  # a pre-scaled FP32 input: read as it is
    torch.cuda.synchronize()
    assert p2.device_bytes == b2
    p2.backproject(y32, "dd")
    p2.backproject(y32, "tf")
    torch.cuda.synchronize()
    assert p2.device_bytes == b2 + 4 * g.nu * g.nv * g.noViews


def test_scaled_input_equals_the_scratch_path():
    """A^T of (w d) * ampv written by the scaled residual, with CTSIM_INPUT_SCALED, equals
    A^T of the plain residual w d bit for bit (the same products in the same order)."""
    import ctypes as C
    import torch
    from ctsim_b200 import _lib
    from ctsim_b200.projector import Plan
    from cases import make_cases
    g = make_cases()["offsets_curved"]
    plan = Plan(g)
    L = _lib.load()
    gen = torch.Generator(device="cuda").manual_seed(5)
    ax = torch.rand(g.sino_shape, device="cuda", generator=gen)
    y = torch.rand(g.sino_shape, device="cuda", generator=gen)
    w = torch.rand(g.sino_shape, device="cuda", generator=gen) * 1e4
    st = torch.cuda.current_stream().cuda_stream
    wd = torch.empty_like(ax)
    wds = torch.empty_like(ax)
    phi = torch.zeros(2, dtype=torch.float64, device="cuda")
    _lib.check(L.ctsim_pwls_residual_ex(ax.data_ptr(), y.data_ptr(), w.data_ptr(), 0, 1.0, wd.data_ptr(), ax.numel(),
                                        phi.data_ptr(), st), "residual")
    _lib.check(L.ctsim_pwls_residual_scaled(plan._h, ax.data_ptr(), y.data_ptr(), w.data_ptr(), 0, 1.0,
                                            wds.data_ptr(), g.noViews, phi.data_ptr() + 8, st), "scaled residual")
    p = phi.cpu().numpy()
    assert p[0] == p[1] or abs(p[0] - p[1]) <= 1e-12 * abs(p[0])  # the same data term
    for m in ("dd", "tf"):
        assert torch.equal(plan.backproject(wd, m, scale=3.0), plan.backproject(wds, m, scale=3.0, scaled=True))
