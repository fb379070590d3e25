"""Precision variants (config 3): volumes and sinograms stored in BF16 / FP16, every
footprint sum accumulated in FP32, the PWLS residual formed in FP32 -- errors against
the FP64 oracle (the restated reference C compiled in double).  Run with -s to see
the per-variant and per-iteration report."""
import numpy as np
import pytest

from ctsim_b200.phantom import config1, to_projector_units
from oracle import pwls_oracle
from oracle.bindings import oracle_cbct

pytestmark = pytest.mark.gpu

BOUNDS = {"float32": 1e-5, "float16": 2e-3, "bfloat16": 1.5e-2}


def _err(got, ref):
    got = np.asarray(got, np.float64)
    return np.linalg.norm(got - ref) / np.linalg.norm(ref), float(np.max(np.abs(got - ref)))


def test_projector_storage_precision():
    import torch
    from ctsim_b200.projector import Plan
    g, x_mm = config1(n_views=60)
    x = to_projector_units(x_mm)
    rng = np.random.default_rng(7)
    y = (oracle_cbct("proj,dd", g, x) + rng.normal(0, 0.01, g.sino_shape)).astype(np.float32)
    ax64 = oracle_cbct("proj,dd", g, x.astype(np.float64), fp64=True)
    aty64 = oracle_cbct("back,dd", g, y.astype(np.float64), fp64=True)
    plan = Plan(g)
    print("\nstorage   | A x rel L2 | A x max abs | A^T y rel L2 | A^T y max abs   (vs FP64 oracle)")
    for name, dt in (("float32", torch.float32), ("bfloat16", torch.bfloat16), ("float16", torch.float16)):
        ax = plan.project(torch.from_numpy(x).cuda().to(dt), "dd").float().cpu().numpy()
        aty = plan.backproject(torch.from_numpy(y).cuda().to(dt), "dd").float().cpu().numpy()
        e1, m1 = _err(ax, ax64)
        e2, m2 = _err(aty, aty64)
        print(f"{name:9s} | {e1:.3e}  | {m1:.3e}   | {e2:.3e}    | {m2:.3e}")
        assert e1 <= BOUNDS[name] and e2 <= BOUNDS[name], (name, e1, e2)


def test_pwls_storage_precision():
    """OS-SQS with the measured data stored in BF16/FP16 (image and residual FP32):
    per-iteration image error against the FP64 oracle reconstruction, and the final
    image within 1% of it."""
    import torch
    from ctsim_b200.pwls import reconPwlsSeSqs
    g, x_mm = config1(n_views=48)
    x = to_projector_units(x_mm)
    rng = np.random.default_rng(11)
    p = oracle_cbct("proj,tf", g, x)
    counts = rng.poisson(1e5 * np.exp(-p)).astype(np.float32)
    y = np.log(1e5 / np.maximum(counts, 10)).astype(np.float32)
    w = pwls_oracle.compute_weights_pwls(counts)
    x0 = np.full(g.image_shape, 0.2, np.float32)
    beta, delta, M, its = 1e3, 0.01, 4, 3
    hist = []
    x64, _, _ = pwls_oracle.recon_pwls_se_sqs(y, w, g, beta, "huber", its, delta, M, x0, fp64=True, history=hist)
    print("\nstorage   | per-iteration image rel RMSE vs FP64 oracle")
    for name, dt in (("float32", torch.float32), ("bfloat16", torch.bfloat16), ("float16", torch.float16)):
        errs = []
        for k in range(1, its + 1):
            xk, _, _ = reconPwlsSeSqs(torch.from_numpy(y).cuda(), torch.from_numpy(w).cuda(), g, beta, "huber", k,
                                      delta, M, torch.from_numpy(x0).cuda(), storage=dt)
            errs.append(_err(xk.cpu().numpy(), hist[k - 1])[0])
        print(f"{name:9s} | " + "  ".join(f"{e:.3e}" for e in errs))
        assert errs[-1] <= 0.01, (name, errs)
        if name == "float32":
            assert errs[-1] <= 1e-4


def test_fdk_storage_precision():
    """reconFDK from a sinogram stored in FP32 / BF16 / FP16 (FP32 filter arithmetic; the
    filtered sinogram kept in the input's storage type and backprojected as it is)
    against FDK in FP64 (the filter in float64 and the double restatement of back,hpd)."""
    import torch
    from ctsim_b200.fdk import FDK
    from oracle import fdk_oracle
    g, x_mm = config1(n_views=120)
    x = to_projector_units(x_mm)
    rng = np.random.default_rng(13)
    p = oracle_cbct("proj,dd", g, x)
    counts = rng.poisson(1e5 * np.exp(-p)).astype(np.float32)
    y = np.log(1e5 / np.maximum(counts, 10)).astype(np.float32)
    filt = fdk_oracle.filtered_sinogram(y, g, "hann")
    betas = np.asarray(g.betas, np.float64)
    dbeta = abs(betas[-1] - betas[0]) / (betas.size - 1) / 2
    img64 = oracle_cbct("back,hpd", g, filt, fp64=True) * dbeta * 10
    f = FDK(g, "hann")
    print("\nstorage   | FDK image rel L2 | max abs   (vs FDK in FP64)")
    for name, dt in (("float32", torch.float32), ("bfloat16", torch.bfloat16), ("float16", torch.float16)):
        img = f(torch.from_numpy(y).cuda().to(dt)).cpu().numpy()
        e, m = _err(img, img64)
        print(f"{name:9s} | {e:.3e}        | {m:.3e}")
        assert e <= BOUNDS[name], (name, e)
