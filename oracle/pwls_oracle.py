"""Oracle for the OS-PWLS path (TEST INFRASTRUCTURE ONLY): numpy restatements of
the reference's MATLAB in single precision, with the projectors of the C oracle.

    compute_weights_pwls   statsrecon/pwls/computeWeightsPwls.m:8-9
    huber_penalty          penalty/huberPenalty.m:101-217 (3-D), :222-238
    quad_penalty           penalty/quadPenalty.m:296-352 (3-D), with dQuad(d) = d
    recon_pwls_se_sqs      statsrecon/pwls/reconPwlsSeSqs.m:36-110
    recon_pwls_nesterov_sqs statsrecon/pwls/reconPwlsSeNesterovSqs.m:35-136

Arrays follow the package layout [nz, ny, nx]; the MATLAB code indexes x(i,j,k)
with i along x, so the slicing below is written on the transposed view.

Parity unpinned: MATLAB (and Octave) cannot run here and the reference holds no golden
output for these functions, so this restatement is checked by reading it against the .m
sources and by property tests (the penalty gradient is the derivative of its value, the
first Nesterov step equals the SQS step), not against MATLAB's own results.
"""
from __future__ import annotations

import numpy as np

from .bindings import oracle_cbct

F32 = np.float32
AXY = F32(1 / np.sqrt(2))
AZ = F32(0.5)


def compute_weights_pwls(sino, r=0.0, v=0.0):
    s = np.asarray(sino, dtype=F32)
    with np.errstate(divide="ignore", invalid="ignore"):  # s = -v divides by zero, as it does in MATLAB
        w = ((s - F32(r)) ** 2 / (s + F32(v))).astype(F32)
    w[s <= F32(r)] = 0
    return w


def _mat(x):
    return np.asarray(x, dtype=F32).transpose(2, 1, 0)  # x(i,j,k)


def _sum_huber(d, delta):
    d = np.abs(d.astype(np.float64))
    t = d ** 2 / 2
    big = d > delta
    t[big] = delta * d[big] - delta ** 2 / 2
    return float(t.sum())


def _dhuber(d, delta):
    d = d.copy()
    d[d > delta] = F32(delta)
    d[d < -delta] = F32(-delta)
    return d


def _chuber(d, delta):
    return (np.abs(d) <= delta).astype(F32)


def _penalty(x, mode, f_sum, f_grad, f_curv):
    X = _mat(x)
    pairs = [((slice(0, -1), slice(None), slice(None)), (slice(1, None), slice(None), slice(None)), F32(1)),
             ((slice(None), slice(0, -1), slice(None)), (slice(None), slice(1, None), slice(None)), F32(1)),
             ((slice(0, -1), slice(0, -1), slice(None)), (slice(1, None), slice(1, None), slice(None)), AXY),
             ((slice(1, None), slice(0, -1), slice(None)), (slice(0, -1), slice(1, None), slice(None)), AXY),
             ((slice(None), slice(None), slice(0, -1)), (slice(None), slice(None), slice(1, None)), AZ)]
    if mode == 0:
        return sum(float(c) * f_sum(X[p] - X[q]) for p, q, c in pairs)
    y = np.zeros(X.shape, dtype=F32)
    for n, (p, q, c) in enumerate(pairs):
        d = X[p] - X[q]
        g = f_grad(d) if mode == 1 else f_curv(d)
        if n >= 2:
            g = (c * g).astype(F32)
        y[p] = y[p] + g
        y[q] = (y[q] - g) if mode == 1 else (y[q] + g)
    return y.transpose(2, 1, 0).copy()


def huber_penalty(x, mode, delta=0.001):
    return _penalty(x, mode, lambda d: _sum_huber(d, delta), lambda d: _dhuber(d, delta),
                    lambda d: _chuber(d, delta))


def quad_penalty(x, mode):
    if mode == 2:
        return np.full(np.asarray(x).shape, F32(4 + 4 * AXY + 2 * AZ), dtype=F32)
    return _penalty(x, mode, lambda d: float((d.astype(np.float64) ** 2 / 2).sum()), lambda d: d, None)


def recon_pwls_se_sqs(y, w, geom, beta, pfun, itnlim, delta, numos, img0, fp64=False, history=None):
    """reconPwlsSeSqs.m with the SF projectors of loadPojectors.m; returns (x, phis, rmsds).
    ``fp64`` runs the same iteration in double with the FP64 projectors (the FP64 oracle);
    ``history``, if a list, receives a copy of x after every outer iteration."""
    if fp64:
        return _recon_pwls_fp64(y, w, geom, beta, pfun, itnlim, delta, numos, img0, history)
    if pfun == "huber":
        R = lambda x: huber_penalty(x, 0, delta)
        S = lambda x: huber_penalty(x, 1, delta)
        T = lambda x: huber_penalty(x, 2, delta)
    else:
        R = lambda x: quad_penalty(x, 0)
        S = lambda x: quad_penalty(x, 1)
        T = lambda x: quad_penalty(x, 2)
    M = numos
    x = np.asarray(img0, dtype=F32).copy()
    a = oracle_cbct("proj,tf", geom, np.ones_like(x))
    precom = oracle_cbct("back,tf", geom, (w * a).astype(F32))
    phis, rmsds = [], []
    for itn in range(1, itnlim + 1):
        xold = x.copy()
        phi = 0.0
        for isub in range(1, M + 1):
            g = geom.subset(M, isub)
            start = isub % M if M > 1 else 0
            ys = y[start::M] if M > 1 else y
            ws = w[start::M] if M > 1 else w
            d = (oracle_cbct("proj,tf", g, x) - ys).astype(F32)
            num = oracle_cbct("back,tf", g, (ws * d).astype(F32))
            if M != 1:
                num = (F32(M) * num).astype(F32)
            num = (num + F32(beta) * S(x)).astype(F32)
            den = (precom + F32(beta) * T(x)).astype(F32)
            x = (x - num / den).astype(F32)
            x[x < 0] = 0
            x[np.isnan(x)] = 0
            x[np.isinf(x)] = 0
            phi += float((ws.astype(np.float64) * d.astype(np.float64) ** 2).sum()) / 2
        phi += beta * R(x)
        rmsd = float(np.sqrt(np.mean((x.astype(np.float64) - xold) ** 2)))
        phis.append(phi)
        rmsds.append(rmsd)
        if history is not None:
            history.append(x.copy())
        if itn > 5 and rmsd < 1e-5:
            break
    return x, np.array(phis), np.array(rmsds)


def _penalty64(x, mode, kind, delta):
    """huberPenalty.m / quadPenalty.m in double (same neighbourhood as _penalty)."""
    X = np.asarray(x, dtype=np.float64).transpose(2, 1, 0)
    pairs = [((slice(0, -1), slice(None), slice(None)), (slice(1, None), slice(None), slice(None)), 1.0),
             ((slice(None), slice(0, -1), slice(None)), (slice(None), slice(1, None), slice(None)), 1.0),
             ((slice(0, -1), slice(0, -1), slice(None)), (slice(1, None), slice(1, None), slice(None)), 1 / np.sqrt(2)),
             ((slice(1, None), slice(0, -1), slice(None)), (slice(0, -1), slice(1, None), slice(None)), 1 / np.sqrt(2)),
             ((slice(None), slice(None), slice(0, -1)), (slice(None), slice(None), slice(1, None)), 0.5)]
    if kind == "quad" and mode == 2:
        return np.full(np.asarray(x).shape, 4 + 4 / np.sqrt(2) + 1.0)
    if mode == 0:
        tot = 0.0
        for p, q, c in pairs:
            d = np.abs(X[p] - X[q])
            h = d ** 2 / 2 if kind == "quad" else np.where(d > delta, delta * d - delta ** 2 / 2, d ** 2 / 2)
            tot += c * h.sum()
        return tot
    y = np.zeros(X.shape)
    for p, q, c in pairs:
        d = X[p] - X[q]
        if mode == 1:
            g = d if kind == "quad" else np.clip(d, -delta, delta)
            y[p] += c * g
            y[q] -= c * g
        else:
            g = (np.abs(d) <= delta).astype(np.float64)
            y[p] += c * g
            y[q] += c * g
    return y.transpose(2, 1, 0).copy()


def _recon_pwls_fp64(y, w, geom, beta, pfun, itnlim, delta, M, img0, history):
    x = np.asarray(img0, dtype=np.float64).copy()
    y = np.asarray(y, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    a = oracle_cbct("proj,tf", geom, np.ones_like(x), fp64=True)
    precom = oracle_cbct("back,tf", geom, w * a, fp64=True)
    phis, rmsds = [], []
    for itn in range(1, itnlim + 1):
        xold = x.copy()
        phi = 0.0
        for isub in range(1, M + 1):
            g = geom.subset(M, isub)
            start = isub % M if M > 1 else 0
            ys = y[start::M] if M > 1 else y
            ws = w[start::M] if M > 1 else w
            d = oracle_cbct("proj,tf", g, x, fp64=True) - ys
            num = M * oracle_cbct("back,tf", g, ws * d, fp64=True) + beta * _penalty64(x, 1, pfun, delta)
            den = precom + beta * _penalty64(x, 2, pfun, delta)
            x = x - num / den
            x[~np.isfinite(x) | (x < 0)] = 0
            phi += float((ws * d ** 2).sum()) / 2
        phi += beta * _penalty64(x, 0, pfun, delta)
        phis.append(phi)
        rmsds.append(float(np.sqrt(np.mean((x - xold) ** 2))))
        if history is not None:
            history.append(x.copy())
        if itn > 5 and rmsds[-1] < 1e-5:
            break
    return x, np.array(phis), np.array(rmsds)


def _matlab_round(v):
    return int(np.floor(abs(v) + 0.5)) * (1 if v >= 0 else -1)


def recon_pwls_nesterov_sqs(y, w, geom, beta, pfun, itnlim, delta, numos, img0, img_opt=None, history=None):
    """reconPwlsSeNesterovSqs.m in single precision (MATLAB: a double scalar times a single
    array is computed in single); returns (x, phis, rmsds).  ``history``, if a list,
    receives a copy of x after every outer iteration."""
    if pfun == "huber":
        R = lambda x: huber_penalty(x, 0, delta)
        S = lambda x: huber_penalty(x, 1, delta)
        T = lambda x: huber_penalty(x, 2, delta)
    else:
        R = lambda x: quad_penalty(x, 0)
        S = lambda x: quad_penalty(x, 1)
        T = lambda x: quad_penalty(x, 2)
    M = numos
    stop_crt = 1e-10
    nrestart = _matlab_round(itnlim * 2)
    x = np.asarray(img0, dtype=F32).copy()
    a = oracle_cbct("proj,tf", geom, np.ones_like(x))
    precom = oracle_cbct("back,tf", geom, (w * a).astype(F32))
    t = 1.0
    z = x.copy()
    s = x.copy()
    phis, rmsds = [], []

    def clean(v):
        v = v.copy()
        v[v < 0] = 0
        v[np.isnan(v)] = 0
        v[np.isinf(v)] = 0
        return v

    for itn in range(1, itnlim + 1):
        xold = x.copy()
        phi = 0.0
        for isub in range(1, M + 1):
            g = geom.subset(M, isub)
            start = isub % M if M > 1 else 0
            ys = y[start::M] if M > 1 else y
            ws = w[start::M] if M > 1 else w
            d = (oracle_cbct("proj,tf", g, z) - ys).astype(F32)
            grad = oracle_cbct("back,tf", g, (ws * d).astype(F32))
            if M != 1:
                grad = (F32(M) * grad).astype(F32)
            grad = (grad + F32(beta) * S(z)).astype(F32)
            du = (grad / (precom + F32(beta) * T(x)).astype(F32)).astype(F32)
            x = (z - du).astype(F32)
            s = (s - F32(t) * du).astype(F32)
            t = (1 + np.sqrt(1 + 4 * t * t)) / 2
            z = (F32(1 - 1 / t) * x + F32(1 / t) * s).astype(F32)
            x, s, z = clean(x), clean(s), clean(z)
            phi += float((ws.astype(np.float64) * d.astype(np.float64) ** 2).sum()) / 2
        phi += beta * R(x)
        if img_opt is None:
            rmsd = float(np.sqrt(np.mean((x.astype(np.float64) - xold) ** 2)))
        else:
            k = x.shape[0] // 2 - 1  # x(:,:,end/2) in the [nz, ny, nx] layout
            rmsd = float(np.sqrt(np.mean((x[k].astype(np.float64) - np.asarray(img_opt, np.float64)[k]) ** 2)))
        phis.append(phi)
        rmsds.append(rmsd)
        if history is not None:
            history.append(x.copy())
        if itn > 5 and rmsd < stop_crt:
            break
        if itn % nrestart == 0:
            t = 1.0
            z = x.copy()
            s = x.copy()
    return x, np.array(phis), np.array(rmsds)
