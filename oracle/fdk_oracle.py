"""Oracle for the FDK path (TEST INFRASTRUCTURE ONLY): numpy restatements of the
reference's MATLAB, line by line, in float64, with the backprojection by the C
oracle.

    design_filter2            fbp/filter/designFilter2.m:18-78
    design_equiangular        fbp/filter/designEquiangularFilter2.m:19-78
    filter_freq               fbp/filter/filterFreq.m:42-50 (filt1D)
    short_scan_parker_weight  fbp/weights/shortScanParkerWeight.m:1-40
    recon_fdk                 fbp/reconFDK.m:1-85

MATLAB itself is not available, and its FFT (FFTW, single precision for single
input) cannot be run here: parity unpinned. The filter step is checked against
this float64 restatement (and its FFT against numpy's FP64 FFT), not against MATLAB;
the backprojection inside it is the pinned C oracle.
"""
from __future__ import annotations

import numpy as np

from .bindings import oracle_cbct


def _order(length):
    # max(64, 2^nextpow2(2*len-1)); nextpow2(n) = ceil(log2(n))
    return max(64, int(2 ** int(np.ceil(np.log2(2 * length - 1)))))


def _window(filt, order, window, crop):
    w = 2 * np.pi * np.arange(filt.size) / order
    f = filt.copy()
    if window == "ram-lak":
        pass
    elif window == "shepp-logan":
        f[1:] = f[1:] * (np.sin(w[1:] / (2 * crop)) / (w[1:] / (2 * crop)))
    elif window == "cosine":
        f[1:] = f[1:] * np.cos(w[1:] / (2 * crop))
    elif window == "hamming":
        f[1:] = f[1:] * (.54 + .46 * np.cos(w[1:] / crop))
    elif window == "hann":
        f[1:] = f[1:] * (1 + np.cos(w[1:] / crop)) / 2
    elif window in ("hann50", "hann75", "hann80"):
        crop = {"hann50": 0.5, "hann75": 0.75, "hann80": 0.80}[window]
        f[1:] = f[1:] * (1 + np.cos(w[1:] / crop)) / 2
    elif window in ("B50", "B75", "B80"):
        crop = {"B50": 0.5, "B75": 0.75, "B80": 0.80}[window]
    elif window in ("C50", "C75", "C80"):
        crop = {"C50": 0.5, "C75": 0.75, "C80": 0.80}[window]
        f[1:] = f[1:] * np.cos(w[1:] / (2 * crop))
    else:
        raise ValueError("Invalid window selected.")
    f[w > np.pi * crop] = 0
    return np.concatenate([f, f[-2:0:-1]])


def design_filter2(gamma, window, length, crop=1.0):
    order = _order(length)
    index = np.arange(-order // 2 + 1, order // 2)
    h = np.zeros(index.size)
    h[index == 0] = 1 / (4 * gamma ** 2)
    odd = np.mod(index, 2) == 1
    h[odd] = -1.0 / (index[odd] * np.pi * gamma) ** 2
    h = np.append(h, 0.0)  # h(order) = 0
    filt = np.abs(np.fft.fft(h))[: order // 2 + 1]
    return _window(filt, order, window, crop)


def design_equiangular(gamma, sdd, window, length, crop=1.0):
    order = _order(length)
    index = np.arange(-order // 2 + 1, order // 2)
    h = np.zeros(index.size)
    h[index == 0] = 1 / (4 * gamma ** 2)
    odd = np.mod(index, 2) == 1
    h[odd] = -1.0 / (sdd * np.pi * np.sin(index[odd] * gamma / sdd)) ** 2
    h = np.append(h, 0.0)
    filt = np.abs(np.fft.fft(h))[: order // 2 + 1]
    return _window(filt, order, window, crop)


def filter_freq(x, H):
    """filterFreq.m filt1D on the last axis: zero-pad to len(H), FFT, x H, IFFT, real, truncate."""
    n = x.shape[-1]
    pad = np.zeros(x.shape[:-1] + (H.size,))
    pad[..., :n] = x
    return np.real(np.fft.ifft(np.fft.fft(pad, axis=-1) * H, axis=-1))[..., :n]


def _s(b):
    b = np.asarray(b, dtype=np.float64)
    return np.where(b <= -0.5, 0.0, np.where(np.abs(b) < 0.5, 0.5 * (1 + np.sin(np.pi * b)), 1.0))


def short_scan_parker_weight(gammas, beta, tau):
    gamma = -np.asarray(gammas, dtype=np.float64)
    return _s(beta / (tau - 2 * gamma) - 0.5) - _s((beta - np.pi + 2 * gamma) / (tau + 2 * gamma) - 0.5)


def filtered_sinogram(sino, geom, window="hamming", crop=1.0):
    """reconFDK.m:19-76: weighted and filtered sinogram, float64 [views, nu, nv]."""
    nu, nv = geom.detSize
    du, dv = geom.detSpacing
    ou, ov = geom.detOffset
    SDD, SAD = float(geom.SDD), float(geom.SAD)
    betas = np.asarray(geom.betas, dtype=np.float64)
    u = (np.arange(nu) - (nu - 1) / 2.0 + ou) * du
    v = (np.arange(nv) - (nv - 1) / 2.0 + ov) * dv
    uu, vv = np.meshgrid(u, v)  # [nv, nu]
    if geom.flatPanel:
        weight = SAD * np.sqrt(1.0 + (uu ** 2 / SDD ** 2)) / np.sqrt(uu ** 2 + vv ** 2 + SDD ** 2)
        H = du * design_filter2(du, window, nu, crop)
        gamma = np.arctan(-u / SDD)
        tau = abs(betas[-1] - betas[0]) - np.pi
    else:
        weight = SAD / SDD * np.cos(uu / (np.sqrt(SDD ** 2 + vv ** 2)))
        H = du * design_equiangular(du, SDD, window, nu, crop)
        gamma = -u / SDD
        tau = abs(betas.max() - betas.min()) - np.pi
    beta_min = betas.min()
    out = np.empty(sino.shape, dtype=np.float64)
    for view in range(betas.size):
        proj = weight * np.asarray(sino[view], dtype=np.float64).T  # [nv, nu]
        if geom.shortScan:
            proj = proj * short_scan_parker_weight(gamma, betas[view] - beta_min, tau)[None, :]
        out[view] = filter_freq(proj, H).T
    return out


def recon_fdk(sino, geom, window="hamming", crop=1.0):
    """reconFDK.m: filter, back,hpd (C oracle, bit-identical to the reference), x dbeta x 10."""
    betas = np.asarray(geom.betas, dtype=np.float64)
    filt = filtered_sinogram(sino, geom, window, crop).astype(np.float32)
    dbeta = abs(betas[-1] - betas[0]) / (betas.size - 1)
    if not geom.shortScan:
        dbeta = dbeta / 2
    img = oracle_cbct("back,hpd", geom, filt).astype(np.float64) * dbeta * 10
    return img.astype(np.float32)
