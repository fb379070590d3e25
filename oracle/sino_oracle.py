"""Oracle for the sinogram pre-processing path (TEST INFRASTRUCTURE ONLY).

    philox4x32_10        the counter-based generator of Salmon, Moraes, Dror and Shaw,
                         "Parallel random numbers: as easy as 1, 2, 3" (SC'11), 10 rounds
    poisson_ptrs         Hoermann's transformed rejection with squeeze (PTRS, 1993) for
                         lambda >= 10, multiplication (inversion) below, driven by the
                         per-element Philox stream the device sampler uses
    simulate_counts      sinogram/sim/simulateSimplePoissonData.m:161-190 (monochromatic):
                         poissrnd(photons * exp(-line)) + sqrt(electronicNoise) * randn
    log_attenuation      sinogram/log/computeSimplePoissonSinogramAttunation.m:14-54:
                         -log(max(I, 10) / I0 [./ flatFieldRatio]) in single precision

MATLAB's poissrnd/randn streams cannot be reproduced; the device sampler is checked
against this restatement of its own published algorithms (bit-exact stream, the same
integer draws) and against the Poisson moments.  Parity unpinned against MATLAB:
the log transform is restated from the .m source, and no reference output exists here.
"""
from __future__ import annotations

import math

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    c0, c1, c2, c3 = (int(v) & MASK for v in ctr)
    k0, k1 = (int(v) & MASK for v in key)
    for r in range(10):
        if r:
            k0 = (k0 + W0) & MASK
            k1 = (k1 + W1) & MASK
        p0 = M0 * c0
        p1 = M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ c3 ^ k1) & MASK, p0 & MASK
    return c0, c1, c2, c3


class _Stream:
    """Uniforms in (0, 1) of element i: Philox block (i_lo, i_hi, j, 0) under the seed
    key, j = 0, 1, ...; each 32-bit word u gives (u + 0.5) * 2^-32."""

    def __init__(self, i, seed):
        self.i, self.key = i, (seed & MASK, (seed >> 32) & MASK)
        self.j, self.buf = 0, []

    def next(self):
        if not self.buf:
            w = philox4x32_10((self.i & MASK, (self.i >> 32) & MASK, self.j, 0), self.key)
            self.j += 1
            self.buf = list(w)
        return (self.buf.pop(0) + 0.5) * 2.0 ** -32


def poisson_ptrs(lam, stream, max_tries=64):
    """One Poisson(lam) draw from the stream; (k, tries)."""
    if lam <= 0.0:
        return 0, 0
    if lam < 10.0:
        # multiplication method: smallest k with U1 ... U(k+1) <= exp(-lam)
        lim = math.exp(-lam)
        k, prod = 0, stream.next()
        while prod > lim and k < 1000:
            k += 1
            prod *= stream.next()
        return k, 1
    slam = math.sqrt(lam)
    loglam = math.log(lam)
    b = 0.931 + 2.53 * slam
    a = -0.059 + 0.02483 * b
    invalpha = 1.1239 + 1.1328 / (b - 3.4)
    vr = 0.9277 - 3.6224 / (b - 2.0)
    for tries in range(1, max_tries + 1):
        U = stream.next() - 0.5
        V = stream.next()
        us = 0.5 - abs(U)
        k = math.floor((2.0 * a / us + b) * U + lam + 0.43)
        if us >= 0.07 and V <= vr:
            return k, tries
        if k < 0 or (us < 0.013 and V > us):
            continue
        if (math.log(V) + math.log(invalpha) - math.log(a / (us * us) + b)) <= (-lam + k * loglam -
                                                                                  math.lgamma(k + 1.0)):
            return k, tries
    return int(math.floor(lam + 0.5)), max_tries + 1


def normal(stream):
    """Box-Muller: sqrt(-2 log u1) cos(2 pi u2)."""
    u1, u2 = stream.next(), stream.next()
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def simulate_counts(line, photons, electronic_noise=0.0, seed=0, add_noise=True):
    """float32 counts: Poisson(photons * exp(-line)) [+ sqrt(electronic_noise) * N(0,1)], or
    round(photons * exp(-line)) without noise.  The Poisson draw uses the element's
    stream (Philox blocks (i, j, 0)), the normal its own (blocks (i, j, 1))."""
    line = np.asarray(line, dtype=np.float32).reshape(-1)
    out = np.empty(line.size, dtype=np.float32)
    sd = float(np.sqrt(np.float32(electronic_noise)))  # the device holds the deviation in float
    for i, li in enumerate(line):
        lam = float(np.float32(np.float32(photons) * np.exp(np.float32(-li))))
        if not add_noise:
            out[i] = np.float32(math.floor(abs(lam) + 0.5))
            continue
        st = _Stream(i, seed)
        k, _ = poisson_ptrs(lam, st)
        v = float(k)
        if electronic_noise > 0:
            v = v + sd * normal(_NormalStream(i, seed))
        out[i] = np.float32(v)
    return out


class _NormalStream(_Stream):
    """The electronic-noise normal of element i: Philox blocks (i_lo, i_hi, j, 1)."""

    def next(self):
        if not self.buf:
            w = philox4x32_10((self.i & MASK, (self.i >> 32) & MASK, self.j, 1), self.key)
            self.j += 1
            self.buf = list(w)
        return (self.buf.pop(0) + 0.5) * 2.0 ** -32


def log_attenuation(intensity, source_intensity, flat_field=None):
    """-log(max(I, 10) / I0 [./ flat]) in float32; intensity [views, nu, nv], flat [nu, nv]."""
    I = np.maximum(np.asarray(intensity, dtype=np.float32), np.float32(10.0))
    r = (I / np.float32(source_intensity)).astype(np.float32)
    if flat_field is not None:
        r = (r / np.asarray(flat_field, dtype=np.float32)[None]).astype(np.float32)
    return (-np.log(r)).astype(np.float32)
