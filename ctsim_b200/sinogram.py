"""Sinogram pre-processing on the device (the data step in front of the projectors).

* ``simulateSimplePoissonData(line, photons, electronicNoise, seed, addCountingNoise)``
      sinogram/sim/simulateSimplePoissonData.m:161-190 for a monochromatic spectrum: the
      counts Poisson(photons * exp(-line)) + sqrt(electronicNoise) * randn, from line
      integrals already in the units of the exponent; photons = DQE * photonsTotal.
* ``computeSimplePoissonSinogramAttunation(intensity, sourceIntensity, flatFieldRatio)``
      sinogram/log/computeSimplePoissonSinogramAttunation.m:14-54: -log(max(I, 10) / I0),
      with the bowtie flat-field ratio of one view if given.
* ``computeWeightsPwls`` (statsrecon/pwls/computeWeightsPwls.m) is in ctsim_b200.pwls.

Torch CUDA tensors in and out ([views, nu, nv] float32); the random draws depend only
on (seed, element), not on the device or launch shape.
"""
from __future__ import annotations

from . import _lib


def _torch():
    import torch
    return torch


def simulateSimplePoissonData(line, photons: float, electronicNoise: float = 0.0, seed: int = 0,
                              addCountingNoise: bool = True, return_fallbacks: bool = False):
    torch = _torch()
    line = line.contiguous()
    if line.dtype != torch.float32 or not line.is_cuda:
        raise TypeError("line must be a float32 CUDA tensor")
    counts = torch.empty_like(line)
    fb = torch.zeros(1, dtype=torch.int32, device=line.device)
    st = torch.cuda.current_stream(line.device).cuda_stream
    _lib.check(_lib.load().ctsim_simulate_counts(line.data_ptr(), line.numel(), float(photons),
                                                 float(electronicNoise), int(seed) & (2 ** 64 - 1),
                                                 1 if addCountingNoise else 0, counts.data_ptr(), fb.data_ptr(), st),
               "ctsim_simulate_counts")
    return (counts, fb) if return_fallbacks else counts


def computeSimplePoissonSinogramAttunation(intensity, sourceIntensity: float, flatFieldRatio=None):
    torch = _torch()
    intensity = intensity.contiguous()
    if intensity.dtype != torch.float32 or not intensity.is_cuda:
        raise TypeError("intensity must be a float32 CUDA tensor")
    flat, nuv = None, 0
    if flatFieldRatio is not None:
        flatFieldRatio = flatFieldRatio.to(intensity.device, torch.float32).contiguous()
        if tuple(flatFieldRatio.shape) != tuple(intensity.shape[1:]):
            raise ValueError("flatFieldRatio must have the shape of one view [nu, nv]")
        flat, nuv = flatFieldRatio.data_ptr(), flatFieldRatio.numel()
    sino = torch.empty_like(intensity)
    st = torch.cuda.current_stream(intensity.device).cuda_stream
    _lib.check(_lib.load().ctsim_log_attenuation(intensity.data_ptr(), intensity.numel(), float(sourceIntensity),
                                                 flat, nuv, sino.data_ptr(), st), "ctsim_log_attenuation")
    return sino
