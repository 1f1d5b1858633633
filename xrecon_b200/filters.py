"""Spatial reconstruction filters of length 2*Nu-1, API-compatible with
``xrecon.projector.filters`` (XRecon xrecon/projector/filters.py:3-71).

The filter tables have to equal the reference's: the Ram-Lak kernel
h[n] = 1/(4 d^2) at n = 0, -1/(pi^2 d^2 n^2) at odd n, 0 at even n; the
Shepp-Logan kernel -2/(pi^2 d^2 (4n^2 - 1)); and the cosine, Hamming and
Hann filters obtained by multiplying the FFT of the Ram-Lak kernel (FP64)
with the window over the frequency index w = k*pi/Nu, k in
[0..Nu-1, -(Nu-1)..-1].  Tables are computed in float64 and rounded once.
"""
from __future__ import annotations

import math

import torch

FILTERS = {}


def register_filter(name):
    def deco(fn):
        FILTERS[name] = fn
        return fn
    return deco


def filter_generate(num_det: int, det_size: float, filter_type: str = "ramp", dtype=None) -> torch.Tensor:
    if filter_type not in FILTERS:
        raise ValueError(f"Filter type {filter_type} not supported. Available: {list(FILTERS.keys())}")
    return FILTERS[filter_type](num_det, det_size, dtype or torch.float32)


def _offsets(num_det: int) -> torch.Tensor:
    return torch.arange(2 * num_det - 1, dtype=torch.float64) - (num_det - 1)


@register_filter("ramp")
def ramp(num_det: int, det_size: float, dtype=torch.float32) -> torch.Tensor:
    n = _offsets(num_det)
    h = torch.zeros_like(n)
    odd = torch.remainder(n, 2) != 0
    h[odd] = -1.0 / (math.pi ** 2 * det_size ** 2 * (n[odd] ** 2 + 1e-12))
    h[num_det - 1] = 1.0 / (4.0 * det_size ** 2)
    return h.to(dtype)


@register_filter("shepplogan")
def shepplogan(num_det: int, det_size: float, dtype=torch.float32) -> torch.Tensor:
    n = _offsets(num_det)
    return (-2.0 / (math.pi ** 2 * det_size ** 2 * (4.0 * n ** 2 - 1.0))).to(dtype)


def _windowed(num_det: int, det_size: float, window) -> torch.Tensor:
    # The window is applied to the float32 Ram-Lak table, as the reference
    # does (filters.py:44-50), so both tables agree to float32 rounding.
    h = ramp(num_det, det_size, torch.float32).to(torch.float64)
    k = torch.cat((torch.arange(0, num_det), torch.arange(-num_det + 1, 0))).to(torch.float64)
    w = window(k * math.pi / num_det)
    return torch.fft.ifft(torch.fft.fft(h) * w).real.to(torch.float32)


@register_filter("cosine")
def cosine(num_det: int, det_size: float, dtype=torch.float32) -> torch.Tensor:
    return _windowed(num_det, det_size, lambda w: torch.cos(w / 2))


@register_filter("hamming")
def hamming(num_det: int, det_size: float, dtype=torch.float32) -> torch.Tensor:
    return _windowed(num_det, det_size, lambda w: 0.54 + 0.46 * torch.cos(w))


@register_filter("hann")
def hann(num_det: int, det_size: float, dtype=torch.float32) -> torch.Tensor:
    return _windowed(num_det, det_size, lambda w: 0.5 * (1 + torch.cos(w)))
