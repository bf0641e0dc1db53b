"""Seeded synthetic single-look InSAR pairs.

The scenes stand in for real interferograms in the benchmarks and tests:

* ground truth: a background reflectivity R0 ~ LogNormal(0, 1) with
  coherence g0 ~ U[0.2, 0.95], overpainted in order by 40 axis-aligned
  rectangles, each with its own R ~ LogNormal(0, 1) and g ~ U[0.2, 0.95];
  rectangle sides are uniform in [ceil(H/16), ceil(H/4)] x [ceil(W/16),
  ceil(W/4)] with a uniform top-left corner, clipped to the image;
* phase: 3 fringes of linear ramp across the width plus 5 Gaussian bumps of
  amplitude 2*pi and sigma 30 px at uniform centres, wrapped to (-pi, pi];
* speckle: single-look circular complex Gaussian with the given coherence,
  built like despeckCL's InSAR simulator (src/compute/nlinsar/insarsim_simu.cpp:34-60):
  l1 = sqrt(R), l2 = l1*g*exp(jB), l3 = l1*sqrt(1-g^2), slc1 = l1*x1,
  slc2 = l2*x1 + l3*x2 with x ~ CN(0, 1); B = -phase so that
  arg(slc1*conj(slc2)) has mean phase.
"""
from __future__ import annotations

import math

import numpy as np


def _speckle(rng, refl, coh, phase):
    H, W = refl.shape
    x1 = (rng.standard_normal((H, W), dtype=np.float32) + 1j * rng.standard_normal((H, W), dtype=np.float32))
    x2 = (rng.standard_normal((H, W), dtype=np.float32) + 1j * rng.standard_normal((H, W), dtype=np.float32))
    x1 *= np.float32(1 / math.sqrt(2))
    x2 *= np.float32(1 / math.sqrt(2))
    l1 = np.sqrt(refl).astype(np.float32)
    l2 = l1 * coh * np.exp(-1j * phase)
    l3 = l1 * np.sqrt(1 - coh * coh)
    slc1 = l1 * x1
    slc2 = l2 * x1 + l3 * x2
    a1 = np.abs(slc1).astype(np.float32)
    a2 = np.abs(slc2).astype(np.float32)
    ph = np.angle(slc1 * np.conj(slc2)).astype(np.float32)
    return a1, a2, ph


def ground_truth(H: int, W: int, seed: int, n_rect: int = 40):
    rng = np.random.default_rng(seed)
    refl = np.full((H, W), rng.lognormal(0.0, 1.0), np.float32)
    coh = np.full((H, W), rng.uniform(0.2, 0.95), np.float32)
    hmin, hmax = math.ceil(H / 16), max(math.ceil(H / 4), math.ceil(H / 16))
    wmin, wmax = math.ceil(W / 16), max(math.ceil(W / 4), math.ceil(W / 16))
    for _ in range(n_rect):
        y0 = int(rng.integers(0, H))
        x0 = int(rng.integers(0, W))
        hh = int(rng.integers(hmin, hmax + 1))
        ww = int(rng.integers(wmin, wmax + 1))
        refl[y0:y0 + hh, x0:x0 + ww] = rng.lognormal(0.0, 1.0)
        coh[y0:y0 + hh, x0:x0 + ww] = rng.uniform(0.2, 0.95)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float32)
    phase = 2 * np.pi * 3 * xx / W
    for _ in range(5):
        cy = rng.uniform(0, H)
        cx = rng.uniform(0, W)
        phase = phase + 2 * np.pi * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * 30.0 ** 2))
    phase = np.angle(np.exp(1j * phase)).astype(np.float32)
    return refl, coh, phase, rng


def insar_scene(H: int, W: int, seed: int):
    """(ampl_master, ampl_slave, phase) float32 arrays of shape (H, W)."""
    refl, coh, phase, rng = ground_truth(H, W, seed)
    return _speckle(rng, refl, coh, phase)


def training_area(size: int = 128, seed: int = 7, reflectivity: float = 1.0, coherence: float = 0.6):
    """A homogeneous training pair (reflectivity 1, coherence 0.6, phase 0)."""
    rng = np.random.default_rng(seed)
    refl = np.full((size, size), reflectivity, np.float32)
    coh = np.full((size, size), coherence, np.float32)
    phase = np.zeros((size, size), np.float32)
    return _speckle(rng, refl, coh, phase)


def insar_scene_device(H: int, W: int, seed: int, device="cuda"):
    """The same recipe drawn with torch's generator on `device`: (ampl_master,
    ampl_slave, phase) float32 tensors of shape (H, W).  Used where many large
    scenes are needed quickly (the serving benchmark); the values differ from
    insar_scene's for the same seed, the distributions do not."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    cpu = np.random.default_rng(seed)
    refl = torch.full((H, W), float(cpu.lognormal(0.0, 1.0)), device=device)
    coh = torch.full((H, W), float(cpu.uniform(0.2, 0.95)), device=device)
    hmin, hmax = math.ceil(H / 16), max(math.ceil(H / 4), math.ceil(H / 16))
    wmin, wmax = math.ceil(W / 16), max(math.ceil(W / 4), math.ceil(W / 16))
    for _ in range(40):
        y0, x0 = int(cpu.integers(0, H)), int(cpu.integers(0, W))
        hh, ww = int(cpu.integers(hmin, hmax + 1)), int(cpu.integers(wmin, wmax + 1))
        refl[y0:y0 + hh, x0:x0 + ww] = float(cpu.lognormal(0.0, 1.0))
        coh[y0:y0 + hh, x0:x0 + ww] = float(cpu.uniform(0.2, 0.95))
    yy = torch.arange(H, device=device, dtype=torch.float32)[:, None]
    xx = torch.arange(W, device=device, dtype=torch.float32)[None, :]
    phase = (2 * math.pi * 3 / W) * xx + torch.zeros_like(yy)
    for _ in range(5):
        cy, cx = float(cpu.uniform(0, H)), float(cpu.uniform(0, W))
        phase = phase + 2 * math.pi * torch.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * 30.0 ** 2))
    phase = torch.atan2(torch.sin(phase), torch.cos(phase))

    def cn():
        re = torch.randn((H, W), generator=g, device=device)
        im = torch.randn((H, W), generator=g, device=device)
        return torch.complex(re, im) * (1 / math.sqrt(2))

    x1, x2 = cn(), cn()
    l1 = torch.sqrt(refl)
    l2 = l1 * coh * torch.exp(torch.complex(torch.zeros_like(phase), -phase))
    l3 = l1 * torch.sqrt(1 - coh * coh)
    slc1 = l1 * x1
    slc2 = l2 * x1 + l3 * x2
    return (slc1.abs().contiguous(), slc2.abs().contiguous(),
            torch.angle(slc1 * torch.conj(slc2)).float().contiguous())
