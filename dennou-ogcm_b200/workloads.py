"""Seeded synthetic workloads of the transform benchmark configurations.

No public dataset is involved: the inputs are seeded spectra with the
power-law shapes the configurations name.  Seed 20261203; complex
a_nm ~ N(0,1) (n+1)^-p with Im a_n0 = 0, stored in the SPML real layout
(wa(l_nm(n,m)) = sqrt2 Re a, wa(l_nm(n,-m)) = sqrt2 Im a for m > 0).

    C0  T21  (64 x 32),    20 levels x 3 fields, p = 1.5
    C1  T85  (256 x 128),  60 levels x 8 fields; vor/div p = 2, T/S p = 1.5
    C2  T170 (512 x 256),  60 levels x 12 fields, p = 1.5
    C3  64 instances T21/T42/T85/T170 in ratio 8:4:2:1, levels U[10,60], 3-8 fields
    C4  T341 (1024 x 512), 60 levels x 16 fields, p = 2, diffusion ~ [n(n+1)]^4
"""
from __future__ import annotations

import numpy as np

SEED = 20261203

GRIDS = {
    "T21": (64, 32, 21),
    "T42": (128, 64, 42),
    "T85": (256, 128, 85),
    "T170": (512, 256, 170),
    "T341": (1024, 512, 341),
}

CONFIGS = {
    "C0": dict(grid="T21", levels=20, fields=3, power=1.5),
    "C1": dict(grid="T85", levels=60, fields=8, power=2.0),
    "C2": dict(grid="T170", levels=60, fields=12, power=1.5),
    "C4": dict(grid="T341", levels=60, fields=16, power=2.0),
}


def spectral_scale(N: int, power: float) -> np.ndarray:
    """(n+1)^-power per SPML index l = n(n+1)+m, with the sqrt2 of the m != 0 entries."""
    L = (N + 1) ** 2
    n = np.floor(np.sqrt(np.arange(L))).astype(np.int64)
    m = np.arange(L) - n * (n + 1)
    s = (n + 1.0) ** (-power)
    return np.where(m == 0, s, s * np.sqrt(2.0))


def seeded_spectra(N: int, nb: int, power: float, seed: int = SEED, rng=None) -> np.ndarray:
    """(nb, (N+1)^2) SPML-layout spectra of the seeded distribution."""
    rng = np.random.default_rng(seed) if rng is None else rng
    L = (N + 1) ** 2
    out = rng.standard_normal((nb, L)) * spectral_scale(N, power)[None, :]
    return out


def seeded_spectra_torch(N: int, nb: int, power: float, device, seed: int = SEED):
    """The same distribution generated directly on a CUDA device (torch Philox)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    L = (N + 1) ** 2
    x = torch.randn((nb, L), generator=g, device=device, dtype=torch.float64)
    return x * torch.from_numpy(spectral_scale(N, power)).to(device)[None, :]


def mixed_instances(count: int = 64, seed: int = SEED):
    """C3: `count` instances with truncations T21/T42/T85/T170 in ratio 8:4:2:1,
    levels uniform in [10, 60] and 3-8 fields; returns a list of dicts."""
    rng = np.random.default_rng(seed)
    kinds = ["T21"] * 8 + ["T42"] * 4 + ["T85"] * 2 + ["T170"]
    out = []
    for k in range(count):
        g = kinds[k % len(kinds)]
        out.append(dict(grid=g, levels=int(rng.integers(10, 61)), fields=int(rng.integers(3, 9))))
    return out


def diffusion_coef(N: int, order: int = 8, dt_nu: float = 1e-3) -> np.ndarray:
    """C4 diagonal: dt c_n = -dt_nu [n(n+1) / (N(N+1))]^(order/2), normalised so the
    highest degree is damped by 1/(1 + dt_nu) (LPhys_DIFF_spm_mod.f90:151-158 with
    NumDiffOrdH = order).  Returned as c_n with dt = 1."""
    L = (N + 1) ** 2
    n = np.floor(np.sqrt(np.arange(L)))
    return -dt_nu * (n * (n + 1.0) / (N * (N + 1.0))) ** (order // 2)
