"""Generate golden vectors for the spherical-harmonic transform.

The reference keeps its transform arithmetic in SPMODEL/ISPACK, which are
not part of the reference tree, and the reference has no test or golden file
for it.  These vectors are therefore an INDEPENDENT evaluation of the written
specification (doc/description/ogcm/space_discretization.tex:161-267,350-381
and model/dogcm/src/util/math/SpmlUtil_mod.f90:299-473) with scipy and numpy:

* Gauss nodes/weights from scipy.special.roots_legendre;
* Pbar_n^m from scipy.special.lpmv with the Condon-Shortley phase removed and
  the normalisation int Pbar^2 dmu = 2 applied;
* (1-mu^2) dPbar/dmu from the classical identity
  (1-x^2) dP_n^m/dx = (n+m) P_{n-1}^m - n x P_n^m (not the eps-recurrence used
  by the oracle and by the CUDA library);
* every transform as a direct O(L * I * J) sum (no FFT, no symmetry).

Seeding follows the C0 workload: a_nm ~ N(0,1) (n+1)^-1.5, Im a_n0 = 0,
numpy default_rng(20261203).

Run:  python tests/golden/make_golden.py   (writes tests/golden/sht_T*.npz)
"""
from __future__ import annotations

import math
import os

import numpy as np
from scipy.special import lpmv, roots_legendre

HERE = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203


def pbar_table(N: int, mu: np.ndarray) -> np.ndarray:
    """P[m, n, j] = Pbar_n^m(mu_j) for 0 <= m <= n <= N+1 (zero elsewhere)."""
    P = np.zeros((N + 1, N + 2, mu.size))
    for m in range(N + 1):
        for n in range(m, N + 2):
            norm = math.sqrt((2 * n + 1) * math.exp(math.lgamma(n - m + 1) - math.lgamma(n + m + 1)))
            P[m, n] = ((-1) ** m) * norm * lpmv(m, n, mu)
    return P


def hbar_table(N: int, mu: np.ndarray) -> np.ndarray:
    """H[m, n, j] = (1-mu^2) dPbar_n^m/dmu via (n+m) P_{n-1} - n mu P_n (unnormalised identity)."""
    H = np.zeros((N + 1, N + 2, mu.size))
    for m in range(N + 1):
        for n in range(m, N + 2):
            norm = math.sqrt((2 * n + 1) * math.exp(math.lgamma(n - m + 1) - math.lgamma(n + m + 1)))
            pnm1 = lpmv(m, n - 1, mu) if n - 1 >= m else 0.0 * mu
            H[m, n] = ((-1) ** m) * norm * ((n + m) * pnm1 - n * mu * lpmv(m, n, mu))
    return H


def lidx(n: int, m: int) -> int:
    return n * (n + 1) + m


def to_complex(N: int, w: np.ndarray) -> np.ndarray:
    """SPML real layout -> complex a[m, n] (m >= 0)."""
    a = np.zeros((N + 1, N + 1), dtype=complex)
    for n in range(N + 1):
        a[0, n] = w[lidx(n, 0)]
        for m in range(1, n + 1):
            a[m, n] = (w[lidx(n, m)] + 1j * w[lidx(n, -m)]) / math.sqrt(2.0)
    return a


def to_real(N: int, a: np.ndarray) -> np.ndarray:
    w = np.zeros((N + 1) ** 2)
    for n in range(N + 1):
        w[lidx(n, 0)] = a[0, n].real
        for m in range(1, n + 1):
            w[lidx(n, m)] = math.sqrt(2.0) * a[m, n].real
            w[lidx(n, -m)] = math.sqrt(2.0) * a[m, n].imag
    return w


class Direct:
    def __init__(self, I: int, J: int, N: int, radius: float):
        self.I, self.J, self.N, self.radius = I, J, N, radius
        self.mu, w2 = roots_legendre(J)          # ascending, sum 2
        self.w = w2 / 2.0                        # sum 1 (space_discretization.tex:205-209)
        self.lam = 2 * np.pi * np.arange(I) / I
        self.cos = np.sqrt(1 - self.mu ** 2)
        self.P = pbar_table(N, self.mu)
        self.H = hbar_table(N, self.mu)
        self.E = np.exp(1j * np.outer(np.arange(N + 1), self.lam))  # [m, i]

    # spectral (complex a[m,n], table T[m,n,j]) -> grid [j, i]
    def synth(self, a: np.ndarray, T: np.ndarray) -> np.ndarray:
        N = self.N
        G = np.einsum("mn,mnj->mj", a, T[:, : a.shape[1], :])  # G^m(mu_j)
        x = np.real(G[0][:, None] * self.E[0][None, :])
        for m in range(1, N + 1):
            x = x + 2.0 * np.real(G[m][:, None] * self.E[m][None, :])
        return x

    # grid [j, i] -> complex c[m, n] with table T, weights w_j * s_j
    def analyse(self, x: np.ndarray, T: np.ndarray, rowscale=None) -> np.ndarray:
        s = np.ones(self.J) if rowscale is None else rowscale
        G = (x * s[:, None]) @ np.conj(self.E).T / self.I  # [j, m]
        c = np.einsum("jm,mnj,j->mn", G, T[:, : self.N + 1, :], self.w)
        tri = np.tril(np.ones((self.N + 1, self.N + 1)), 0).T  # n >= m
        return c * tri

    def w_xy(self, x):
        return to_real(self.N, self.analyse(x, self.P))

    def xy_w(self, w):
        return self.synth(to_complex(self.N, w), self.P)

    def w_divlambda(self, x):
        c = self.analyse(x, self.P, 1.0 / (1.0 - self.mu ** 2))
        return to_real(self.N, 1j * np.arange(self.N + 1)[:, None] * c)

    def w_divmu(self, x):
        c = self.analyse(x, self.H, 1.0 / (1.0 - self.mu ** 2))
        return to_real(self.N, -c)

    def xy_gradlambda(self, w):
        a = to_complex(self.N, w)
        return self.synth(1j * np.arange(self.N + 1)[:, None] * a, self.P)

    def xy_gradmu(self, w):
        return self.synth(to_complex(self.N, w), self.H)

    def xy_gradlon(self, w):
        return self.xy_gradlambda(w) / self.cos[:, None]

    def xy_gradlat(self, w):
        return self.xy_gradmu(w) / self.cos[:, None]

    def laplainv(self, w):
        out = np.zeros_like(w)
        for n in range(1, self.N + 1):
            for m in range(-n, n + 1):
                out[lidx(n, m)] = -w[lidx(n, m)] / (n * (n + 1))
        return out

    def w_alpha(self, A, B):
        return (self.w_divlambda(A) + self.w_divmu(B)) / self.radius

    def xy_alpha(self, wA, wB):
        return (self.xy_gradlambda(wA) + self.xy_gradmu(wB)) / (self.radius * self.cos[:, None] ** 2)

    def vordiv2uv(self, vor, div):
        psi = self.laplainv(vor) * self.radius ** 2
        chi = self.laplainv(div) * self.radius ** 2
        return self.cos[:, None] * self.xy_alpha(chi, -psi), self.cos[:, None] * self.xy_alpha(psi, chi)

    def uv2vordiv(self, U, V):
        return self.w_alpha(V, -U), self.w_alpha(U, V)

    def avrlonlat(self, x):
        return float(np.sum(x * (2 * np.pi / self.I) * (2 * self.w)[:, None]) / (4 * np.pi))


def seeded_spectra(rng, N: int, nb: int, power: float) -> np.ndarray:
    """SPML-layout spectra with complex a_nm ~ N(0,1) (n+1)^-power, Im a_n0 = 0."""
    out = np.zeros((nb, (N + 1) ** 2))
    for b in range(nb):
        a = np.zeros((N + 1, N + 1), dtype=complex)
        for n in range(N + 1):
            amp = (n + 1.0) ** (-power)
            for m in range(n + 1):
                re, im = rng.standard_normal(2)
                a[m, n] = amp * (re + (1j * im if m > 0 else 0.0))
        out[b] = to_real(N, a)
    return out


def make(I: int, J: int, N: int, radius: float, nb: int, tag: str) -> str:
    rng = np.random.default_rng(SEED)
    d = Direct(I, J, N, radius)
    w = seeded_spectra(rng, N, nb, 1.5)
    w2 = seeded_spectra(rng, N, nb, 2.0)
    grid_rand = rng.standard_normal((nb, J, I))
    res = dict(I=I, J=J, N=N, radius=radius, seed=SEED, mu=d.mu, wgt=d.w,
               w=w, w2=w2, grid_rand=grid_rand)
    res["xy_w"] = np.stack([d.xy_w(x) for x in w])
    res["w_xy_rand"] = np.stack([d.w_xy(x) for x in grid_rand])
    res["gradlambda"] = np.stack([d.xy_gradlambda(x) for x in w])
    res["gradmu"] = np.stack([d.xy_gradmu(x) for x in w])
    res["gradlon"] = np.stack([d.xy_gradlon(x) for x in w])
    res["gradlat"] = np.stack([d.xy_gradlat(x) for x in w])
    # analysis-side derivative forms on band-limited products (U cos phi-like)
    A = res["xy_w"] * d.cos[None, :, None] ** 2
    B = np.stack([d.xy_w(x) for x in w2]) * d.cos[None, :, None] ** 2
    res["divA"], res["divB"] = A, B
    res["divlambda"] = np.stack([d.w_divlambda(x) for x in A])
    res["divmu"] = np.stack([d.w_divmu(x) for x in B])
    res["w_alpha"] = np.stack([d.w_alpha(a, b) for a, b in zip(A, B)])
    res["xy_alpha"] = np.stack([d.xy_alpha(a, b) for a, b in zip(w, w2)])
    uv = [d.vordiv2uv(a, b) for a, b in zip(w, w2)]
    res["U"] = np.stack([u for u, _ in uv])
    res["V"] = np.stack([v for _, v in uv])
    vd = [d.uv2vordiv(u * d.cos[:, None], v * d.cos[:, None]) for u, v in uv]
    res["vor"] = np.stack([a for a, _ in vd])
    res["div"] = np.stack([b for _, b in vd])
    res["avr"] = np.array([d.avrlonlat(x) for x in res["xy_w"]])
    path = os.path.join(HERE, f"sht_{tag}.npz")
    np.savez_compressed(path, **res)
    return path


def main():
    print(make(64, 32, 21, 6.371e6, 2, "T21"))
    print(make(32, 16, 10, 1.0, 3, "T10"))
    print(make(48, 24, 15, 1.0, 2, "T15_I48"))  # non-power-of-two longitude count


if __name__ == "__main__":
    main()
