"""Known answers used to pin the oracle and the GPU solver (test helpers).

* Mie series of a PEC sphere (bistatic RCS), written from the published
  series (Bohren & Huffman, "Absorption and Scattering of Light by Small
  Particles", ch. 4; PEC limit): a_n = [x j_n(x)]' / [x h_n(x)]',
  b_n = j_n(x) / h_n(x), S1 = sum (2n+1)/(n(n+1)) (a_n pi_n + b_n tau_n),
  S2 = sum (2n+1)/(n(n+1)) (a_n tau_n + b_n pi_n), sigma = 4 pi |S|^2 / k^2.
* RCS of an RWG current: the one-point far-field sum of
  EFIEMatrix::getRCS_OnePointQuadrature (src/EFIEMatrix.cpp:916-930) with
  the centroid currents of getJAtCentroids (:1100-1130).
"""
from __future__ import annotations

import numpy as np
from scipy import special


def mie_pec_rcs(ka: float, k: float, theta: np.ndarray, phi: float) -> np.ndarray:
    x = ka
    nmax = int(x + 4 * x ** (1 / 3) + 10)
    n = np.arange(1, nmax + 1)
    jn = special.spherical_jn(n, x)
    jnp = special.spherical_jn(n, x, derivative=True)
    yn = special.spherical_yn(n, x)
    ynp = special.spherical_yn(n, x, derivative=True)
    hn = jn + 1j * yn
    hnp = jnp + 1j * ynp
    a = (jn + x * jnp) / (hn + x * hnp)  # [x j_n]' / [x h_n]'
    b = jn / hn
    mu = np.cos(theta)
    out = np.zeros_like(theta, dtype=float)
    for t, m in enumerate(mu):
        pi = np.zeros(nmax + 1)
        tau = np.zeros(nmax + 1)
        pi[1] = 1.0
        if nmax >= 2:
            pi[2] = 3 * m
        for q in range(3, nmax + 1):
            pi[q] = (2 * q - 1) / (q - 1) * m * pi[q - 1] - q / (q - 1) * pi[q - 2]
        for q in range(1, nmax + 1):
            tau[q] = q * m * pi[q] - (q + 1) * pi[q - 1]
        c = (2 * n + 1) / (n * (n + 1))
        S1 = np.sum(c * (a * pi[1:] + b * tau[1:]))
        S2 = np.sum(c * (a * tau[1:] + b * pi[1:]))
        out[t] = 4 * np.pi / k ** 2 * (abs(S2) ** 2 * np.cos(phi) ** 2 + abs(S1) ** 2 * np.sin(phi) ** 2)
    return out


def centroid_currents(mesh, rwg: np.ndarray, length: np.ndarray, coeff: np.ndarray) -> np.ndarray:
    """J at triangle centroids, EFIEMatrix::getJAtCentroids (src/EFIEMatrix.cpp:1100-1130).
    rwg rows: (n1, n2, t+, t-, free+, free-) with one-based node ids."""
    nodes = np.vstack([np.zeros((1, 3)), mesh.nodes])
    tri = mesh.tris
    cen = nodes[tri].mean(axis=1)
    v = nodes[tri]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    J = np.zeros((len(tri), 3), dtype=np.complex128)
    tp, tm, fp, fm = rwg[:, 2], rwg[:, 3], rwg[:, 4], rwg[:, 5]
    rp = cen[tp] - nodes[fp]
    rm = cen[tm] - nodes[fm]
    np.add.at(J, tp, (coeff * length / 2 / area[tp])[:, None] * rp)
    np.add.at(J, tm, -(coeff * length / 2 / area[tm])[:, None] * rm)
    return J, cen, area


def rcs_one_point(J: np.ndarray, cen: np.ndarray, area: np.ndarray, k: float, theta: np.ndarray,
                  phi: float) -> np.ndarray:
    """Far-field RCS of centroid currents (sign convention exp(+i k.r) as the reference)."""
    eta = 377.0
    out = []
    for th in theta:
        kv = k * np.array([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)])
        ph = np.exp(1j * cen @ kv) * area
        st = np.sum((J[:, 0] * np.cos(th) * np.cos(phi) + J[:, 1] * np.cos(th) * np.sin(phi)
                     - J[:, 2] * np.sin(th)) * ph)
        sp = np.sum((-J[:, 0] * np.sin(phi) + J[:, 1] * np.cos(phi)) * ph)
        out.append(k * k / (4 * np.pi) * eta ** 2 * (abs(st) ** 2 + abs(sp) ** 2))
    return np.asarray(out)
