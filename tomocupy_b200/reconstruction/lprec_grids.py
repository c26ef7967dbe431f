"""Log-polar grid geometry of the lprec backprojector (host setup).

Restates ``create_gl``, ``getparameters``, ``osg``, ``splineB3``,
``create_adj`` and ``fzeta_loop_weights_adj``
(src/tomocupy/reconstruction/lprec.py:82-289) with NumPy standing in for
CuPy; the operation order and dtypes are kept so the float32 grids and the
complex64 kernel match the reference's.  Three angular spans of width
beta = pi/3 are mapped to log-polar coordinates (theta, rho) with
ntheta = 2^round(log2 nproj) and nrho = 2 * 2^round(log2 n).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Pgl:
    Nspan: int
    N: int
    Nproj: int
    Ntheta: int
    Nrho: int
    proj: np.ndarray
    thsp: np.ndarray
    rhosp: np.ndarray
    aR: float
    beta: float
    am: float
    g: float
    B3com: np.ndarray


@dataclass
class Padj:
    fZ: np.ndarray
    lp2p1: np.ndarray
    lp2p2: np.ndarray
    lp2p1w: np.ndarray
    lp2p2w: np.ndarray
    C2lp1: np.ndarray
    C2lp2: np.ndarray
    cids: np.ndarray
    lpids: np.ndarray
    wids: np.ndarray


def getparameters(beta, dtheta, ds, N, Nproj, Ntheta, Nrho):
    aR = np.sin(beta / 2) / (1 + np.sin(beta / 2))
    am = (np.cos(beta / 2) - np.sin(beta / 2)) / (1 + np.sin(beta / 2))
    g = osg(aR, beta / 2)
    dtheta = (2 * beta) / Ntheta
    drho = (g - np.log(am)) / Nrho
    return dtheta, drho, aR, am, g


def osg(aR, theta):
    t = np.linspace(-np.pi / 2, np.pi / 2, 1000)
    w = aR * np.cos(t) + (1 - aR) + 1j * aR * np.sin(t)
    return float(np.max(np.log(abs(w)) + np.log(np.cos(theta - np.arctan2(w.imag, w.real)))))


def splineB3(x2, r):
    sizex = len(x2)
    x2 = x2 - (x2[-1] + x2[0]) / 2
    stepx = x2[1] - x2[0]
    ri = int(np.ceil(2 * r))
    r = r * stepx
    x2c = x2[int(np.ceil((sizex + 1) / 2.0)) - 1]
    x = x2[int(np.ceil((sizex + 1) / 2.0) - ri - 1):int(np.ceil((sizex + 1) / 2.0) + ri)]
    d = np.abs(x - x2c) / r
    B3 = x * 0
    for ix in range(-ri, ri + 1):
        idx = ix + ri
        if d[idx] < 1:
            B3[idx] = (3 * d[idx] ** 3 - 6 * d[idx] ** 2 + 4) / 6
        elif d[idx] < 2:
            B3[idx] = (-d[idx] ** 3 + 6 * d[idx] ** 2 - 12 * d[idx] + 8) / 6
    B3f = x2 * 0
    B3f[int(np.ceil((sizex + 1) / 2.0) - ri - 1):int(np.ceil((sizex + 1) / 2.0) + ri)] = B3
    return B3f


def create_gl(N, Nproj, Ntheta, Nrho) -> Pgl:
    Nspan = 3
    beta = np.pi / Nspan
    proj = np.arange(0, Nproj) * np.pi / Nproj - beta / 2
    dtheta, drho, aR, am, g = getparameters(beta, proj[1] - proj[0], 2.0 / (N - 1), N, Nproj,
                                            Ntheta, Nrho)
    thsp = (np.arange(-Ntheta / 2, Ntheta / 2) * np.float32(dtheta)).astype("float32")
    rhosp = (np.arange(-Nrho, 0) * drho).astype("float32")
    B3th = splineB3(thsp, 1)
    B3th = np.fft.fft(np.fft.ifftshift(B3th))
    B3rho = splineB3(rhosp, 1)
    B3rho = np.fft.fft(np.fft.ifftshift(B3rho))
    B3com = np.outer(B3rho, B3th)
    return Pgl(Nspan, N, Nproj, Ntheta, Nrho, proj, thsp, rhosp, aR, beta, am, g, B3com)


def fzeta_loop_weights_adj(Ntheta, Nrho, betas, rhos, a, osthlarge):
    Nthetalarge = osthlarge * Ntheta
    krho = np.linspace(-Nrho / 2, Nrho / 2, Nrho, endpoint=False, dtype="float32")
    thsplarge = np.linspace(-1 / 2, 1 / 2, Nthetalarge, endpoint=False, dtype="float32") * betas
    correcting = 1 + np.array([-216254335, 679543284, -1412947389, 2415881496, -3103579086,
                               2939942400, -2023224114, 984515304, -321455811, 63253516,
                               -5675265], dtype="float64") / 958003200.0
    correcting[0] = 2 * (correcting[0] - 0.5)
    h = np.ones(Nthetalarge, dtype="float32")
    h[0] *= correcting[0]
    idx = np.arange(1, len(correcting))
    h[idx] *= correcting[idx]
    h[-idx] *= correcting[idx]
    s = (1 - 2 * (np.arange(1, Nthetalarge + 1) % 2)).astype("float32")
    h *= s
    log_cos = np.log(np.cos(thsplarge)).astype("float32")
    phases = np.outer(krho, log_cos) * np.float32(2 * np.pi / rhos)
    if a != 0:
        phases -= np.float32(a) * log_cos[None, :]
    fcosa = (np.cos(phases) + 1j * np.sin(phases)).astype("complex64")
    fZ = (s[None, :] * np.fft.fft(h[None, :] * fcosa, axis=1)).astype("complex64")
    fZ = fZ[:, Nthetalarge // 2 - Ntheta // 2:Nthetalarge // 2 + Ntheta // 2] * float(
        thsplarge[1] - thsplarge[0])
    fZ[0] = 0
    fZ[:, 0] = 0
    return fZ


def create_adj(P: Pgl) -> Padj:
    fZ = np.fft.fftshift(fzeta_loop_weights_adj(P.Ntheta, P.Nrho, 2 * P.beta,
                                                float(P.g) - float(np.log(P.am)), 0, 4))
    fZ = np.ascontiguousarray(fZ[:, :P.Ntheta // 2 + 1] / (P.B3com[:, :P.Ntheta // 2 + 1]))
    const = np.float32((P.N + 1) * (P.N - 1) / P.N ** 2 / 2 / np.sqrt(2) * np.pi / 6 * 0.86 * 4)
    fZ = (fZ * const).astype("complex64")
    if bool(np.any(np.isnan(fZ))):
        b = P.B3com[:, :P.Ntheta // 2 + 1]
        raise RuntimeError(f"fZ has NaN after division. B3com range: "
                           f"[{float(abs(b).min()):.3e}, {float(abs(b).max()):.3e}]")
    # (C2lp1, C2lp2): Cartesian -> log-polar
    x1, x2 = np.meshgrid(np.linspace(-1, 1, P.N, dtype="float32"),
                         np.linspace(-1, 1, P.N, dtype="float32"))
    x1 = x1.flatten()
    x2 = x2.flatten()
    x2 = x2 * (-1)  # adjust for tomocupy
    x1 -= 1 / P.N
    x2 -= 1 / P.N
    cids = np.where(x1 ** 2 + x2 ** 2 <= 1)[0].astype("int32")
    C2lp1 = np.zeros([P.Nspan, len(cids)], dtype="float32")
    C2lp2 = np.zeros([P.Nspan, len(cids)], dtype="float32")
    for k in range(P.Nspan):
        z1 = P.aR * (x1[cids] * np.cos(k * P.beta + P.beta / 2) + x2[cids] *
                     np.sin(k * P.beta + P.beta / 2)) + (1 - P.aR)
        z2 = P.aR * (-x1[cids] * np.sin(k * P.beta + P.beta / 2) +
                     x2[cids] * np.cos(k * P.beta + P.beta / 2))
        C2lp1[k] = np.arctan2(z2, z1)
        C2lp2[k] = np.log(np.sqrt(z1 ** 2 + z2 ** 2))
    # (lp2p1, lp2p2): log-polar -> polar
    z1, z2 = np.meshgrid(P.thsp, np.exp(P.rhosp))
    z1 = z1.flatten()
    z2 = z2.flatten()
    z2n = z2 - (1 - P.aR) * np.cos(z1)
    z2n = z2n / P.aR
    lpids = np.where((z1 >= -P.beta / 2) & (z1 < P.beta / 2) & (abs(z2n) <= 1))[0].astype("int32")
    lp2p1 = np.zeros([P.Nspan, len(lpids)], dtype="float32")
    lp2p2 = np.zeros([P.Nspan, len(lpids)], dtype="float32")
    for k in range(P.Nspan):
        lp2p1[k] = z1[lpids] + k * P.beta
        lp2p2[k] = z2n[lpids]
    # (lp2p1w, lp2p2w): log-polar -> polar, wrapped points
    log_z2 = np.log(z2)
    am_eg = float(P.am) * np.exp(-P.g)
    eg_am = np.exp(P.g) / float(P.am)
    wids = np.where(log_z2 > +P.g)[0].astype("int32")
    z2n = z2[wids] * am_eg - (1 - P.aR) * np.cos(z1[wids])
    z2n = z2n / P.aR
    lpidsw = np.where((z1[wids] >= -P.beta / 2) & (z1[wids] < P.beta / 2) & (abs(z2n) <= 1))[0]
    wids2 = np.where(log_z2 < float(np.log(P.am)) - P.g +
                     float(P.rhosp[1] - P.rhosp[0]))[0].astype("int32")
    z2n2 = z2[wids2] * eg_am - (1 - P.aR) * np.cos(z1[wids2])
    z2n2 = z2n2 / P.aR
    lpidsw2 = np.where((z1[wids2] >= -P.beta / 2) & (z1[wids2] < P.beta / 2) &
                       (abs(z2n2) <= 1))[0]
    lp2p1w = np.zeros([P.Nspan, len(lpidsw) + len(lpidsw2)], dtype="float32")
    lp2p2w = np.zeros([P.Nspan, len(lpidsw) + len(lpidsw2)], dtype="float32")
    for k in range(P.Nspan):
        lp2p1w[k] = z1[np.concatenate((lpidsw, lpidsw2))] + k * P.beta
        lp2p2w[k] = np.concatenate((z2n[lpidsw], z2n2[lpidsw2]))
    wids = np.concatenate((wids[lpidsw], wids2[lpidsw2])).astype("int32")
    # pids: polar indices of each span
    pids = [np.where((P.proj >= k * P.beta - P.beta / 2) & (P.proj < k * P.beta + P.beta / 2))[0]
            for k in range(P.Nspan)]
    proj0 = [P.proj[pids[k][0]] for k in range(P.Nspan)]
    projl = [P.proj[pids[k][-1]] - P.proj[pids[k][0]] for k in range(P.Nspan)]
    projp = (P.Nproj - 1) / (proj0[P.Nspan - 1] + projl[P.Nspan - 1] - proj0[0])
    for k in range(P.Nspan):
        lp2p1[k] = (lp2p1[k] - proj0[k]) / projl[k] * (len(pids[k]) - 1) + (proj0[k] - proj0[0]) * projp
        lp2p1w[k] = (lp2p1w[k] - proj0[k]) / projl[k] * (len(pids[k]) - 1) + (proj0[k] - proj0[0]) * projp
        lp2p2[k] = (lp2p2[k] + 1) / 2 * (P.N - 1)
        lp2p2w[k] = (lp2p2w[k] + 1) / 2 * (P.N - 1)
        C2lp1[k] = (C2lp1[k] - P.thsp[0]) / (P.thsp[-1] - P.thsp[0]) * (P.Ntheta - 1)
        C2lp2[k] = (C2lp2[k] - P.rhosp[0]) / (P.rhosp[-1] - P.rhosp[0]) * (P.Nrho - 1)
    return Padj(fZ, lp2p1, lp2p2, lp2p1w, lp2p2w, C2lp1, C2lp2, cids, lpids, wids)


def lp_sizes(n: int, nproj: int):
    """ntheta, nrho of lprec.py:300-301."""
    ntheta = 2 ** int(np.round(np.log2(nproj)))
    nrho = 2 * 2 ** int(np.round(np.log2(n)))
    return ntheta, nrho


def check_angles(theta, nproj) -> None:
    """lprec works only with equally spaced angles in [0, pi) (lprec.py:295-299)."""
    nproj_test = int(np.round(np.pi / (float(theta[1]) - float(theta[0]))))
    if nproj != nproj_test:
        raise ValueError("lprec method works only with equally spaced angles in the interval "
                         f"[0,180) deg. (nproj={nproj}, pi/dtheta={nproj_test})")
