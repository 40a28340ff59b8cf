"""Numpy restatement of the clustering estimators (test infrastructure only).

The reference has no estimator source: it calls external programs
(example/fit/pyclustering.py:173-186; POWSPEC configured by
example/fit/conf/powspec.conf: cubic box, CIC, grid interlacing, multipoles
0 and 2, linear bins).  This file states the standard periodic-box estimator
that the GPU implementation follows, in float64 with numpy's FFT, so the GPU
results can be checked on the same catalogue.  Parity unpinned: no reference
output exists to pin it; tests/test_oracle_pkest.py checks it against mode
counts, a plane-wave catalogue and hand counts instead.
"""
import numpy as np


def redshift_z(z, vz, rsd_fac, L):
    """z + rsd_fac vz wrapped into [0, L) (save_res.c:147-158)."""
    z = np.asarray(z, np.float64)
    if vz is None or rsd_fac == 0:
        return z
    v = z + rsd_fac * np.asarray(vz, np.float64)
    return np.where(v < 0, v + L, np.where(v >= L, v - L, v))


def grid_coord(p, L, Ng):
    u = np.asarray(p, np.float64) * (Ng / L)
    u = u - np.floor(u / Ng) * Ng
    u = np.where(u >= Ng, u - Ng, u)
    return np.where(u < 0, 0.0, u)


def cic_grid(pos, L, Ng, shift):
    """CIC counts on grid points (i + shift) h."""
    g = np.zeros((Ng, Ng, Ng))
    u = [grid_coord(p, L, Ng) - shift for p in pos]
    i0, w1 = [], []
    for d in range(3):
        f = np.floor(u[d])
        w1.append(u[d] - f)
        i0.append(f.astype(np.int64) % Ng)
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                w = ((w1[0] if a else 1 - w1[0]) * (w1[1] if b else 1 - w1[1]) *
                     (w1[2] if c else 1 - w1[2]))
                np.add.at(g, ((i0[0] + a) % Ng, (i0[1] + b) % Ng, (i0[2] + c) % Ng), w)
    return g


def powspec(x, y, z, L, Ng, interlace=True, kmin=0.0, kmax=0.3, nbin=30, vz=None,
            rsd_fac=0.0):
    """k_mean, nmodes, P0, P2 per linear |k| bin (see ez_pk.cu)."""
    pos = [x, y, redshift_z(z, vz, rsd_fac, L)]
    n = len(pos[0])
    F = np.fft.rfftn(cic_grid(pos, L, Ng, 0.0))
    f = np.fft.fftfreq(Ng, 1.0 / Ng).round().astype(np.int64)      # signed integers
    kk = np.arange(Ng // 2 + 1)
    ki, kj, kz = np.meshgrid(f, f, kk, indexing="ij")
    if interlace:
        F1 = np.fft.rfftn(cic_grid(pos, L, Ng, 0.5))
        F = 0.5 * (F + np.exp(-1j * np.pi * (ki + kj + kz) / Ng) * F1)
    W = (np.sinc(ki / Ng) * np.sinc(kj / Ng) * np.sinc(kz / Ng)) ** 2
    F = F / W
    V = L ** 3
    P = np.abs(F) ** 2 * V / float(n) ** 2
    q2 = ki ** 2 + kj ** 2 + kz ** 2
    kmag = 2 * np.pi / L * np.sqrt(q2)
    dk = (kmax - kmin) / nbin
    b = np.floor((kmag - kmin) / dk)
    ok = (q2 > 0) & (b >= 0) & (b < nbin)
    m = np.where((kz == 0) | (kz == Ng // 2), 1.0, 2.0)
    mu2 = np.where(q2 > 0, kz ** 2 / np.maximum(q2, 1), 0.0)
    L2 = 1.5 * mu2 - 0.5
    bi = b[ok].astype(np.int64)
    nm = np.bincount(bi, m[ok], nbin)
    sk = np.bincount(bi, (m * kmag)[ok], nbin)
    sp = np.bincount(bi, (m * P)[ok], nbin)
    s2 = np.bincount(bi, (m * P * L2)[ok], nbin)
    with np.errstate(invalid="ignore", divide="ignore"):
        kmean = np.where(nm > 0, sk / nm, kmin + (np.arange(nbin) + 0.5) * dk)
        p0 = np.where(nm > 0, sp / nm - V / n, 0.0)
        p2 = np.where(nm > 0, 5 * s2 / nm, 0.0)
    return {"k_mean": kmean, "nmodes": nm, "P0": p0, "P2": p2, "shot": V / n}


def cic_pdf(x, y, z, L, Ng, nbin=32, vz=None, rsd_fac=0.0):
    """Fraction of cells holding c tracers (last bin: c >= nbin - 1)."""
    pos = [x, y, redshift_z(z, vz, rsd_fac, L)]
    c = [np.minimum(grid_coord(p, L, Ng).astype(np.int64), Ng - 1) for p in pos]
    cnt = np.bincount((c[0] * Ng + c[1]) * Ng + c[2], minlength=Ng ** 3)
    h = np.bincount(np.minimum(cnt, nbin - 1), minlength=nbin)
    return h / float(Ng ** 3)
