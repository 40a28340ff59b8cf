"""Synthetic inputs with the shapes of the benchmark workloads.

The reference ships no benchmark inputs; the workloads are defined by the
run configurations this package is measured on.  The linear power spectrum is
P(k) = A k^ns T_BBKS(k/Gamma)^2 with Gamma = Omega_m h and no baryon term
(Bardeen, Bond, Kaiser & Szalay 1986), normalised to sigma_8 at z = 0 with a
top-hat of radius 8 Mpc/h, and tabulated at log-spaced k.  BBKS has no BAO
wiggles, so the non-wiggle spectrum equals P(k) and BAO enhancement is a no-op
(libEZmock/EZmock/linear_pk.c:140-155 with Pnw == P).  ``wiggle_pk`` adds a
project-defined damped sinusoid for exercising the BAO code path.
"""
import math
from dataclasses import dataclass, field

import numpy as np


def bbks_transfer(k, gamma):
    q = np.asarray(k, np.float64) / gamma
    return (np.log1p(2.34 * q) / (2.34 * q) *
            (1 + 3.89 * q + (16.1 * q) ** 2 + (5.46 * q) ** 3 + (6.71 * q) ** 4) ** -0.25)


def _sigma_r(kk, pk, R):
    x = kk * R
    w = 3 * (np.sin(x) - x * np.cos(x)) / x ** 3
    integrand = kk ** 3 * pk * w * w / (2 * math.pi ** 2)      # d ln k
    lnk = np.log(kk)
    return math.sqrt(np.trapezoid(integrand, lnk))


def bbks_pk(omega_m=0.31, h=0.676, ns=0.965, sigma8=0.81, n=1000, kmin=1e-4, kmax=10.0):
    """(k, P) with P(k) normalised to sigma_8 at z = 0 (k in h/Mpc)."""
    gamma = omega_m * h
    kk = np.logspace(-6, 4, 200001)
    shape = kk ** ns * bbks_transfer(kk, gamma) ** 2
    amp = (sigma8 / _sigma_r(kk, shape, 8.0)) ** 2
    k = np.logspace(math.log10(kmin), math.log10(kmax), n)
    return k, amp * k ** ns * bbks_transfer(k, gamma) ** 2


def wiggle_pk(k, pnw, amp=0.05, r_s=105.0, k_silk=0.2):
    """A smooth spectrum with a damped BAO-like sinusoid (project-defined)."""
    return pnw * (1 + amp * np.sin(k * r_s) * np.exp(-(k / k_silk) ** 2))


def rsd_factor(z, omega_m):
    """(1+z) / (100 E(z)) in Mpc/h per km/s for flat LCDM."""
    ez = math.sqrt(omega_m * (1 + z) ** 3 + 1 - omega_m)
    return (1 + z) / (100 * ez)


@dataclass
class MockConfig:
    name: str
    Ng: int
    Lbox: float
    seed: int
    n_tracer: float             # number density, (h/Mpc)^3
    rho_c: float
    rho_exp: float
    pdf_base: float
    sigma_v: float
    rng: int = 1                # 1 = MT19937 (reference default), 0 = MRG32k3a
    z: float = 0.8
    omega_m: float = 0.31
    populations: list = field(default_factory=list)

    @property
    def nexp(self):
        return int(round(self.n_tracer * self.Lbox ** 3))

    def params(self):
        return [self.rho_c, self.rho_exp, self.pdf_base, self.sigma_v]

    def population_list(self):
        """(n_tracer, rho_c, rho_exp, pdf_base, sigma_v) of every population
        drawn from one field (the base parameters when none are listed)."""
        return [tuple(p) for p in self.populations] or [(self.n_tracer, *self.params())]


CONFIGS = {
    # Plain EZmock at 128^3, box 1000 Mpc/h, seed 1 (parity case).
    "plain128": MockConfig("plain128", 128, 1000.0, 1, 3e-4, 0.6, 15.0, 0.35, 300.0),
    # Single mock at 512^3, box 2500 Mpc/h (the bench workload).
    "single512": MockConfig("single512", 512, 2500.0, 1, 2e-4, 0.8, 20.0, 0.3, 400.0),
    # The 512^3 mock at half the size and box (same cell size and tracer
    # density): the profiling case, fields still larger than the 126 MB L2.
    "single256": MockConfig("single256", 256, 1250.0, 1, 2e-4, 0.8, 20.0, 0.3, 400.0),
    # 1024^3, box 5000 Mpc/h, one field populated three times.
    "multi1024": MockConfig(
        "multi1024", 1024, 5000.0, 1, 2e-4, 0.5, 10.0, 0.3, 250.0,
        populations=[(2e-4, 0.5, 10.0, 0.3, 250.0), (1e-4, 0.9, 20.0, 0.4, 350.0),
                     (2e-5, 1.3, 30.0, 0.5, 450.0)]),
}
