"""GPU parity on the benchmark configurations themselves, against the
reference's own libEZmock build (oracle/_ref: its unmodified sources,
OpenMP) on the same seed and parameters.

* 128^3 FP64 (box 1000 Mpc/h, seed 1, BBKS P(k), z = 0.8; rho_c 0.6,
  rho_exp 15, pdf_base 0.35, sigma_v 300 km/s, n = 3e-4 (h/Mpc)^3, RSD along
  z): psi and rho within 1e-12 of the reference, identical catalogue size,
  per-cell counts and positions, velocities and redshift-space z within
  1e-9 of the largest speed.
* 512^3 FP64 (box 2500 Mpc/h; rho_c 0.8, rho_exp 20, pdf_base 0.3,
  sigma_v 400 km/s, n = 2e-4): the same bar for the FP64 GPU mode.
* 512^3 FP32 production mode against the FP64 GPU mode over four seeds: the
  stated field error, the count of cells whose side of rho_c differs, and
  tracer P0/P2 in 40 bins over 0.005-0.3 h/Mpc.  The bias Gaussians are
  indexed by a cell's rank among the valid cells (rho >= rho_c,
  libEZmock/EZmock/pop_tracer.c:233-237), so one cell that changes side
  shifts the Gaussians of every later valid cell and the two catalogues
  become different draws of the bias noise on the same density field (the
  reference's own FP32 build behaves the same).  Tolerances: the band power
  over all 40 bins (mode-weighted P0, and P2 relative to it), averaged over
  the four seeds, within 0.5%, and within 1% for every seed (one seed's
  difference is a draw of the tracer-sampling noise, about 0.3% for this
  band); per bin, the seed-averaged relative P0 difference within 6 standard
  deviations of the sampling noise of one bin (its measured scatter over the
  40 bins and 4 seeds is printed).
"""
import numpy as np
import pytest

from ezmock_b200 import EZmock
from ezmock_b200.workloads import bbks_pk
from oracle.pyoracle import RefLib

from conftest import has_ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_ref(), reason="oracle/_ref not built")]

TOL64 = 1e-12
Z_OUT, OMEGA_M = 0.8, 0.31


def relmax(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def cell_index(x, y, z, Ng, L):
    gs = L / Ng
    i = [np.floor(np.asarray(a, np.float64) / gs + 0.5).astype(np.int64) % Ng for a in (x, y, z)]
    return (i[0] * Ng + i[1]) * Ng + i[2]


def rsd_factor(z, Om):
    """(1+z) / (100 E(z)) in Mpc/h per km/s, flat LCDM."""
    return (1 + z) / (100 * np.sqrt(Om * (1 + z) ** 3 + 1 - Om))


def gpu_mock(prec, Ng, L, seed):
    k, P = bbks_pk()
    m = EZmock(Lbox=L, Ngrid=Ng, rng=1, seed=seed, prec=prec)
    m.eval_growth_params(Z_OUT, OMEGA_M)
    m.setup_linear_pk(k, P)
    m.create_dens_field_from_ic()
    return m


def ref_mock(Ng, L, seed):
    k, P = bbks_pk()
    R = RefLib(64, nthread=0)
    r = R.new(L, Ng, 1, seed)
    r.eval_growth(Z_OUT, OMEGA_M)
    r.setup_pk(k, P)
    r.create()
    return r


def check_against_reference(Ng, L, seed, params, n):
    nexp = int(round(n * L ** 3))
    r = ref_mock(Ng, L, seed)
    m = gpu_mock(64, Ng, L, seed)
    err = [relmax(m.field(d), r.field(d)) for d in range(4)]
    print(f"{Ng}^3 FP64 field error vs reference: psi {err[0]:.2e} {err[1]:.2e} "
          f"{err[2]:.2e}, rho {err[3]:.2e}")
    assert max(err) <= TOL64
    ref = r.populate(params, nexp)
    cat = m.populate_tracer(*params, nexp)
    print(f"{Ng}^3 FP64 catalogue: {len(cat[0])} tracers (reference {len(ref[0])})")
    assert len(cat[0]) == len(ref[0])
    ci, cr = cell_index(*cat[:3], Ng, L), cell_index(*ref[:3], Ng, L)
    assert np.array_equal(np.bincount(ci, minlength=Ng ** 3), np.bincount(cr, minlength=Ng ** 3))
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])
    vmax = max(float(np.abs(ref[a]).max()) for a in range(3, 6))
    dv = max(float(np.abs(cat[a] - ref[a]).max()) for a in range(3, 6))
    print(f"{Ng}^3 FP64 velocities: max difference {dv:.3e} of max |v| {vmax:.1f}")
    assert dv <= 1e-9 * vmax
    # redshift-space z along the line of sight (save_res.c:147-158)
    f = rsd_factor(Z_OUT, OMEGA_M)
    zs = [np.mod(c[2] + f * c[5], L) for c in (cat, ref)]
    assert np.abs(zs[0] - zs[1]).max() <= 1e-9 * vmax * f + 1e-12 * L
    return m, r


def test_config_128_fp64():
    """128^3, box 1000 Mpc/h, seed 1: the FP64 GPU mode against the
    reference's FP64 build."""
    check_against_reference(128, 1000.0, 1, [0.6, 15.0, 0.35, 300.0], 3e-4)


def test_config_512_fp64():
    """512^3, box 2500 Mpc/h, seed 1: the FP64 GPU mode against the
    reference's FP64 build (all host threads)."""
    check_against_reference(512, 2500.0, 1, [0.8, 20.0, 0.3, 400.0], 2e-4)


def test_config_512_fp32_vs_fp64():
    Ng, L = 512, 2500.0
    params = [0.8, 20.0, 0.3, 400.0]
    nexp = int(round(2e-4 * L ** 3))
    f = rsd_factor(Z_OUT, OMEGA_M)
    nbin, kmin, kmax = 40, 0.005, 0.3
    rows, rel0 = [], []
    nmodes = None
    for seed in (1, 2, 3, 4):
        m64 = gpu_mock(64, Ng, L, seed)
        rho64 = m64.field(3)
        cat64 = m64.populate_tracer(*params, nexp)
        m32 = gpu_mock(32, Ng, L, seed)
        rho32 = m32.field(3)
        cat32 = m32.populate_tracer(*params, nexp)
        err = relmax(rho32, rho64)
        assert err <= 1e-5                        # stated FP32 field error
        tol = err * float(np.abs(rho64).max())
        near = int(np.count_nonzero(np.abs(rho64 - params[0]) <= tol))
        cross = int(np.count_nonzero((rho32 >= np.float32(params[0])) != (rho64 >= params[0])))
        n64 = np.bincount(cell_index(*cat64[:3], Ng, L), minlength=Ng ** 3)
        n32 = np.bincount(cell_index(*cat32[:3], Ng, L), minlength=Ng ** 3)
        occ = int(np.count_nonzero(n64))
        diff = int(np.count_nonzero((n64 != n32) & (n64 > 0)))
        del rho32, rho64, n32, n64
        p64 = m64.powspec(cat=(cat64[0], cat64[1], cat64[2], cat64[5]), rsd_fac=f, ngrid=256,
                          kmin=kmin, kmax=kmax, nbin=nbin)
        p32 = m64.powspec(cat=(cat32[0], cat32[1], cat32[2], cat32[5]), rsd_fac=f, ngrid=256,
                          kmin=kmin, kmax=kmax, nbin=nbin)
        has = p64["nmodes"] > 0
        nmodes = p64["nmodes"]
        band0 = np.sum(nmodes * (p32["P0"] - p64["P0"])) / np.sum(nmodes * p64["P0"])
        band2 = np.sum(nmodes * (p32["P2"] - p64["P2"])) / np.sum(nmodes * p64["P0"])
        r0 = np.where(has, (p32["P0"] - p64["P0"]) / np.where(has, p64["P0"], 1), 0)
        rel0.append(r0)
        rows.append((seed, err, near, cross, occ, diff, len(cat32[0]), len(cat64[0]),
                     float(np.median(np.abs(r0[has]))), float(np.abs(r0[has]).max()),
                     band0, band2))
        del m32, m64
    print("\nseed | rho error | cells within it of rho_c | cells changing side | "
          "occupied cells | with other counts | n32 | n64 | P0 per bin median / max | "
          "band P0 | band P2")
    for r in rows:
        print(f"{r[0]} | {r[1]:.2e} | {r[2]} | {r[3]} | {r[4]} | {r[5]} | {r[6]} | {r[7]} | "
              f"{100 * r[8]:.2f}% / {100 * r[9]:.1f}% | {100 * r[10]:+.3f}% | {100 * r[11]:+.3f}%")
    mean0 = float(np.mean([r[10] for r in rows]))
    mean2 = float(np.mean([r[11] for r in rows]))
    print(f"band power over seeds: P0 {100 * mean0:+.3f}%, P2 {100 * mean2:+.3f}% of P0")
    assert abs(mean0) <= 5e-3 and abs(mean2) <= 5e-3
    for r in rows:
        assert abs(r[10]) <= 1e-2 and abs(r[11]) <= 1e-2
    rel0 = np.array(rel0)
    has = nmodes > 0
    bins0 = rel0.mean(axis=0)
    # per-bin scatter of one seed's relative difference, from the 4 x 40
    # values scaled by the bin's mode count (the noise goes as 1/sqrt(modes))
    z = rel0[:, has] * np.sqrt(nmodes[has])
    sigma_unit = float(np.sqrt(np.mean(z ** 2)))
    sig_mean = sigma_unit / np.sqrt(nmodes[has]) / np.sqrt(rel0.shape[0])
    worst = float(np.abs(bins0[has] / sig_mean).max())
    print(f"per-bin scatter: {sigma_unit:.3f} / sqrt(modes); seed-averaged P0 difference at "
          f"most {worst:.2f} standard deviations; mean over bins "
          f"{100 * float(bins0[has].mean()):.3f}%")
    assert worst <= 6.0
