"""The numpy restatement of the clustering estimators (oracle/pkest.py) on
cases with known answers."""
import numpy as np

from oracle import pkest


def test_mode_counts_match_full_grid():
    Ng, L, nbin, kmax = 16, 100.0, 7, 0.5
    rng = np.random.default_rng(1)
    x, y, z = rng.uniform(0, L, (3, 200))
    r = pkest.powspec(x, y, z, L, Ng, interlace=False, kmin=0.0, kmax=kmax, nbin=nbin)
    f = np.fft.fftfreq(Ng, 1.0 / Ng)
    a, b, c = np.meshgrid(f, f, f, indexing="ij")
    kmag = 2 * np.pi / L * np.sqrt(a ** 2 + b ** 2 + c ** 2)
    bi = np.floor(kmag / (kmax / nbin))
    full = [np.sum((bi == i) & (kmag > 0)) for i in range(nbin)]
    assert np.array_equal(r["nmodes"], np.array(full, float))


def test_lattice_has_no_power_below_its_frequency():
    Ng, L, M = 32, 64.0, 4                      # lattice of 4^3 points on grid points
    g = (np.arange(M) + 0.0) * L / M
    x, y, z = [a.ravel() for a in np.meshgrid(g, g, g, indexing="ij")]
    kl = 2 * np.pi / L * M
    for inter in (False, True):
        r = pkest.powspec(x, y, z, L, Ng, interlace=inter, kmin=0.0, kmax=0.9 * kl, nbin=8)
        has = r["nmodes"] > 0                       # bins without modes report 0
        assert has.sum() >= 5
        assert np.allclose((r["P0"] + r["shot"])[has], 0, atol=1e-9 * r["shot"])
        assert np.allclose(r["P2"][has], 0, atol=1e-9 * r["shot"])


def test_modulation_along_line_of_sight_gives_p2_over_p0_of_5():
    Ng, L = 32, 128.0
    # x, y on grid points; z density 1 + A cos(k0 z), k0 = 3 kf (inverse CDF)
    k0, A = 3 * 2 * np.pi / L, 0.4
    nz = 4096
    zz = np.linspace(0, L, 200001)
    cdf = (zz + A / k0 * np.sin(k0 * zz)) / L
    z1 = np.interp((np.arange(nz) + 0.5) / nz, cdf, zz)
    g = np.arange(4) * L / 4
    x, y, z = [a.ravel() for a in np.meshgrid(g, g, z1, indexing="ij")]
    kf = 2 * np.pi / L
    r = pkest.powspec(x, y, z, L, Ng, interlace=True, kmin=2.5 * kf, kmax=3.5 * kf, nbin=1)
    raw = r["P0"][0] + r["shot"]
    assert raw > 20 * r["shot"]                   # the two z modes dominate the bin
    assert abs(r["P2"][0] / raw - 5.0) < 1e-9


def test_cic_pdf_counts():
    L, Ng = 10.0, 2
    # cells of side 5: 3 tracers in cell (0,0,0), 1 in (1,1,1), none elsewhere
    x = np.array([1.0, 2.0, 3.0, 7.0])
    y = np.array([1.0, 2.0, 4.9, 9.0])
    z = np.array([0.1, 0.2, 0.3, 6.0])
    pdf = pkest.cic_pdf(x, y, z, L, Ng, nbin=3)
    assert np.allclose(pdf, [6 / 8, 1 / 8, 1 / 8])   # last bin: >= 2
    # redshift-space shift moves the fourth tracer into cell (1,1,0)
    pdf = pkest.cic_pdf(x, y, z, L, Ng, nbin=5, vz=np.array([0, 0, 0, 50.0]), rsd_fac=0.1)
    assert np.allclose(pdf, [6 / 8, 1 / 8, 0, 1 / 8, 0])
