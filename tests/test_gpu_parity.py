"""GPU parity: the CUDA library, called through its C-ABI (ctypes), against
the CPU oracle and the reference's golden vectors.

Tolerances:
  * random draws, per-cell tracer counts, tracer positions: bit-exact;
  * FP64 fields (psi, rho): max|gpu - oracle| <= 1e-12 * max|oracle|;
  * FP64 velocities: <= 1e-9 * max|v| (atomic summation order of the
    painted displacement grids);
  * FP32 fields against the FP64 oracle (stated field error of the
    production mode): psi <= 5e-6 * max|oracle|; rho <= 5e-6 at 64^3 and
    <= 1e-5 up to 512^3 (its error grows with the grid because particle
    positions psi Ng/L + i are rounded to single precision, as in the
    reference's FP32 build).
"""
import ctypes
import os

import numpy as np
import pytest

from ezmock_b200 import EZmock, _lib
from ezmock_b200.workloads import wiggle_pk
from oracle import pkest
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
PARAMS = [0.6, 15.0, 0.35, 300.0]


def relmax(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make(prec, Ng, L, rng, seed, k, P, Pnw=None, mBAO=0.0, logint=False):
    m = EZmock(Lbox=L, Ngrid=Ng, rng=rng, seed=seed, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P, Pnw, mBAO, logint)
    return m


def oracle_field(prec, Ng, L, rng, seed, k, P, fixamp=False, iphase=False, Pnw=None,
                 mBAO=0.0, logint=False):
    O = Oracle(prec)
    g2, vf = O.growth(0.8, 0.0, 0.31)
    t = O.pk_setup(Ng, L, g2, k, P, Pnw, mBAO, logint)
    psi, rho = O.dens_field(t, Ng, L, rng, seed, fixamp, iphase)
    return O, t, vf, psi, rho


def cell_counts(x, y, z, Ng, L):
    gs = L / Ng
    idx = [np.floor(np.asarray(a, np.float64) / gs + 0.5).astype(np.int64) % Ng for a in (x, y, z)]
    flat = (idx[0] * Ng + idx[1]) * Ng + idx[2]
    return np.bincount(flat, minlength=Ng ** 3)


@pytest.mark.parametrize("rng", [0, 1])
@pytest.mark.parametrize("start,count", [(0, 2000), (12345, 70000), ((1 << 28) + 777, 5000),
                                         (8 * 512 ** 3 + 3, 3000), (5 * 64 ** 3, 400000)])
def test_rng_streams(rng, start, count):
    L = _lib.load(64)
    out = np.zeros(count, np.uint32)
    assert L.EZmockB200_rng_raw(rng, 7, start, count, out.ctypes.data_as(ctypes.c_void_p)) == 0
    assert np.array_equal(out, Oracle(64).rng_raw(rng, 7, start, count))


@pytest.mark.parametrize("rng", [0, 1])
@pytest.mark.parametrize("fixamp,iphase", [(False, False), (True, False), (False, True)])
@pytest.mark.parametrize("Ng,L", [(32, 250.0), (40, 320.0), (24, 400.0)])
def test_dens_field_fp64(pk_table, rng, fixamp, iphase, Ng, L):
    k, P = pk_table
    m = make(64, Ng, L, rng, 5, k, P)
    m.create_dens_field_from_ic(fixamp=fixamp, iphase=iphase)
    O, t, vf, psi, rho = oracle_field(64, Ng, L, rng, 5, k, P, fixamp, iphase)
    for d in range(3):
        assert relmax(m.field(d), psi[d]) <= TOL64
    assert relmax(m.field(3), rho) <= TOL64


@pytest.mark.parametrize("logint", [False, True])
def test_dens_field_bao_logint_fp64(pk_table, logint):
    k, Pnw = pk_table
    P = wiggle_pk(k, Pnw)
    m = make(64, 32, 250.0, 1, 9, k, P, Pnw, 3.0, logint)
    m.create_dens_field_from_ic()
    O, t, vf, psi, rho = oracle_field(64, 32, 250.0, 1, 9, k, P, Pnw=Pnw, mBAO=3.0, logint=logint)
    assert relmax(m.field(3), rho) <= TOL64
    assert relmax(m.field(0), psi[0]) <= TOL64


def test_dens_field_fp32_error(pk_table):
    k, P = pk_table
    m = make(32, 64, 500.0, 1, 3, k, P)
    m.create_dens_field_from_ic()
    O, t, vf, psi, rho = oracle_field(64, 64, 500.0, 1, 3, k, P)
    for d in range(3):
        assert relmax(m.field(d), psi[d]) <= 5e-6
    assert relmax(m.field(3), rho) <= 5e-6


@pytest.mark.parametrize("rng,fixamp,iphase,Ng,L", [
    (0, False, False, 64, 500.0), (1, True, False, 64, 500.0), (1, False, True, 64, 500.0),
    (0, True, True, 64, 500.0), (1, False, False, 40, 320.0), (0, True, False, 40, 320.0)])
def test_dens_field_fp32_modes(pk_table, rng, fixamp, iphase, Ng, L):
    """FP32 fields of both generators with fixed amplitudes and inverted
    phases, against the FP64 oracle within the stated FP32 field error
    (1e-5), on a grid of the warp-shuffle FFT (64^3) and of the block FFT
    (40^3)."""
    k, P = pk_table
    m = make(32, Ng, L, rng, 3, k, P)
    m.create_dens_field_from_ic(fixamp=fixamp, iphase=iphase)
    O, t, vf, psi, rho = oracle_field(64, Ng, L, rng, 3, k, P, fixamp, iphase)
    err = [relmax(m.field(d), psi[d]) for d in range(3)] + [relmax(m.field(3), rho)]
    print(f"FP32 field error {Ng}^3 rng {rng} fixamp {fixamp} iphase {iphase}: {err}")
    assert max(err) <= 1e-5


@pytest.mark.parametrize("Ng", [128, 256, 512])
def test_dens_field_fp32_large_grids(pk_table, Ng):
    """FP32 fields on the grids whose transforms hold 4, 8 and 16 points per
    lane (512^3 is the benchmark grid), cell size of the benchmark (4.88
    Mpc/h), against the FP64 oracle within the stated FP32 field error for
    grids up to 512^3 (1e-5).  Measured: psi about 3e-7 on every grid; rho
    1.8e-6, 3.8e-6 and 7.5e-6 on 128^3, 256^3 and 512^3, growing with the
    single-precision rounding of particle positions near the upper grid
    indices (the reference's FP32 build rounds them the same way)."""
    k, P = pk_table
    L = 2500.0 * Ng / 512
    m = make(32, Ng, L, 1, 3, k, P)
    m.create_dens_field_from_ic()
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, 3, k, P)
    err = [relmax(m.field(d), psi[d]) for d in range(3)] + [relmax(m.field(3), rho)]
    print(f"FP32 field error {Ng}^3: psi {err[0]:.2e} {err[1]:.2e} {err[2]:.2e} rho {err[3]:.2e}")
    assert max(err) <= 1e-5


@pytest.mark.parametrize("tile", [16, 32])
@pytest.mark.parametrize("halo", [2, 3])
def test_dens_field_fp32_large_displacements(pk_table, halo, tile):
    """FP32 density with displacements of about two cells (box 100 Mpc/h on
    64^3): many particles move beyond the assignment halo and are deposited
    by the global-atomic pass.  Three fields in a row (the set halo, then the
    halo the engine picks) all match the oracle, with either column tile."""
    k, P = pk_table
    m = make(32, 64, 100.0, 1, 3, k, P)
    m.set_option(5, halo)
    m.set_option(7, tile)
    O, t, vf, psi, rho = oracle_field(64, 64, 100.0, 1, 3, k, P)
    O32 = Oracle(32)
    painted = None
    for _ in range(3):
        m.create_dens_field_from_ic()
        assert relmax(m.field(3), rho) <= 5e-6
        if painted is None:
            # the oracle's painting of the GPU displacements, divided by ones
            # (pop_tracer.c:593-683 before its division by rho)
            psi32 = [m.field(d) for d in range(3)]
            ones = np.ones((64, 64, 64), np.float32)
            painted = [O32.paint(64, 100.0, psi32, ones, d) for d in range(3)]
        for d in range(3):
            assert relmax(m.field(4 + d), painted[d]) <= 1e-5
    with pytest.raises(RuntimeError):
        m.set_option(5, 4)


@pytest.mark.parametrize("Ng,L", [(64, 500.0), (128, 625.0), (256, 1250.0)])
def test_cic_tiles_agree(pk_table, Ng, L):
    """The FP32 density and painted displacement grids of the 32 x 32 column
    tiles (the z range cut into 1 to 16 pieces, by grid) are bit for bit
    those of the 16 x 16 tiles wherever no particle displaced beyond the halo
    (3 cells) deposits: both sum the same fixed-point deposits, which is
    exact; the few far particles go through float atomics, whose order
    differs between the two (at most 1e-5 of the cells, within 1e-6)."""
    k, P = pk_table
    out = []
    for tile in (16, 32):
        m = make(32, Ng, L, 1, 6, k, P)
        m.set_option(5, 3)
        m.set_option(7, tile)
        m.create_dens_field_from_ic()
        out.append([m.field(w) for w in (3, 4, 5, 6)])
    for a, b in zip(*out):
        assert np.count_nonzero(a != b) <= 1e-5 * a.size
        assert relmax(b, a) <= 1e-6
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, 6, k, P)
    assert relmax(out[1][0], rho) <= 1e-5


@pytest.mark.parametrize("Ng,L", [(256, 1250.0), (512, 2500.0)])
def test_fft_tma_matches_cp_async(pk_table, Ng, L):
    """The FP32 transforms along y staged by the Tensor Memory Accelerator
    (the default on 256^3 and 512^3) and by per-thread cp.async copies give
    the same displacement fields to single-precision rounding (their line
    transforms differ in the order of the 32-point stages), and the TMA
    fields are within the stated FP32 error of the FP64 oracle."""
    k, P = pk_table
    out = []
    for tma in (1, 0):
        m = make(32, Ng, L, 1, 9, k, P)
        m.set_option(8, tma)
        m.create_dens_field_from_ic()
        out.append([m.field(d) for d in range(3)])
        del m
    for a, b in zip(*out):
        assert relmax(a, b) <= 1e-6
    if Ng == 256:
        O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, 9, k, P)
        for d in range(3):
            assert relmax(out[0][d], psi[d]) <= 5e-6


@pytest.mark.parametrize("Ng,L", [(512, 2500.0), (1024, 5000.0)])
def test_fft_pass_i_tma_bit_identical(pk_table, Ng, L):
    """The FP32 transform along x with its tiles moved by the Tensor Memory
    Accelerator (the default) and by per-thread cp.async copies runs the same
    line transforms, so the displacement fields agree bit for bit (1024^3:
    psi_x, the field whose pass-I output is the separate A_x spectrum, and
    psi_z)."""
    k, P = pk_table
    comps = (0, 2) if Ng >= 1024 else (0, 1, 2)
    out = []
    for tma in (1, 0):
        m = make(32, Ng, L, 1, 13, k, P)
        m.set_option(10, tma)
        m.create_dens_field_from_ic()
        out.append([m.field(d) for d in comps])
        del m
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("rng", [0, 1])
def test_golden_reference_fp64(golden, pk_table, rng):
    """16^3 fields, counts and catalogue of the reference's own build."""
    k, P = pk_table
    tag = f"f64_rng{rng}_fa0"
    m = make(64, 16, 200.0, rng, 7, k, P)
    m.create_dens_field_from_ic()
    psi = golden[tag + "_psi"]
    for d in range(3):
        assert relmax(m.field(d), psi[d]) <= TOL64
    assert relmax(m.field(3), golden[tag + "_rho"]) <= TOL64
    nexp = int(round(3e-4 * 200.0 ** 3))
    cat = m.populate_tracer(*PARAMS, nexp)
    ref = golden[tag + "_cat"]
    assert len(cat[0]) == ref.shape[1]
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])
    vmax = np.abs(ref[3:]).max()
    for a in range(3, 6):
        assert np.abs(cat[a] - ref[a]).max() <= 1e-9 * vmax
    assert np.array_equal(cell_counts(*cat[:3], 16, 200.0),
                          golden[tag + "_nt"].reshape(-1).astype(np.int64))


@pytest.mark.parametrize("rng", [0, 1])
@pytest.mark.parametrize("params,n", [([0.6, 15.0, 0.35, 300.0], 3e-4),
                                      ([1.2, 5.0, 0.2, 150.0], 1e-4),
                                      ([0.3, 30.0, 0.6, 500.0], 5e-4),
                                      ([0.0, 10.0, 0.3, 0.0], 2e-4)])
def test_populate_fp64(pk_table, rng, params, n):
    k, P = pk_table
    Ng, L = 48, 400.0
    m = make(64, Ng, L, rng, 2, k, P)
    m.create_dens_field_from_ic()
    nexp = int(n * L ** 3)
    cat = m.populate_tracer(*params, nexp)
    O, t, vf, psi, rho = oracle_field(64, Ng, L, rng, 2, k, P)
    e, ref = O.populate(Ng, L, rng, 2, vf, psi, rho, params, nexp)
    assert e == 0
    assert len(cat[0]) == len(ref[0])
    assert np.array_equal(cell_counts(*cat[:3], Ng, L), cell_counts(*ref[:3], Ng, L))
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])
    vmax = np.abs(np.stack(ref[3:])).max()
    for a in range(3, 6):
        assert np.abs(cat[a] - ref[a]).max() <= 1e-9 * vmax


def test_populate_fp32_against_fp64_oracle(pk_table):
    """The FP32 mode against the FP64 oracle on the benchmark's cell size and
    tracer density (64^3, box 312.5 Mpc/h): the FP32 field error moves no
    cell across rho_c, so the valid-cell ranks that index the bias Gaussians
    (pop_tracer.c:233-237) are the same, and every cell gets the same number
    of tracers; P0 and P2 (40 bins, 0.005-0.3 h/Mpc, RSD) agree within 0.5%
    of P0.  (Where the error moves a cell across rho_c, the Gaussians of
    every later valid cell shift, in the reference's own FP32 build as
    here.)"""
    k, P = pk_table
    Ng, L, seed = 64, 312.5, 7
    params = [0.8, 20.0, 0.3, 400.0]
    nexp = int(round(2e-4 * L ** 3))
    m = make(32, Ng, L, 1, seed, k, P)
    m.create_dens_field_from_ic()
    cat = m.populate_tracer(*params, nexp)
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, seed, k, P)
    e, ref = O.populate(Ng, L, 1, seed, vf, psi, rho, params, nexp)
    assert e == 0
    rho32 = m.field(3)
    assert relmax(rho32, rho) <= 5e-6
    # the precondition: the same valid cells (float and double comparisons)
    assert np.array_equal(rho32 >= np.float32(params[0]), rho >= params[0])
    assert np.array_equal(cell_counts(*cat[:3], Ng, L), cell_counts(*ref[:3], Ng, L))
    rsd = 0.0114
    p32 = pkest.powspec(*cat[:3], L, 64, True, 0.005, 0.3, 40, vz=cat[5], rsd_fac=rsd)
    p64 = pkest.powspec(*ref[:3], L, 64, True, 0.005, 0.3, 40, vz=ref[5], rsd_fac=rsd)
    has = p64["nmodes"] > 0
    scale = np.abs(p64["P0"])[has]
    assert np.all(np.abs(p32["P0"] - p64["P0"])[has] <= 5e-3 * scale)
    assert np.all(np.abs(p32["P2"] - p64["P2"])[has] <= 5e-3 * scale)


def test_populate_fp32_positions(pk_table):
    """FP32: on the GPU's own density field the oracle reproduces the
    catalogue positions bit for bit."""
    k, P = pk_table
    Ng, L = 64, 500.0
    m = make(32, Ng, L, 1, 4, k, P)
    m.create_dens_field_from_ic()
    nexp = int(3e-4 * L ** 3)
    cat = m.populate_tracer(*PARAMS, nexp)
    O = Oracle(32)
    _, vf = O.growth(0.8, 0.0, 0.31)
    e, ref = O.populate(Ng, L, 1, 4, vf, [m.field(d) for d in range(3)], m.field(3), PARAMS, nexp)
    assert e == 0 and len(ref[0]) == len(cat[0])
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])
    vmax = np.abs(np.stack(ref[3:])).max()
    for a in range(3, 6):
        assert np.abs(cat[a] - ref[a]).max() <= 1e-4 * vmax


def test_repeated_populations_fp64(pk_table):
    """Several populations on one density field (the field is not modified)."""
    k, P = pk_table
    Ng, L = 32, 250.0
    m = make(64, Ng, L, 0, 11, k, P)
    m.create_dens_field_from_ic()
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 0, 11, k, P)
    for params, n in [([0.5, 10.0, 0.3, 250.0], 2e-4), ([0.9, 20.0, 0.4, 350.0], 1e-4),
                      ([1.3, 30.0, 0.5, 450.0], 2e-5 * 10)]:
        nexp = int(n * L ** 3)
        cat = m.populate_tracer(*params, nexp)
        e, ref = O.populate(Ng, L, 0, 11, vf, psi, rho, params, nexp)
        assert e == 0 and len(cat[0]) == len(ref[0])
        for a in range(3):
            assert np.array_equal(cat[a], ref[a])


def test_catalogue_host_pool(pk_table):
    """Catalogues of over 4 MB per array come from pre-faulted host blocks
    (EZMOCKB200_OPT_HOST_POOL): repeated populations of one field give the
    same catalogue with the pool filled, with a second population size in
    between, and with the pool turned off."""
    k, P = pk_table
    Ng, L = 128, 1000.0
    m = make(32, Ng, L, 1, 5, k, P)
    m.create_dens_field_from_ic()
    params = [0.3, 10.0, 0.3, 300.0]
    nexp = 1_200_000
    first = m.populate_tracer(*params, nexp)
    assert len(first[0]) >= nexp
    for n2 in (nexp, 600_000, nexp):
        cat = m.populate_tracer(*params, n2)
        if n2 == nexp:
            for a in range(6):
                assert np.array_equal(cat[a], first[a])
    m.set_option(6, 0)
    cat = m.populate_tracer(*params, nexp)
    for a in range(6):
        assert np.array_equal(cat[a], first[a])
    m.set_option(6, 64)
    with pytest.raises(RuntimeError):
        m.set_option(6, -1)


def test_white_noise_fp64(pk_table):
    k, P = pk_table
    Ng, L = 32, 250.0
    delta = np.random.default_rng(8).standard_normal(Ng ** 3)
    m = make(64, Ng, L, 1, 1, k, P)
    m.create_dens_field_from_wn(delta)
    O = Oracle(64)
    g2, vf = O.growth(0.8, 0.0, 0.31)
    t = O.pk_setup(Ng, L, g2, k, P)
    psi = O.disp_whitenoise(t, Ng, L, delta)
    for d in range(3):
        assert relmax(m.field(d), psi[d]) <= TOL64
    assert relmax(m.field(3), O.cic(Ng, L, psi)) <= TOL64


@pytest.mark.parametrize("deepcopy", [False, True])
def test_user_displacements_fp64(pk_table, deepcopy):
    k, P = pk_table
    Ng, L = 32, 250.0
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, 6, k, P)
    m = make(64, Ng, L, 1, 6, k, P)
    m.create_dens_field_from_disp(*[p.reshape(-1) for p in psi], deepcopy=deepcopy)
    assert relmax(m.field(3), rho) <= TOL64
    nexp = int(3e-4 * L ** 3)
    cat = m.populate_tracer(*PARAMS, nexp)
    e, ref = O.populate(Ng, L, 1, 6, vf, psi, rho, PARAMS, nexp)
    assert e == 0 and len(cat[0]) == len(ref[0])
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])


@pytest.mark.parametrize("prec", [32, 64])
def test_deterministic_cic(pk_table, prec):
    k, P = pk_table
    Ng, L = 48, 400.0
    m = make(prec, Ng, L, 1, 2, k, P)
    m.set_option(1, 1)
    m.create_dens_field_from_ic()
    r1 = m.field(3).copy()
    q1 = m.field(4).copy()
    m.create_dens_field_from_ic()
    assert np.array_equal(r1, m.field(3)) and np.array_equal(q1, m.field(4))
    O, t, vf, psi, rho = oracle_field(64, Ng, L, 1, 2, k, P)
    assert relmax(r1, rho) <= (TOL64 if prec == 64 else 5e-6)


def _select(m, prec, rhot, hist, pdf, nmax, ncell, ntot):
    L = m._L
    rdt = np.float32 if prec == 32 else np.float64
    rhot = np.ascontiguousarray(rhot, rdt).reshape(-1)
    hist = np.ascontiguousarray(hist, np.uintp)
    pdf = np.array(pdf, np.uintp)
    nc, no = ctypes.c_size_t(ncell), ctypes.c_size_t(ntot)
    nt = np.zeros(rhot.size, np.int16)
    err = ctypes.c_int(0)
    r = L.EZmockB200_select_counts(m._ez, rhot.ctypes.data, hist.ctypes.data, pdf.ctypes.data,
                                   nmax, ctypes.byref(nc), ctypes.byref(no), nt.ctypes.data,
                                   ctypes.byref(err))
    return r, nt, pdf, nc.value, no.value


def test_selection_ties_golden(golden, pk_table):
    k, P = pk_table
    m = make(64, 16, 200.0, 1, 3, k, P)
    m.create_dens_field_from_ic()
    nmax, ncell, ntot = (int(v) for v in golden["ties_in"])
    r, nt, pdf, nc, no = _select(m, 64, golden["ties_rhot"], golden["ties_hist"],
                                 golden["ties_pdf_in"], nmax, ncell, ntot)
    assert r == 0
    assert np.array_equal(nt.reshape(16, 16, 16), golden["ties_nt"])
    assert list(pdf) == list(golden["ties_pdf_out"])
    assert [nc, no] == list(golden["ties_out"])


@pytest.mark.parametrize("sort", [0, 1])
@pytest.mark.parametrize("prec", [32, 64])
def test_selection_ties_random(pk_table, prec, sort):
    """Selection on tracer densities with many ties against the oracle, with
    the boundaries from the value buckets (option 9 = 0; the heaviest ties
    overflow the gather buffer and fall back to the full sort) and from the
    full sort (option 9 = 1)."""
    k, P = pk_table
    Ng = 32
    m = make(prec, Ng, 250.0, 1, 3, k, P)
    m.set_option(9, sort)
    m.create_dens_field_from_ic()
    O = Oracle(prec)
    rs = np.random.default_rng(5)
    done = 0
    paths = set()
    for trial in range(10):
        nv = int(rs.choice([300, 3000, 30000]))
        vals = np.exp(rs.uniform(-3, 3.5, nv)).astype(O.rdt)
        rhot = vals[rs.integers(0, nv, Ng ** 3)]
        rhot[rs.random(Ng ** 3) < 0.3] = 0
        lb = np.floor(np.log2(rhot[rhot > 0].astype(np.float64))).astype(int)
        hist = np.zeros(64, np.uintp)
        np.add.at(hist, np.clip(5 - lb, 0, 63), 1)
        e, pdf, nmax, ncell, ntot = O.eval_pdf(Ng, int(rs.integers(500, 8000)),
                                               float(rs.uniform(0.2, 0.6)))
        if e or ncell > (rhot > 0).sum():
            continue
        e2, nt_o, pdf_o, nc_o, no_o = O.select(Ng, rhot.reshape(Ng, Ng, Ng), hist, pdf,
                                               nmax, ncell, ntot)
        r, nt, pdf_g, nc, no = _select(m, prec, rhot, hist, pdf, nmax, ncell, ntot)
        assert r == e2
        if r:
            continue
        paths.add(m.select_path())
        assert np.array_equal(nt, nt_o.reshape(-1))
        assert list(pdf_g) == list(pdf_o) and (nc, no) == (nc_o, no_o)
        done += 1
    assert done >= 3
    if sort:
        assert paths == {1}
    else:
        assert 0 in paths and paths <= {0, 2}


@pytest.mark.parametrize("prec", [32, 64])
def test_selection_tie_flood(pk_table, prec):
    """A PDF-bin boundary inside a run of 17000 equal tracer densities: the
    bucket search finds more candidates in the boundary's bucket than it
    gathers, falls back to the full sort (path 2), and the counts equal the
    oracle's and the full sort's."""
    k, P = pk_table
    Ng = 32
    m = make(prec, Ng, 250.0, 1, 3, k, P)
    m.create_dens_field_from_ic()
    O = Oracle(prec)
    rs = np.random.default_rng(11)
    rhot = np.zeros(Ng ** 3, O.rdt)
    cells = rs.permutation(Ng ** 3)
    rhot[cells[:200]] = rs.uniform(2.0, 8.0, 200)
    rhot[cells[200:17200]] = 1.5
    rhot[cells[17200:27200]] = rs.uniform(1.0, 1.5, 10000)
    lb = np.floor(np.log2(rhot[rhot > 0].astype(np.float64))).astype(int)
    hist = np.zeros(64, np.uintp)
    np.add.at(hist, np.clip(5 - lb, 0, 63), 1)
    pdf = [50, 400, 3000]
    ncell, ntot = sum(pdf), 50 * 3 + 400 * 2 + 3000
    e2, nt_o, pdf_o, nc_o, no_o = O.select(Ng, rhot.reshape(Ng, Ng, Ng), hist, pdf, 3,
                                           ncell, ntot)
    assert e2 == 0 and nc_o == 200 + 17000 + 3000
    for sort, path in ((0, 2), (1, 1)):
        m.set_option(9, sort)
        r, nt, pdf_g, nc, no = _select(m, prec, rhot, hist, pdf, 3, ncell, ntot)
        assert r == 0 and m.select_path() == path
        assert np.array_equal(nt, nt_o.reshape(-1))
        assert list(pdf_g) == list(pdf_o) and (nc, no) == (nc_o, no_o)


@pytest.mark.parametrize("Ng,L,n", [(128, 625.0, 2e-4), (256, 1250.0, 2e-4), (128, 625.0, 3e-3)])
def test_select_buckets_match_sort(pk_table, Ng, L, n):
    """FP32 catalogues with the selection boundaries from the value buckets
    (the default, which must not fall back at these densities) and from the
    full radix sort are identical."""
    k, P = pk_table
    m = make(32, Ng, L, 1, 4, k, P)
    m.create_dens_field_from_ic()
    nexp = int(n * L ** 3)
    cats = []
    for sort in (0, 1):
        m.set_option(9, sort)
        cats.append(m.populate_tracer(0.8, 20.0, 0.3, 400.0, nexp))
        assert m.select_path() == sort
    for a, b in zip(*cats):
        assert np.array_equal(a, b)


def test_write_ascii(pk_table, tmp_path):
    k, P = pk_table
    m = make(32, 32, 250.0, 1, 1, k, P)
    m.create_dens_field_from_ic()
    fn = tmp_path / "cat.txt"
    m.populate_tracer_to_file(*PARAMS, int(3e-4 * 250.0 ** 3), str(fn), rsd_fac=0.0113)
    lines = fn.read_text().splitlines()
    assert lines[0].startswith("# BOX_SIZE=250 , NUM_GRID=32")
    assert lines[3] == "# RAND_GENERATOR=MT19937 , RAND_SEED=1"
    assert lines[4] == "# x(1) y(2) z_rsd(3)"
    cat = m.populate_tracer(*PARAMS, int(3e-4 * 250.0 ** 3))
    x, z, vz = cat[0][0], cat[2][0], cat[5][0]
    zr = float(z) + 0.0113 * float(vz)
    if zr >= 250.0:
        zr -= 250.0
    if zr < 0:
        zr += 250.0
    assert lines[5].split()[0] == "%.6g" % x
    assert lines[5].split()[2] == "%.6g" % zr
    assert len(lines) == 5 + len(cat[0])


def test_error_paths(pk_table):
    k, P = pk_table
    m = make(64, 32, 250.0, 1, 1, k, P)
    with pytest.raises(RuntimeError, match="density fields uninitialized"):
        m.populate_tracer(*PARAMS, 4000)
    m = make(64, 32, 250.0, 1, 1, k, P)
    m.create_dens_field_from_ic()
    with pytest.raises(RuntimeError, match="too many expected"):
        m.populate_tracer(*PARAMS, 32 ** 3)
    m = make(64, 32, 250.0, 1, 1, k, P)
    m.create_dens_field_from_ic()
    with pytest.raises(RuntimeError, match="invalid base number"):
        m.populate_tracer(0.6, 15.0, 1.0, 300.0, 4000)
    m = make(64, 32, 250.0, 1, 1, k, P)
    m.create_dens_field_from_ic()
    with pytest.raises(RuntimeError, match="not enough cells"):
        m.populate_tracer(50.0, 15.0, 0.35, 300.0, 20000)
