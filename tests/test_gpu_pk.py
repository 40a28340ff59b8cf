"""GPU clustering estimators (EZmockB200_powspec, EZmockB200_cic_pdf) against
the numpy restatement in oracle/pkest.py, through the C ABI."""
import ctypes

import numpy as np
import pytest

from ezmock_b200 import EZmock
from ezmock_b200.workloads import bbks_pk
from oracle import pkest

pytestmark = pytest.mark.gpu

# raw power (P0 + shot noise) relative tolerance; FP32 grids are accumulated
# with float atomics and transformed in single precision
RTOL = {32: 2e-4, 64: 1e-9}


def _catalogue(n, L, seed, dt):
    rng = np.random.default_rng(seed)
    # clustered: half the tracers in Gaussian blobs
    c = rng.uniform(0, L, (3, 40))
    k = rng.integers(0, 40, n // 2)
    blob = (c[:, k] + rng.normal(0, 0.02 * L, (3, n // 2))) % L
    uni = rng.uniform(0, L, (3, n - n // 2))
    x, y, z = np.concatenate([blob, uni], axis=1).astype(dt)
    vz = rng.normal(0, 300, n).astype(dt)
    return x, y, z, vz


def _compare(res, ref, prec):
    raw = res["P0"] + ref["shot"]
    rraw = ref["P0"] + ref["shot"]
    assert np.array_equal(res["nmodes"], ref["nmodes"])
    assert np.allclose(res["k_mean"], ref["k_mean"], rtol=1e-12)
    has = ref["nmodes"] > 0
    assert np.all(np.abs(raw - rraw)[has] <= RTOL[prec] * np.abs(rraw)[has])
    assert np.all(np.abs(res["P2"] - ref["P2"])[has] <= RTOL[prec] * np.abs(rraw)[has])


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("interlace,rsd", [(True, 0.0), (False, 0.0), (True, 0.01)])
def test_powspec_host_catalogue(prec, interlace, rsd):
    L, ng = 500.0, 64
    dt = np.float32 if prec == 32 else np.float64
    x, y, z, vz = _catalogue(30000, L, 3, dt)
    m = EZmock(Lbox=L, Ngrid=32, prec=prec)
    res = m.powspec((x, y, z, vz), rsd_fac=rsd, ngrid=ng, interlace=interlace, kmin=0.005,
                    kmax=0.3, nbin=40)
    ref = pkest.powspec(x, y, z, L, ng, interlace, 0.005, 0.3, 40, vz=vz, rsd_fac=rsd)
    _compare(res, ref, prec)


@pytest.mark.parametrize("prec", [32, 64])
def test_cic_pdf_host_catalogue(prec):
    L = 500.0
    dt = np.float32 if prec == 32 else np.float64
    x, y, z, vz = _catalogue(30000, L, 5, dt)
    m = EZmock(Lbox=L, Ngrid=32, prec=prec)
    for rsd in (0.0, 0.01):
        got = m.cic_pdf((x, y, z, vz), rsd_fac=rsd, ngrid=24, nbin=32)
        ref = pkest.cic_pdf(x, y, z, L, 24, 32, vz=vz, rsd_fac=rsd)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("prec", [32, 64])
def test_estimators_on_device_catalogue(prec):
    """The catalogue left on the GPU by populate_device gives the same result
    as its host copy, and matches the oracle."""
    k, P = bbks_pk()
    Ng, L = 64, 500.0
    m = EZmock(Lbox=L, Ngrid=Ng, rng=1, seed=11, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P)
    m.create_dens_field_from_ic()
    n = m.populate_device(0.6, 15.0, 0.35, 300.0, int(3e-4 * L ** 3))
    rt = m._L._rt
    arrs = [(rt * n)() for _ in range(6)]
    err = ctypes.c_int(0)
    assert m._L.EZmockB200_copy_catalog(m._ez, *[ctypes.cast(a, ctypes.c_void_p) for a in arrs],
                                       n, ctypes.byref(err)) == 0
    x, y, z, vx, vy, vz = [np.frombuffer(a, dtype=np.dtype(rt)).copy() for a in arrs]
    rsd = 0.0114
    dev = m.powspec(None, rsd_fac=rsd, ngrid=64, kmin=0.005, kmax=0.3, nbin=40)
    host = m.powspec((x, y, z, vz), rsd_fac=rsd, ngrid=64, kmin=0.005, kmax=0.3, nbin=40)
    ref = pkest.powspec(x, y, z, L, 64, True, 0.005, 0.3, 40, vz=vz, rsd_fac=rsd)
    _compare(dev, ref, prec)
    _compare(host, ref, prec)
    assert np.array_equal(m.cic_pdf(None, rsd_fac=rsd, ngrid=32),
                          pkest.cic_pdf(x, y, z, L, 32, 32, vz=vz, rsd_fac=rsd))


def test_estimator_errors():
    m = EZmock(Lbox=100.0, Ngrid=32)
    x = np.zeros(10, np.float32)
    with pytest.raises(RuntimeError):          # no catalogue on the GPU yet
        m.powspec(None)
    m._err.value = 0
    with pytest.raises(RuntimeError):          # grid not supported by the FFT
        m.powspec((x, x, x), ngrid=7)
    m._err.value = 0
    with pytest.raises(RuntimeError):          # empty k range
        m.powspec((x, x, x), kmin=0.3, kmax=0.1)
