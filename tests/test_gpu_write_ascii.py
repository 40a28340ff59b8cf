"""EZmock_write_ascii byte for byte against the reference's own writer
(libEZmock/EZmock/save_res.c:95-178, compiled unmodified in oracle/_ref):
the same catalogue written by both libraries, header on and off, real space
(rsd_fac = 0: positions and velocities) and redshift space (rsd_fac > 0:
z + rsd_fac vz wrapped into the box, save_res.c:147-158), both `real`
builds."""
import ctypes

import numpy as np
import pytest

from ezmock_b200 import EZmock
from ezmock_b200.workloads import bbks_pk
from oracle.pyoracle import RefLib

from conftest import has_ref

pytestmark = pytest.mark.skipif(not has_ref(), reason="oracle/_ref not built")

PARAMS = [0.6, 15.0, 0.35, 300.0]


def gpu_write(m, cat, fname, rsd_fac, header):
    L = m._L
    rp = ctypes.POINTER(L._rt)
    arrs = [np.ascontiguousarray(a, m._rdt) for a in cat]
    err = ctypes.c_int(0)
    r = L.EZmock_write_ascii(m._ez, *[a.ctypes.data_as(rp) for a in arrs], len(arrs[0]),
                             float(rsd_fac), bool(header), str(fname).encode(),
                             ctypes.byref(err))
    return r, err.value


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("fixamp,iphase", [(False, False), (True, True)])
def test_write_ascii_bytes(tmp_path, prec, fixamp, iphase):
    k, P = bbks_pk()
    Ng, L, seed, rng = 32, 250.0, 3, 0
    nexp = int(3e-4 * L ** 3)
    m = EZmock(Lbox=L, Ngrid=Ng, rng=rng, seed=seed, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P)
    m.create_dens_field_from_ic(fixamp=fixamp, iphase=iphase)
    cat = m.populate_tracer(*PARAMS, nexp)
    assert len(cat[0]) > 1000
    # the reference instance in the same state: its header prints the
    # instance's box, grid, IC flags, growth, bias parameters and generator
    R = RefLib(prec, nthread=1)
    r = R.new(L, Ng, rng, seed)
    r.eval_growth(0.8, 0.31)
    r.setup_pk(k, P)
    r.create(fixamp=fixamp, iphase=iphase)
    r.populate(PARAMS, nexp)
    # a z coordinate pushed over the box edge by the velocity, and one below 0
    cat = [np.array(a) for a in cat]
    cat[2][1], cat[5][1] = L - 0.01, 250.0
    cat[2][2], cat[5][2] = 0.01, -250.0
    for rsd in (0.0, 0.0114):
        for header in (True, False):
            fg, fr = tmp_path / f"g_{rsd}_{header}.txt", tmp_path / f"r_{rsd}_{header}.txt"
            assert gpu_write(m, cat, fg, rsd, header) == (0, 0)
            assert r.write_ascii(cat, fr, rsd, header) == 0
            bg, br = fg.read_bytes(), fr.read_bytes()
            assert len(bg) > 1000 * (20 if rsd else 40)
            assert bg == br, f"rsd {rsd} header {header}: files differ"


@pytest.mark.parametrize("prec", [32, 64])
def test_write_ascii_errors_match_reference(tmp_path, prec):
    """Argument errors of the writer, code for code with the reference's:
    no tracers, rsd_fac above the box size, an empty file name, a first
    element equal to zero (the reference's `!(*x)` test), an unwritable
    path.  Host code only: runs without a GPU."""
    k, P = bbks_pk()
    m = EZmock(Lbox=250.0, Ngrid=32, rng=1, seed=1, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P)
    R = RefLib(prec, nthread=1)
    r = R.new(250.0, 32, 1, 1)
    r.eval_growth(0.8, 0.31)
    r.setup_pk(k, P)
    rdt = np.float32 if prec == 32 else np.float64
    good = [np.full(10, 1.5, rdt) for _ in range(6)]
    zero = [a.copy() for a in good]
    zero[3][0] = 0
    ok = str(tmp_path / "ok.txt")
    cases = [(good, 0, ok, 0.0), (good, 10, ok, 300.0), (good, 10, "", 0.0),
             (zero, 10, ok, 0.0), (good, 10, str(tmp_path / "missing" / "x.txt"), 0.0)]
    rp = ctypes.POINTER(m._L._rt)
    for cat, n, name, rsd in cases:
        err = ctypes.c_int(0)
        m._L.EZmock_write_ascii(m._ez, *[a.ctypes.data_as(rp) for a in cat], n, rsd, True,
                                name.encode(), ctypes.byref(err))
        rerr = ctypes.c_int(0)
        R.lib.EZmock_write_ascii(r.ez, *[a.ctypes.data for a in cat], n, rsd, True,
                                 name.encode(), ctypes.byref(rerr))
        assert err.value == rerr.value and err.value != 0, (n, name, rsd, err.value, rerr.value)
