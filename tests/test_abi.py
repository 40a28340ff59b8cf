"""The C-ABI library on the CPU: it loads, exports every function that
include/*.h declares, and its host-side validation gives the reference's
error codes for the same calls (no GPU work is triggered here)."""
import ctypes

import numpy as np
import pytest

from ezmock_b200 import _lib
from conftest import has_ref

_vp = ctypes.c_void_p


@pytest.mark.parametrize("prec", [32, 64])
def test_exports(prec):
    L = _lib.load(prec)
    syms = _lib.header_symbols()
    assert "EZmock_init" in syms and "EZmock_populate_tracer" in syms
    for s in syms:
        assert hasattr(L, s), s
    assert L.EZmockB200_real_size() == prec // 8


def test_errmsg_table():
    L = _lib.load(64)
    assert L.EZmock_errmsg(0) == b"no error"
    assert L.EZmock_errmsg(8) == b"invalid grid size"
    assert L.EZmock_errmsg(39) == b"failed to initialise FFTW with OpenMP"
    assert L.EZmock_errmsg(41) == b"unknown error"
    assert L.EZmock_errmsg(99) == b"unregistered error code"


class _Api:
    """Drives EZmock.h of one library (ours or the reference build)."""

    def __init__(self, lib):
        self.L = lib
        L = lib
        ip = ctypes.POINTER(ctypes.c_int)
        L.EZmock_init.restype = _vp
        L.EZmock_init.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                  ctypes.c_int, ip]
        L.EZmock_set_cosmology.restype = ctypes.c_int
        L.EZmock_set_cosmology.argtypes = [_vp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_bool] + [ctypes.c_double] * 5 + [ip]
        L.EZmock_setup_linear_pk.restype = ctypes.c_int
        L.EZmock_setup_linear_pk.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_double,
                                             ctypes.c_bool, ip]
        L.EZmock_create_dens_field.restype = ctypes.c_int
        L.EZmock_create_dens_field.argtypes = [_vp, _vp, ctypes.c_bool, _vp, ctypes.c_bool,
                                               ctypes.c_bool, ip]
        pp = ctypes.POINTER(_vp)
        L.EZmock_populate_tracer.restype = ctypes.c_int
        L.EZmock_populate_tracer.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_bool,
                                             ctypes.POINTER(ctypes.c_size_t)] + [pp] * 6 + [ip]
        L.EZmock_destroy.argtypes = [_vp]

    def init(self, L, Ng, rng, seed, nth=1):
        err = ctypes.c_int(0)
        ez = self.L.EZmock_init(L, Ng, rng, seed, nth, ctypes.byref(err))
        return ez, err.value

    def cosmo(self, ez, *a):
        err = ctypes.c_int(0)
        r = self.L.EZmock_set_cosmology(ez, *a, ctypes.byref(err))
        return r, err.value

    def pk(self, ez, k, P, Pnw=None, mBAO=0.0, logint=False):
        err = ctypes.c_int(0)
        k = np.ascontiguousarray(k, np.float64)
        P = np.ascontiguousarray(P, np.float64)
        pnw = None if Pnw is None else np.ascontiguousarray(Pnw, np.float64).ctypes.data
        r = self.L.EZmock_setup_linear_pk(ez, k.ctypes.data, len(k), P.ctypes.data, pnw,
                                          mBAO, logint, ctypes.byref(err))
        return r, err.value

    def populate(self, ez, params, nexp):
        err = ctypes.c_int(0)
        prm = np.array(params, np.float64)
        n = ctypes.c_size_t()
        ptrs = [_vp() for _ in range(6)]
        r = self.L.EZmock_populate_tracer(ez, prm.ctypes.data, nexp, False, ctypes.byref(n),
                                          *[ctypes.byref(p) for p in ptrs], ctypes.byref(err))
        return r, err.value


def _apis():
    out = [("b200", _Api(_lib.load(64)))]
    if has_ref():
        from oracle.pyoracle import RefLib
        out.append(("ref", _Api(RefLib(64).lib)))
    return out


def _script(api, k, P):
    """A sequence of invalid and valid host-side calls; returns the codes."""
    codes = []
    for args in [(0.0, 16, 1, 1), (-5.0, 16, 1, 1), (100.0, 0, 1, 1), (100.0, 70000, 1, 1),
                 (100.0, 16, 2, 1), (100.0, 16, 1, 0)]:
        ez, e = api.init(*args)
        codes.append(("init", e, ez is None))
    ez, e = api.init(100.0, 16, 1, 1, -1)
    codes.append(("init-thread", e))
    ez, e = api.init(200.0, 16, 1, 7)
    assert e == 0
    codes.append(("pk-before-cosmo", api.pk(ez, k, P)))
    codes.append(("cosmo-bad", api.cosmo(ez, 0.0, 0.0, True, -1.0, 0.0, 0.31, 0.0, -1.0)))
    codes.append(("cosmo-w", api.cosmo(ez, 0.0, 0.0, True, 0.5, 0.0, 0.31, 0.0, -0.2)))
    codes.append(("cosmo-direct-bad", api.cosmo(ez, -1.0, 1.0, False, 0, 0, 0, 0, 0)))
    codes.append(("cosmo-null", api.cosmo(None, 1.0, 1.0, False, 0, 0, 0, 0, 0)))
    codes.append(("cosmo-ok", api.cosmo(ez, 0.0, 0.0, True, 0.8, 0.0, 0.31, 0.0, -1.0)))
    codes.append(("pk-nbin", api.pk(ez, k[:3], P[:3])))
    kb = k.copy(); kb[5] = kb[4]
    codes.append(("pk-nonasc", api.pk(ez, kb, P)))
    Pb = P.copy(); Pb[7] = -1
    codes.append(("pk-nonpos", api.pk(ez, k, Pb)))
    Pb = P.copy(); Pb[7] = np.inf
    codes.append(("pk-finite", api.pk(ez, k, Pb)))
    codes.append(("pk-range", api.pk(ez, k[400:], P[400:])))
    codes.append(("pk-bao-null", api.pk(ez, k, P, None, 1.0)))
    codes.append(("pk-bao-bad", api.pk(ez, k, P, P * 10, 50.0)))
    codes.append(("populate-no-field", api.populate(ez, [0.6, 15, 0.35, 300], 2400)))
    codes.append(("populate-lowexp", api.populate(ez, [0.6, 15, 0.35, 300], 100)))
    codes.append(("populate-hiexp", api.populate(ez, [0.6, 15, 0.35, 300], 16 ** 3)))
    codes.append(("pk-ok", api.pk(ez, k, P)))
    # sticky error: a call with *err already set returns it unchanged
    err = ctypes.c_int(23)
    r = api.L.EZmock_setup_linear_pk(ez, k.ctypes.data, len(k), P.ctypes.data, None, 0.0,
                                     False, ctypes.byref(err))
    codes.append(("sticky", r, err.value))
    api.L.EZmock_destroy(ez)
    return codes


def test_error_codes_match_reference(pk_table):
    k, P = pk_table
    res = {name: _script(api, k, P) for name, api in _apis()}
    ours = res["b200"]
    assert ours[0] == ("init", 7, True)
    assert ours[3] == ("init", 8, True)
    assert ours[4] == ("init", 9, True)
    assert ours[5] == ("init", 10, True)
    if "ref" in res:
        assert ours == res["ref"]


def test_growth_matches_reference_struct():
    """The cosmo sub-structure keeps {growth2, vfac} as its first members,
    which the reference CLI reads (src/main/run_mock.c:119-121)."""
    api = _Api(_lib.load(64))
    ez, e = api.init(1000.0, 32, 1, 1)
    assert e == 0
    api.cosmo(ez, 0.0, 0.0, True, 0.8, 0.0, 0.31, 0.0, -1.0)
    cosmo = ctypes.cast(ez, ctypes.POINTER(_vp * 6)).contents[2]
    g2, vf = (ctypes.c_double * 2).from_address(cosmo)
    from oracle.pyoracle import Oracle
    og2, ovf = Oracle(64).growth(0.8, 0.0, 0.31)
    assert g2 == og2 and vf == ovf
    api.L.EZmock_destroy(ez)


def test_python_wrapper_interface(pk_table):
    """ezmock_b200.EZmock exposes the reference wrapper's methods and raises
    RuntimeError with the library's message."""
    from ezmock_b200 import EZmock
    for name in ["set_growth_params", "eval_growth_params", "setup_linear_pk",
                 "create_dens_field_from_ic", "create_dens_field_from_wn",
                 "create_dens_field_from_disp", "populate_tracer", "populate_tracer_to_file"]:
        assert callable(getattr(EZmock, name))
    with pytest.raises(KeyError):
        EZmock(Ngrid=16)
    with pytest.raises(RuntimeError, match="invalid grid size"):
        EZmock(Lbox=100.0, Ngrid=15)
    m = EZmock(Lbox=200.0, Ngrid=16)
    with pytest.raises(RuntimeError, match="EZmock cosmology uninitialized"):
        m.setup_linear_pk(*pk_table)
    # errors are sticky, as in the reference wrapper (the return value is
    # stored back into the instance's error code)
    with pytest.raises(RuntimeError, match="EZmock cosmology uninitialized"):
        m.eval_growth_params(0.8, 0.31)
    m = EZmock(Lbox=200.0, Ngrid=16)
    m.eval_growth_params(0.8, 0.31)
    with pytest.raises(RuntimeError, match="k range insufficient"):
        m.setup_linear_pk(pk_table[0][500:], pk_table[1][500:])


def test_extension_options():
    """EZmockB200_set_option (include/ezmock_b200.h) accepts each option's
    documented values and rejects the others with the sticky argument error,
    on the host (no GPU work)."""
    from ezmock_b200 import EZmock
    valid = {1: [0, 1], 2: [0, 1], 3: [0, 1], 4: [1, 12345], 5: [2, 3], 6: [0, 64, 2048],
             7: [16, 32], 8: [0, 1], 9: [0, 1], 10: [0, 1]}
    invalid = {3: [-1], 4: [0, -5], 5: [1, 4], 6: [-1], 7: [8, 64], 8: [2, -1], 9: [2],
               10: [2, -1], 11: [0], 0: [0]}
    for opt, vals in valid.items():
        m = EZmock(Lbox=200.0, Ngrid=16)
        for v in vals:
            m.set_option(opt, v)
    for opt, vals in invalid.items():
        for v in vals:
            m = EZmock(Lbox=200.0, Ngrid=16)
            with pytest.raises(RuntimeError):
                m.set_option(opt, v)
            # the error is sticky: a valid call afterwards still fails
            with pytest.raises(RuntimeError):
                m.set_option(2, 0)
