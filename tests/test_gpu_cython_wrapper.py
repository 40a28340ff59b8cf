"""The reference's own Python package as a caller of the GPU library.

oracle/Makefile (`make cython REF=<reference tree>`) compiles the reference's
Cython wrapper, python/EZmock/EZmock.pyx with python/EZmock/cEZmock.pxd,
unmodified, against include/EZmock.h and links it to
ezmock_b200/lib/libEZmock_f32.so, as python/setup.py:48-70 does with its own
libEZmock.so.  The module it builds (oracle/_ref/cython/EZmock) is the
reference's class; these tests drive a mock through it and check that it
gives the catalogue of the ctypes mirror ezmock_b200.EZmock bit for bit, and
the same file from populate_tracer_to_file.
"""
import importlib
import os
import sys

import numpy as np
import pytest

from ezmock_b200 import EZmock as Mirror
from ezmock_b200.workloads import bbks_pk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CYDIR = os.path.join(ROOT, "oracle", "_ref", "cython")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(CYDIR, "EZmock")),
                                reason="reference Cython wrapper not built")


def reference_package():
    if CYDIR not in sys.path:
        sys.path.insert(0, CYDIR)
    return importlib.import_module("EZmock")


def test_wrapper_loads_gpu_library():
    """The compiled wrapper resolves its EZmock_* symbols from the GPU
    library (host-side calls only: no GPU needed)."""
    mod = reference_package()
    so = [f for f in os.listdir(os.path.join(CYDIR, "EZmock")) if f.endswith(".so")]
    assert so
    m = mod.EZmock(Lbox=500.0, Ngrid=64, rng=1, seed=3)
    m.eval_growth_params(0.8, 0.31)
    with pytest.raises(RuntimeError, match="power spectrum uninitialized"):
        m.create_dens_field_from_ic()
    maps = open("/proc/self/maps").read()
    assert "libEZmock_f32.so" in maps


@pytest.mark.gpu
@pytest.mark.parametrize("rng,seed,fixamp,iphase", [(1, 3, False, False), (0, 8, True, True)])
def test_wrapper_matches_mirror(tmp_path, rng, seed, fixamp, iphase):
    mod = reference_package()
    k, P = bbks_pk()
    Ng, L = 64, 500.0
    params = (0.6, 15.0, 0.35, 300.0)
    nexp = int(3e-4 * L ** 3)
    out = []
    for cls in (mod.EZmock, Mirror):
        m = cls(Lbox=L, Ngrid=Ng, rng=rng, seed=seed)
        m.eval_growth_params(0.8, 0.31)
        m.setup_linear_pk(k, P)
        m.create_dens_field_from_ic(fixamp=fixamp, iphase=iphase)
        cat = m.populate_tracer(*params, nexp)
        fn = tmp_path / f"{cls.__module__}.txt"
        m.populate_tracer_to_file(*params, nexp, str(fn), rsd_fac=0.0114)
        out.append((cat, fn.read_bytes()))
        del m
    (ca, fa), (cb, fb) = out
    assert len(ca[0]) == len(cb[0]) > 1000
    for a in range(6):
        assert ca[a].dtype == np.float32
        assert np.array_equal(ca[a], cb[a])
    assert fa == fb
