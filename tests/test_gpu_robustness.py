"""Host-side failure paths on the GPU, none of which faults the device.

* Out of device memory: a 2048^3 FP32 instance needs about 380 GB of device
  buffers (three spectra, three displacement fields, the density, three
  painted grids, the random draws), a 1536^3 FP64 one about 490 GB, more than
  one B200 holds.  Creating its
  field must fail with EZMOCK_ERR_MEMORY (libEZmock/EZmock/errmsg.h:33-88,
  the reference's code for a failed allocation), keep the error sticky, free
  what was allocated, and leave the device usable for the next instance.
"""
import ctypes

import numpy as np
import pytest

from ezmock_b200 import EZmock, _lib
from ezmock_b200.workloads import bbks_pk

pytestmark = pytest.mark.gpu

ERR_MEMORY = 1


@pytest.mark.parametrize("prec", [32, 64])
def test_out_of_device_memory(prec):
    L = _lib.load(prec)
    k, P = bbks_pk()
    # the largest grid of each build's transforms: about 380 GB (FP32) and
    # 490 GB (FP64, 1536^3) of device buffers
    m = EZmock(Lbox=20000.0, Ngrid=2048 if prec == 32 else 1536, rng=1, seed=1, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P)
    with pytest.raises(RuntimeError, match="failed to allocate memory"):
        m.create_dens_field_from_ic()
    assert m._err.value == ERR_MEMORY
    # sticky: the next call returns the same code without doing anything
    err = ctypes.c_int(ERR_MEMORY)
    assert L.EZmock_create_dens_field(m._ez, None, False, None, False, False,
                                      ctypes.byref(err)) == ERR_MEMORY
    del m                                  # EZmock_destroy of the failed instance
    # the device is still usable: a small mock with its catalogue
    s = EZmock(Lbox=250.0, Ngrid=32, rng=1, seed=2, prec=prec)
    s.eval_growth_params(0.8, 0.31)
    s.setup_linear_pk(k, P)
    s.create_dens_field_from_ic()
    cat = s.populate_tracer(0.6, 15.0, 0.35, 300.0, int(3e-4 * 250.0 ** 3))
    assert len(cat[0]) > 0 and np.all(np.isfinite(cat[5]))
