"""att_part = true on the GPU (tracers attached to particles,
pop_tracer.c:517-582, :804-879) against the oracle run on the GPU's own
displacement and density fields."""
import numpy as np
import pytest

from ezmock_b200 import EZmock
from ezmock_b200.workloads import bbks_pk
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

VTOL = {64: 1e-9, 32: 1e-4}


@pytest.fixture(scope="module")
def pk_table():
    return bbks_pk()


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("rng", [0, 1])
@pytest.mark.parametrize("params,n", [([0.6, 15.0, 0.35, 300.0], 3e-4),
                                      ([1.2, 5.0, 0.2, 150.0], 1e-4),
                                      ([0.0, 10.0, 0.3, 0.0], 1e-3)])
def test_attached_tracers(pk_table, prec, rng, params, n):
    k, P = pk_table
    Ng, L, seed = 48, 400.0, 7
    m = EZmock(Lbox=L, Ngrid=Ng, rng=rng, seed=seed, prec=prec)
    m.eval_growth_params(0.8, 0.31)
    m.setup_linear_pk(k, P)
    m.create_dens_field_from_ic()
    nexp = int(n * L ** 3)
    cat = m.populate_tracer(*params, nexp, att_part=True)
    O = Oracle(prec)
    _, vf = O.growth(0.8, 0.0, 0.31)
    e, ref = O.populate(Ng, L, rng, seed, vf, [m.field(d).ravel() for d in range(3)],
                        m.field(3).ravel(), params, nexp, att_part=True)
    assert e == 0 and len(ref[0]) == len(cat[0])
    for a in range(3):
        assert np.array_equal(cat[a], ref[a])
    vmax = np.abs(np.stack(ref[3:])).max()
    for a in range(3, 6):
        assert np.abs(cat[a] - ref[a]).max() <= VTOL[prec] * vmax
    # a later population without attachment on the same field is unaffected
    plain = m.populate_tracer(*params, nexp)
    e, pref = O.populate(Ng, L, rng, seed, vf, [m.field(d).ravel() for d in range(3)],
                         m.field(3).ravel(), params, nexp)
    assert len(plain[0]) == len(pref[0])
    for a in range(3):
        assert np.array_equal(plain[a], pref[a])
