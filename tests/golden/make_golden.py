"""Generate the golden vectors in tests/golden/ from the reference's own
libEZmock sources (built unmodified by `make -C oracle ref`, against the
oracle's prand and FFTW stand-ins).

Run from the repository root:  python tests/golden/make_golden.py
The reference tree is only needed here; the fixtures are committed.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import RefLib, build  # noqa: E402
from ezmock_b200.workloads import bbks_pk  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def raw_draws(ref_prec_lib, rng, seed, start, count):
    # prand restatement is linked into the reference build; expose it through
    # the oracle library, which shares the same prand sources
    from oracle.pyoracle import Oracle
    return Oracle(64).rng_raw(rng, seed, start, count)


def main():
    build(ref=True)
    k, P = bbks_pk()
    out = {}
    # -- random streams (prand restatement, as linked into the reference build)
    for rng in (0, 1):
        for seed in (1, 7, (1 << 40) + 5):
            for start in (0, 1000, (1 << 22) + 3, (1 << 28) + 777):
                out[f"rng{rng}_s{seed}_o{start}"] = raw_draws(None, rng, seed, start, 64)
    # -- growth factors
    R = RefLib(64, nthread=1)
    cos = []
    for z, zpk, om, onu, w in [(0.8, 0.0, 0.31, 0.0, -1.0), (0.5, 0.0, 0.3, 0.0, -0.9),
                               (1.5, 0.5, 0.25, 0.01, -1.1), (0.0, 0.0, 0.31, 0.0, -1.0)]:
        m = R.new(1000.0, 16, 1, 1)
        g2, vf = m.eval_growth(z, om, zpk, onu, w)
        cos.append([z, zpk, om, onu, w, g2, vf])
    out["cosmo"] = np.array(cos)
    # -- fields and catalogues at 16^3, box 200 Mpc/h
    Ng, L = 16, 200.0
    params = [0.6, 15.0, 0.35, 300.0]
    nexp = int(round(3e-4 * L ** 3))
    for prec in (64, 32):
        Rp = RefLib(prec, nthread=1)
        for rng in (0, 1):
            for fixamp, iphase in ((False, False), (True, True)):
                m = Rp.new(L, Ng, rng, 7)
                g2, vf = m.eval_growth(0.8, 0.31)
                m.setup_pk(k, P)
                m.create(fixamp=fixamp, iphase=iphase)
                tag = f"f{prec}_rng{rng}_fa{int(fixamp)}"
                out[tag + "_psi"] = np.stack([m.field(d) for d in range(3)])
                out[tag + "_rho"] = m.field(3)
                if fixamp:
                    continue
                rhot, nt, hist, pdf, ncell, ntot = m.bias_select(params, nexp)
                out[tag + "_rhot"] = rhot
                out[tag + "_nt"] = nt
                out[tag + "_hist"] = hist.astype(np.int64)
                out[tag + "_pdf"] = pdf.astype(np.int64)
                out[tag + "_counts"] = np.array([ncell, ntot], np.int64)
                m2 = Rp.new(L, Ng, rng, 7)
                m2.eval_growth(0.8, 0.31)
                m2.setup_pk(k, P)
                m2.create()
                out[tag + "_cat"] = np.stack(m2.populate(params, nexp))
    # -- selection with ties (reference n_tracer_in_cell on an injected field)
    rs = np.random.default_rng(11)
    Rp = RefLib(64, nthread=1)
    m = Rp.new(L, Ng, 1, 3)
    m.eval_growth(0.8, 0.31)
    m.setup_pk(k, P)
    m.create()
    vals = np.exp(rs.uniform(-3, 3.5, 400))
    rhot = vals[rs.integers(0, 400, Ng ** 3)]
    rhot[rs.random(Ng ** 3) < 0.3] = 0
    hist = np.zeros(64, np.uintp)
    for v in rhot[rhot > 0]:
        hist[min(max(5 - int(np.floor(np.log2(v))), 0), 63)] += 1
    from oracle.pyoracle import Oracle
    e, pdf, nmax, ncell, ntot = Oracle(64).eval_pdf(Ng, 700, 0.4)
    nt, pdf_out, nc, no = m.select_from(rhot, hist, pdf, nmax, ncell, ntot)
    out["ties_rhot"] = rhot.reshape(Ng, Ng, Ng)
    out["ties_hist"] = hist.astype(np.int64)
    out["ties_pdf_in"] = pdf.astype(np.int64)
    out["ties_in"] = np.array([nmax, ncell, ntot], np.int64)
    out["ties_nt"] = nt
    out["ties_pdf_out"] = pdf_out.astype(np.int64)
    out["ties_out"] = np.array([nc, no], np.int64)
    np.savez_compressed(os.path.join(OUT, "reference_16.npz"), **out)
    print("wrote", os.path.join(OUT, "reference_16.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
