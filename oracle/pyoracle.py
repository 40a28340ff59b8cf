"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries are exposed:

* ``Oracle`` -- the restatement in ``oracle/ezoracle.c`` (built by
  ``make -C oracle``), stage by stage;
* ``RefLib`` -- the reference's own libEZmock sources compiled unmodified by
  ``make -C oracle ref`` (needs the reference tree at build time; the built
  ``oracle/_ref/*.so`` travel with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(_HERE, "_build")
REFDIR = os.path.join(_HERE, "_ref")

_c_size_p = ctypes.POINTER(ctypes.c_size_t)
_vp = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def build(ref=False):
    """Compile the oracle (and, with ref=True, the reference build)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", _HERE, "ref"], check=True)


class PkTable(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("log", ctypes.c_int),
                ("kmin", ctypes.c_double), ("kmax", ctypes.c_double),
                ("k", ctypes.c_double * 8192), ("P", ctypes.c_double * 8192),
                ("P2", ctypes.c_double * 8192)]


class Oracle:
    """The restatement, in FP64 (``prec=64``) or FP32 (``prec=32``)."""

    def __init__(self, prec=64):
        path = os.path.join(BUILD, f"libezoracle_f{prec}.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        self.prec = prec
        self.rdt = np.float64 if prec == 64 else np.float32
        L = self.lib
        L.ezo_pk_interp.restype = ctypes.c_double
        L.ezo_pk_interp.argtypes = [ctypes.POINTER(PkTable), ctypes.c_double]
        L.ezo_growth.argtypes = [ctypes.c_double] * 5 + [ctypes.POINTER(ctypes.c_double)] * 2
        L.ezo_pk_setup.argtypes = [ctypes.POINTER(PkTable), ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, _vp, ctypes.c_int, _vp, _vp,
                                   ctypes.c_double, ctypes.c_int]
        L.ezo_ic_spectrum.argtypes = [ctypes.POINTER(PkTable), ctypes.c_int, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                      ctypes.c_int, _vp]
        L.ezo_disp_from_spectrum.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int]
        L.ezo_disp_whitenoise.argtypes = [ctypes.POINTER(PkTable), ctypes.c_int,
                                          ctypes.c_double, _vp, _vp, _vp, _vp, ctypes.c_int]
        L.ezo_cic.argtypes = [ctypes.c_int, ctypes.c_double, _vp, _vp, _vp, _vp]
        rt = ctypes.c_float if prec == 32 else ctypes.c_double
        self._rt = rt
        L.ezo_eval_pdf.argtypes = [ctypes.c_int, ctypes.c_size_t, rt, _vp,
                                   ctypes.POINTER(ctypes.c_int), _c_size_p, _c_size_p]
        L.ezo_bias.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _vp, rt, rt,
                               ctypes.c_size_t, _vp, _vp, _c_size_p]
        L.ezo_select.argtypes = [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _c_size_p,
                                 _c_size_p, _vp]
        L.ezo_positions.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_uint64, _vp, ctypes.c_size_t, _vp, _vp, _vp]
        L.ezo_paint.argtypes = [ctypes.c_int, ctypes.c_double, _vp, _vp, _vp, _vp,
                                ctypes.c_int, _vp]
        L.ezo_assign_vel.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _vp,
                                     _vp, ctypes.c_size_t, _vp, _vp, _vp, _vp]
        L.ezo_vel_scatter.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                      ctypes.c_size_t, rt, _vp, _vp, _vp]
        L.ezo_rsd.argtypes = [ctypes.c_size_t, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp]
        L.ezo_populate.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_uint64, ctypes.c_double, _vp, _vp, _vp, _vp,
                                   _vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t,
                                   _c_size_p, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ezo_rng_raw.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                  ctypes.c_uint64, _vp]

    # --- host-side scalars -------------------------------------------------
    def growth(self, z, z_pk, Om, Onu=0.0, w=-1.0):
        g2, vf = ctypes.c_double(), ctypes.c_double()
        e = self.lib.ezo_growth(z, z_pk, Om, Onu, w, ctypes.byref(g2), ctypes.byref(vf))
        if e:
            raise RuntimeError(f"ezo_growth error {e}")
        return g2.value, vf.value

    def pk_setup(self, Ng, Lbox, growth2, k, P, Pnw=None, mBAO=0.0, logint=False):
        t = PkTable()
        k = np.ascontiguousarray(k, np.float64)
        P = np.ascontiguousarray(P, np.float64)
        Pnw = None if Pnw is None else np.ascontiguousarray(Pnw, np.float64)
        e = self.lib.ezo_pk_setup(ctypes.byref(t), Ng, Lbox, growth2, _ptr(k), len(k),
                                  _ptr(P), _ptr(Pnw), mBAO, int(logint))
        if e:
            raise RuntimeError(f"ezo_pk_setup error {e}")
        return t

    def pk_interp(self, table, kv):
        return self.lib.ezo_pk_interp(ctypes.byref(table), kv)

    # --- fields ------------------------------------------------------------
    def ic_spectrum(self, table, Ng, Lbox, rng, seed, fixamp=False, iphase=False):
        out = np.zeros((Ng, Ng, Ng // 2 + 1, 2), self.rdt)
        e = self.lib.ezo_ic_spectrum(ctypes.byref(table), Ng, Lbox, rng, seed,
                                     int(fixamp), int(iphase), _ptr(out))
        if e:
            raise RuntimeError(f"ezo_ic_spectrum error {e}")
        return out

    def disp_from_spectrum(self, Ng, rhok, nthread=0):
        psi = [np.zeros((Ng, Ng, Ng), self.rdt) for _ in range(3)]
        rhok = np.ascontiguousarray(rhok, self.rdt)
        self.lib.ezo_disp_from_spectrum(Ng, _ptr(rhok), *[_ptr(p) for p in psi], nthread)
        return psi

    def disp_whitenoise(self, table, Ng, Lbox, delta, nthread=0):
        psi = [np.zeros((Ng, Ng, Ng), self.rdt) for _ in range(3)]
        delta = np.ascontiguousarray(delta, self.rdt)
        self.lib.ezo_disp_whitenoise(ctypes.byref(table), Ng, Lbox, _ptr(delta),
                                     *[_ptr(p) for p in psi], nthread)
        return psi

    def cic(self, Ng, Lbox, psi):
        rho = np.zeros((Ng, Ng, Ng), self.rdt)
        psi = [np.ascontiguousarray(p, self.rdt) for p in psi]
        self.lib.ezo_cic(Ng, Lbox, *[_ptr(p) for p in psi], _ptr(rho))
        return rho

    def dens_field(self, table, Ng, Lbox, rng, seed, fixamp=False, iphase=False):
        rhok = self.ic_spectrum(table, Ng, Lbox, rng, seed, fixamp, iphase)
        psi = self.disp_from_spectrum(Ng, rhok)
        return psi, self.cic(Ng, Lbox, psi)

    # --- population stages ---------------------------------------------------
    def eval_pdf(self, Ng, nexp, pbase):
        pdf = np.zeros(1025, np.uintp)
        nmax, ncell, ntot = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
        e = self.lib.ezo_eval_pdf(Ng, nexp, self._rt(pbase), _ptr(pdf), ctypes.byref(nmax),
                                  ctypes.byref(ncell), ctypes.byref(ntot))
        return e, pdf[:nmax.value].copy(), nmax.value, ncell.value, ntot.value

    def bias(self, Ng, rng, seed, rho, rho_c, rho_exp, ncell):
        rho = np.ascontiguousarray(rho, self.rdt)
        rhot = np.zeros_like(rho)
        hist = np.zeros(64, np.uintp)
        nv = ctypes.c_size_t()
        e = self.lib.ezo_bias(Ng, rng, seed, _ptr(rho), self._rt(rho_c), self._rt(rho_exp),
                              ncell, _ptr(rhot), _ptr(hist), ctypes.byref(nv))
        return e, rhot, hist, nv.value

    def select(self, Ng, rhot, hist, pdf, nmax, ncell, ntot):
        pdf = np.array(pdf, np.uintp)
        hist = np.ascontiguousarray(hist, np.uintp)
        nt = np.zeros(rhot.shape, np.int16)
        nc, no = ctypes.c_size_t(ncell), ctypes.c_size_t(ntot)
        e = self.lib.ezo_select(Ng, _ptr(np.ascontiguousarray(rhot, self.rdt)), _ptr(hist),
                                _ptr(pdf), nmax, ctypes.byref(nc), ctypes.byref(no), _ptr(nt))
        return e, nt, pdf, nc.value, no.value

    def positions(self, Ng, Lbox, rng, seed, nt, ntot):
        x, y, z = (np.zeros(ntot, self.rdt) for _ in range(3))
        e = self.lib.ezo_positions(Ng, Lbox, rng, seed, _ptr(np.ascontiguousarray(nt)),
                                   ntot, _ptr(x), _ptr(y), _ptr(z))
        return e, x, y, z

    def paint(self, Ng, Lbox, psi, rho, dim):
        out = np.zeros((Ng, Ng, Ng), self.rdt)
        self.lib.ezo_paint(Ng, Lbox, *[_ptr(np.ascontiguousarray(p, self.rdt)) for p in psi],
                           _ptr(np.ascontiguousarray(rho, self.rdt)), dim, _ptr(out))
        return out

    def assign_vel(self, Ng, Lbox, vfac, painted, rho, x, y, z):
        v = np.zeros(len(x), self.rdt)
        self.lib.ezo_assign_vel(Ng, Lbox, vfac, _ptr(painted), _ptr(rho), len(x),
                                _ptr(x), _ptr(y), _ptr(z), _ptr(v))
        return v

    def vel_scatter(self, Ng, rng, seed, sigma_v, vx, vy, vz):
        vx, vy, vz = (np.array(a, self.rdt) for a in (vx, vy, vz))
        self.lib.ezo_vel_scatter(Ng, rng, seed, len(vx), self._rt(sigma_v),
                                 _ptr(vx), _ptr(vy), _ptr(vz))
        return vx, vy, vz

    def rsd(self, z, vz, rsd_fac, Lbox):
        out = np.zeros(len(z), np.float64)
        self.lib.ezo_rsd(len(z), _ptr(np.ascontiguousarray(z, self.rdt)),
                         _ptr(np.ascontiguousarray(vz, self.rdt)), rsd_fac, Lbox, _ptr(out))
        return out

    def populate(self, Ng, Lbox, rng, seed, vfac, psi, rho, params, nexp, cap=None,
                 att_part=False):
        if cap is None:
            cap = 4 * nexp + 1024
        prm = np.array(params, self.rdt)
        cat = [np.zeros(cap, self.rdt) for _ in range(6)]
        n = ctypes.c_size_t()
        psi = [np.ascontiguousarray(p, self.rdt) for p in psi]
        e = self.lib.ezo_populate(Ng, Lbox, rng, seed, vfac, *[_ptr(p) for p in psi],
                                  _ptr(np.ascontiguousarray(rho, self.rdt)), _ptr(prm), nexp,
                                  int(bool(att_part)), cap, ctypes.byref(n),
                                  *[_ptr(c) for c in cat])
        if e:
            return e, None
        return 0, [c[:n.value].copy() for c in cat]

    def rng_raw(self, rng, seed, start, count):
        out = np.zeros(count, np.uint32)
        self.lib.ezo_rng_raw(rng, seed, start, count, _ptr(out))
        return out


class RefLib:
    """The reference's libEZmock (unmodified sources) through its C API."""

    def __init__(self, prec=64, nthread=1):
        path = os.path.join(REFDIR, f"libezref_f{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = ctypes.CDLL(path)
        self.prec = prec
        self.rdt = np.float64 if prec == 64 else np.float32
        self.nthread = nthread
        ip = ctypes.POINTER(ctypes.c_int)
        L.EZmock_init.restype = _vp
        L.EZmock_init.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                  ctypes.c_int, ip]
        L.EZmock_set_cosmology.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_bool,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ip]
        L.EZmock_setup_linear_pk.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_double,
                                             ctypes.c_bool, ip]
        L.EZmock_create_dens_field.argtypes = [_vp, _vp, ctypes.c_bool, _vp, ctypes.c_bool,
                                               ctypes.c_bool, ip]
        pp = ctypes.POINTER(_vp)
        L.EZmock_populate_tracer.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_bool, _c_size_p,
                                             pp, pp, pp, pp, pp, pp, ip]
        L.EZmock_destroy.argtypes = [_vp]
        L.EZmock_errmsg.restype = ctypes.c_char_p
        L.EZmock_errmsg.argtypes = [ctypes.c_int]
        L.EZmock_write_ascii.restype = ctypes.c_int
        L.EZmock_write_ascii.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_size_t, ctypes.c_double,
                                                             ctypes.c_bool, ctypes.c_char_p, ip]
        L.ezref_mesh_ptr.restype = _vp
        L.ezref_mesh_ptr.argtypes = [_vp, ctypes.c_int]
        L.ezref_growth2.restype = ctypes.c_double
        L.ezref_growth2.argtypes = [_vp]
        L.ezref_vfac.restype = ctypes.c_double
        L.ezref_vfac.argtypes = [_vp]
        L.ezref_bias_select.argtypes = [_vp, _vp, ctypes.c_size_t, _vp, _vp, _vp, _vp,
                                        ip, _c_size_p, _c_size_p, ip]
        L.ezref_select_from.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int, ctypes.c_size_t,
                                        ctypes.c_size_t, _vp, _vp, _c_size_p, _c_size_p, ip]
        self._libc = ctypes.CDLL(None)
        self._libc.free.argtypes = [_vp]

    def new(self, Lbox, Ng, rng, seed):
        err = ctypes.c_int(0)
        ez = self.lib.EZmock_init(Lbox, Ng, rng, seed, self.nthread, ctypes.byref(err))
        if not ez:
            raise RuntimeError(self.lib.EZmock_errmsg(err.value).decode())
        return _RefMock(self, ez, Ng, Lbox)


class _RefMock:
    def __init__(self, owner, ez, Ng, Lbox):
        self.o, self.ez, self.Ng, self.Lbox = owner, ez, Ng, Lbox
        self.err = ctypes.c_int(0)

    def _chk(self):
        if self.err.value:
            raise RuntimeError(self.o.lib.EZmock_errmsg(self.err.value).decode())

    def __del__(self):
        try:
            self.o.lib.EZmock_destroy(self.ez)
        except Exception:
            pass

    def eval_growth(self, z, Om, z_pk=0.0, Onu=0.0, w=-1.0):
        self.o.lib.EZmock_set_cosmology(self.ez, 0.0, 0.0, True, z, z_pk, Om, Onu, w,
                                        ctypes.byref(self.err))
        self._chk()
        return self.o.lib.ezref_growth2(self.ez), self.o.lib.ezref_vfac(self.ez)

    def setup_pk(self, k, P, Pnw=None, mBAO=0.0, logint=False):
        k = np.ascontiguousarray(k, np.float64)
        P = np.ascontiguousarray(P, np.float64)
        Pnw = None if Pnw is None else np.ascontiguousarray(Pnw, np.float64)
        self.o.lib.EZmock_setup_linear_pk(self.ez, _ptr(k), len(k), _ptr(P), _ptr(Pnw), mBAO,
                                          logint, ctypes.byref(self.err))
        self._chk()

    def create(self, fixamp=False, iphase=False, delta=None):
        d = None if delta is None else np.ascontiguousarray(delta, self.o.rdt)
        self._delta = d
        self.o.lib.EZmock_create_dens_field(self.ez, None, False, _ptr(d), fixamp, iphase,
                                            ctypes.byref(self.err))
        self._chk()

    def field(self, which):
        p = self.o.lib.ezref_mesh_ptr(self.ez, which)
        n = self.Ng ** 3
        buf = (ctypes.c_char * (n * np.dtype(self.o.rdt).itemsize)).from_address(p)
        return np.frombuffer(buf, self.o.rdt).reshape(self.Ng, self.Ng, self.Ng).copy()

    def bias_select(self, params, nexp):
        n = self.Ng ** 3
        rhot = np.zeros(n, self.o.rdt)
        nt = np.zeros(n, np.int16)
        hist = np.zeros(64, np.uintp)
        pdf = np.zeros(1025, np.uintp)
        nmax, ncell, ntot = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
        prm = np.array(params, self.o.rdt)
        self.o.lib.ezref_bias_select(self.ez, _ptr(prm), nexp, _ptr(rhot), _ptr(nt), _ptr(hist),
                                     _ptr(pdf), ctypes.byref(nmax), ctypes.byref(ncell),
                                     ctypes.byref(ntot), ctypes.byref(self.err))
        self._chk()
        shp = (self.Ng,) * 3
        return (rhot.reshape(shp), nt.reshape(shp), hist, pdf[:nmax.value].copy(),
                ncell.value, ntot.value)

    def select_from(self, rhot, hist, pdf, nmax, ncell, ntot):
        n = self.Ng ** 3
        nt = np.zeros(n, np.int16)
        pdf_out = np.zeros(nmax, np.uintp)
        nc, no = ctypes.c_size_t(), ctypes.c_size_t()
        rhot = np.ascontiguousarray(rhot, self.o.rdt)
        self.o.lib.ezref_select_from(self.ez, _ptr(rhot), _ptr(np.ascontiguousarray(hist, np.uintp)),
                                     _ptr(np.ascontiguousarray(pdf, np.uintp)), nmax, ncell, ntot,
                                     _ptr(nt), _ptr(pdf_out), ctypes.byref(nc), ctypes.byref(no),
                                     ctypes.byref(self.err))
        self._chk()
        return nt.reshape((self.Ng,) * 3), pdf_out, nc.value, no.value

    def write_ascii(self, cat, fname, rsd_fac=0.0, header=True):
        """The reference's EZmock_write_ascii (save_res.c:95-178) on six
        arrays; returns its error code."""
        arrs = [np.ascontiguousarray(a, self.o.rdt) for a in cat]
        err = ctypes.c_int(0)
        self.o.lib.EZmock_write_ascii(self.ez, *[_ptr(a) for a in arrs], len(arrs[0]),
                                      float(rsd_fac), bool(header), str(fname).encode(),
                                      ctypes.byref(err))
        return err.value

    def populate(self, params, nexp, att_part=False):
        prm = np.array(params, self.o.rdt)
        n = ctypes.c_size_t()
        ptrs = [_vp() for _ in range(6)]
        self.o.lib.EZmock_populate_tracer(self.ez, _ptr(prm), nexp, bool(att_part),
                                          ctypes.byref(n),
                                          *[ctypes.byref(p) for p in ptrs],
                                          ctypes.byref(self.err))
        self._chk()
        out = []
        isz = np.dtype(self.o.rdt).itemsize
        for p in ptrs:
            buf = (ctypes.c_char * (n.value * isz)).from_address(p.value)
            out.append(np.frombuffer(buf, self.o.rdt).copy())
            self.o._libc.free(p)
        return out
