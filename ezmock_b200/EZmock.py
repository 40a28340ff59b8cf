"""Python interface of the B200 EZmock engine.

``EZmock`` mirrors the reference's Cython wrapper (python/EZmock/EZmock.pyx,
class EZmock at :36-485) method by method: same names, keyword arguments,
defaults, and RuntimeError messages taken from EZmock_errmsg.  The wrapper is
built in single precision in the reference (python/setup.py:56); here
``prec=32`` (default) loads libEZmock_f32.so and ``prec=64`` libEZmock_f64.so.
Catalogue arrays are returned as numpy arrays that own their memory.
"""
import ctypes

import numpy as np

from . import _lib

__all__ = ["EZmock"]

_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]
_libc.free.restype = None


def _owned_array(ptr, n, ctype):
    """numpy view of n `ctype` values at a malloc()'d pointer; the memory is
    released with free() once the array (and every view of it) is gone."""
    import weakref
    addr = ctypes.cast(ptr, ctypes.c_void_p).value
    if not n:
        _libc.free(addr)
        return np.zeros(0, np.dtype(ctype))
    buf = (ctype * n).from_address(addr)
    arr = np.frombuffer(buf, dtype=np.dtype(ctype))
    weakref.finalize(buf, _libc.free, addr)
    return arr


class EZmock:
    def __init__(self, *args, prec=32, **kwargs):
        """Lbox, Ngrid (required); rng (0: MRG32K3A, 1: MT19937, default 1);
        seed (default 1); nthread (default 0)."""
        if "Lbox" in kwargs:
            Lbox = float(kwargs["Lbox"])
        else:
            raise KeyError("`Lbox` is a required argument")
        if "Ngrid" in kwargs:
            Ngrid = int(kwargs["Ngrid"])
        else:
            raise KeyError("`Ngrid` is a required argument")
        rng = int(kwargs.get("rng", 1))
        seed = int(kwargs.get("seed", 1))
        nthread = int(kwargs.get("nthread", 0))
        self._L = _lib.load(prec)
        self._rdt = np.float32 if prec == 32 else np.float64
        self._err = ctypes.c_int(0)
        self._Ng = Ngrid
        self._Lbox = Lbox
        self._ez = self._L.EZmock_init(Lbox, Ngrid, rng, seed, nthread, ctypes.byref(self._err))
        if not self._ez:
            raise RuntimeError(self._L.EZmock_errmsg(self._err.value).decode("utf-8"))

    def __del__(self):
        ez = getattr(self, "_ez", None)
        if ez:
            self._L.EZmock_destroy(ez)
            self._ez = None

    def _assert_return_value(self):
        if self._err.value != 0:
            raise RuntimeError(self._L.EZmock_errmsg(self._err.value).decode("utf-8"))

    # -- EZmock.pyx:113-133
    def set_growth_params(self, growth_pk, vel_fac):
        self._err.value = self._L.EZmock_set_cosmology(
            self._ez, float(growth_pk), float(vel_fac), False, 0.0, 0.0, 0.0, 0.0, 0.0,
            ctypes.byref(self._err))
        self._assert_return_value()

    # -- EZmock.pyx:136-158
    def eval_growth_params(self, z_out, Omega_m, z_pk=0, Omega_nu=0, w=-1):
        self._err.value = self._L.EZmock_set_cosmology(
            self._ez, 0.0, 0.0, True, float(z_out), float(z_pk), float(Omega_m),
            float(Omega_nu), float(w), ctypes.byref(self._err))
        self._assert_return_value()

    # -- EZmock.pyx:161-226
    def setup_linear_pk(self, k, Plin, Pnw=None, BAO_enhance=0, interp_log=False):
        try:
            k = np.ascontiguousarray(np.asarray(k), dtype=np.float64)
            Plin = np.ascontiguousarray(np.asarray(Plin), dtype=np.float64)
        except Exception:
            raise TypeError("`k` and `Plin` are expected to be float numpy arrays")
        assert k.ndim == 1 and Plin.ndim == 1 and k.shape[0] == Plin.shape[0], \
            "`k` and `Plin` must be 1d arrays with the same length"
        if BAO_enhance != 0:
            try:
                Pnw = np.ascontiguousarray(np.asarray(Pnw), dtype=np.float64)
            except Exception:
                raise TypeError("`Pnw` is expected to be a float numpy array")
            assert Pnw.ndim == 1 and k.shape[0] == Pnw.shape[0], \
                "`Pnw` must be an 1d array with the same length as k"
            pnw = Pnw.ctypes.data_as(ctypes.c_void_p)
        else:
            pnw = None
        self._err.value = self._L.EZmock_setup_linear_pk(
            self._ez, k.ctypes.data_as(ctypes.c_void_p), k.shape[0],
            Plin.ctypes.data_as(ctypes.c_void_p), pnw, float(BAO_enhance),
            bool(interp_log), ctypes.byref(self._err))
        self._assert_return_value()

    # -- EZmock.pyx:229-251
    def create_dens_field_from_ic(self, fixamp=False, iphase=False):
        self._err.value = self._L.EZmock_create_dens_field(
            self._ez, None, False, None, bool(fixamp), bool(iphase), ctypes.byref(self._err))
        self._assert_return_value()

    # -- EZmock.pyx:254-283
    def create_dens_field_from_wn(self, delta):
        try:
            delta = np.ascontiguousarray(np.asarray(delta), dtype=self._rdt)
        except Exception:
            raise TypeError("`delta` is expected to be a float numpy array")
        assert delta.ndim == 1 and delta.shape[0] == self._Ng ** 3, \
            f"`delta` must be a 1d array with {self._Ng:d}**3 elements"
        self._err.value = self._L.EZmock_create_dens_field(
            self._ez, None, False, delta.ctypes.data_as(ctypes.c_void_p), False, False,
            ctypes.byref(self._err))
        self._assert_return_value()

    # -- EZmock.pyx:286-334
    def create_dens_field_from_disp(self, dx, dy, dz, deepcopy=False):
        try:
            dx, dy, dz = (np.ascontiguousarray(np.asarray(a), dtype=self._rdt)
                          for a in (dx, dy, dz))
        except Exception:
            raise TypeError("`dx`, `dy`, and `dz` must be float numpy arrays")
        ntot = self._Ng ** 3
        assert all(a.ndim == 1 and a.shape[0] == ntot for a in (dx, dy, dz)), \
            f"`dx`, `dy`, `dz` must be 1d arrays with {self._Ng:d}**3 elements"
        disp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in (dx, dy, dz)])
        self._err.value = self._L.EZmock_create_dens_field(
            self._ez, ctypes.cast(disp, ctypes.c_void_p), bool(deepcopy), None, False, False,
            ctypes.byref(self._err))
        self._assert_return_value()

    def _populate(self, rho_c, rho_exp, pdf_base, sigma_v, ntracer, att_part):
        rt = self._L._rt
        params = (rt * 4)(rho_c, rho_exp, pdf_base, sigma_v)
        ptrs = [ctypes.POINTER(rt)() for _ in range(6)]
        num = ctypes.c_size_t(0)
        self._err.value = self._L.EZmock_populate_tracer(
            self._ez, ctypes.cast(params, ctypes.c_void_p), int(ntracer), bool(att_part),
            ctypes.byref(num), *[ctypes.byref(p) for p in ptrs], ctypes.byref(self._err))
        self._assert_return_value()
        return num.value, ptrs

    # -- EZmock.pyx:337-405: the arrays own the library's malloc() memory
    #    (no copy), released with free() when numpy drops them
    def populate_tracer(self, rho_c, rho_exp, pdf_base, sigma_v, ntracer, att_part=False):
        n, ptrs = self._populate(rho_c, rho_exp, pdf_base, sigma_v, ntracer, att_part)
        return tuple(_owned_array(p, n, self._L._rt) for p in ptrs)

    # -- EZmock.pyx:408-485
    def populate_tracer_to_file(self, rho_c, rho_exp, pdf_base, sigma_v, ntracer, fname,
                                att_part=False, rsd_fac=0, header=True):
        n, ptrs = self._populate(rho_c, rho_exp, pdf_base, sigma_v, ntracer, att_part)
        self._err.value = self._L.EZmock_write_ascii(
            self._ez, *ptrs, n, float(rsd_fac), bool(header), str(fname).encode("utf-8"),
            ctypes.byref(self._err))
        libc = ctypes.CDLL(None)
        libc.free.argtypes = [ctypes.c_void_p]
        for p in ptrs:
            libc.free(ctypes.cast(p, ctypes.c_void_p))
        self._assert_return_value()

    # ---- extensions (no counterpart in the reference wrapper) ----
    def set_option(self, option, value):
        self._err.value = self._L.EZmockB200_set_option(self._ez, int(option), int(value),
                                                        ctypes.byref(self._err))
        self._assert_return_value()

    def select_path(self):
        """How the last selection found its boundaries: 0 value buckets, 1 full
        sort, 2 buckets then full sort."""
        return int(self._L.EZmockB200_select_path(self._ez))

    def field(self, which):
        """Copy of a device field: 0..2 psi, 3 rho, 4..6 painted displacements."""
        out = np.empty(self._Ng ** 3, self._rdt)
        self._err.value = self._L.EZmockB200_copy_field(
            self._ez, int(which), out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(self._err))
        self._assert_return_value()
        return out.reshape((self._Ng,) * 3)

    def stage_times(self):
        ms = (ctypes.c_double * 11)()
        n = self._L.EZmockB200_stage_times(self._ez, ms, 11)
        names = ["rng", "ic", "fft_i", "fft_j", "fft_k", "cic", "bias", "select", "emit",
                 "vel", "d2h"]
        return {names[i]: ms[i] for i in range(n)}

    def populate_device(self, rho_c, rho_exp, pdf_base, sigma_v, ntracer):
        rt = self._L._rt
        params = (rt * 4)(rho_c, rho_exp, pdf_base, sigma_v)
        num = ctypes.c_size_t(0)
        self._err.value = self._L.EZmockB200_populate_device(
            self._ez, ctypes.cast(params, ctypes.c_void_p), int(ntracer), ctypes.byref(num),
            ctypes.byref(self._err))
        self._assert_return_value()
        return num.value

    def sync(self):
        return self._L.EZmockB200_sync(self._ez)

    def _cat_args(self, cat):
        """(x, y, z, vz, n, keep-alive) for host arrays, or NULLs for the
        instance's last catalogue on the GPU."""
        if cat is None:
            return None, None, None, None, 0, None
        arrs = [np.ascontiguousarray(np.asarray(a), dtype=self._rdt) for a in cat]
        if len(arrs) not in (3, 4) or any(a.ndim != 1 or a.shape != arrs[0].shape for a in arrs):
            raise ValueError("catalogue: x, y, z[, vz] as 1d arrays of equal length")
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in arrs]
        if len(ptrs) == 3:
            ptrs.append(None)
        return ptrs[0], ptrs[1], ptrs[2], ptrs[3], arrs[0].shape[0], arrs

    def powspec(self, cat=None, rsd_fac=0.0, ngrid=256, interlace=True, kmin=0.0,
                kmax=0.3, nbin=30):
        """Power-spectrum multipoles of the last catalogue (cat=None, kept on
        the GPU) or of host arrays cat = (x, y, z[, vz]).  Returns a dict of
        k_mean, nmodes, P0, P2 (arrays of nbin)."""
        x, y, z, vz, n, keep = self._cat_args(cat)
        out = [np.zeros(int(nbin)) for _ in range(4)]
        dp = ctypes.POINTER(ctypes.c_double)
        self._err.value = self._L.EZmockB200_powspec(
            self._ez, x, y, z, vz, n, float(rsd_fac), int(ngrid), int(bool(interlace)),
            float(kmin), float(kmax), int(nbin), *[o.ctypes.data_as(dp) for o in out],
            ctypes.byref(self._err))
        del keep
        self._assert_return_value()
        return dict(zip(("k_mean", "nmodes", "P0", "P2"), out))

    def cic_pdf(self, cat=None, rsd_fac=0.0, ngrid=64, nbin=32):
        """Fraction of the ngrid^3 cells holding c = 0 .. nbin-2 tracers, and
        at least nbin-1 tracers in the last bin."""
        x, y, z, vz, n, keep = self._cat_args(cat)
        out = np.zeros(int(nbin))
        self._err.value = self._L.EZmockB200_cic_pdf(
            self._ez, x, y, z, vz, n, float(rsd_fac), int(ngrid), int(nbin),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(self._err))
        del keep
        self._assert_return_value()
        return out


def powspec_table(res, kmin=0.0, kmax=0.3):
    """Rows in the column order the reference's plotting reads
    (example/fit/pyclustering.py:249-251: k in column 0, P0 in 5, P2 in 6):
    k_center, k_low, k_high, k_mean, nmodes, P0, P2."""
    nb = len(res["P0"])
    edges = np.linspace(kmin, kmax, nb + 1)
    return np.column_stack([0.5 * (edges[:-1] + edges[1:]), edges[:-1], edges[1:],
                            res["k_mean"], res["nmodes"], res["P0"], res["P2"]])
