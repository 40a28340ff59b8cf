"""Loader for the in-tree C-ABI libraries ``lib/libEZmock_f32.so`` and
``lib/libEZmock_f64.so`` (built by ``make -C ezmock_b200/csrc``).

There is no CPU fallback: if the library is missing, loading raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(_HERE, "lib")
INCLUDE = os.path.join(os.path.dirname(_HERE), "include")

_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_sp = ctypes.POINTER(ctypes.c_size_t)

_cache = {}


def lib_path(prec):
    return os.path.join(LIBDIR, f"libEZmock_f{prec}.so")


def build():
    import subprocess
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(_HERE, "csrc")], check=True)


def load(prec=32):
    """The library for `real` = float (prec=32) or double (prec=64)."""
    if prec not in (32, 64):
        raise ValueError("prec must be 32 or 64")
    if prec in _cache:
        return _cache[prec]
    path = lib_path(prec)
    if not os.path.exists(path):
        raise ImportError(f"EZmock GPU library not built: {path} "
                          "(run `make -C ezmock_b200/csrc`)")
    L = ctypes.CDLL(path)
    rt = ctypes.c_float if prec == 32 else ctypes.c_double
    rp = ctypes.POINTER(rt)
    rpp = ctypes.POINTER(rp)
    L.EZmock_init.restype = _vp
    L.EZmock_init.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                              ctypes.c_int, _ip]
    L.EZmock_set_cosmology.restype = ctypes.c_int
    L.EZmock_set_cosmology.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_bool,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, _ip]
    L.EZmock_setup_linear_pk.restype = ctypes.c_int
    L.EZmock_setup_linear_pk.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_double,
                                         ctypes.c_bool, _ip]
    L.EZmock_create_dens_field.restype = ctypes.c_int
    L.EZmock_create_dens_field.argtypes = [_vp, _vp, ctypes.c_bool, _vp, ctypes.c_bool,
                                           ctypes.c_bool, _ip]
    L.EZmock_populate_tracer.restype = ctypes.c_int
    L.EZmock_populate_tracer.argtypes = [_vp, _vp, ctypes.c_size_t, ctypes.c_bool, _sp,
                                         rpp, rpp, rpp, rpp, rpp, rpp, _ip]
    L.EZmock_write_ascii.restype = ctypes.c_int
    L.EZmock_write_ascii.argtypes = [_vp, rp, rp, rp, rp, rp, rp, ctypes.c_size_t,
                                     ctypes.c_double, ctypes.c_bool, ctypes.c_char_p, _ip]
    L.EZmock_destroy.restype = None
    L.EZmock_destroy.argtypes = [_vp]
    L.EZmock_errmsg.restype = ctypes.c_char_p
    L.EZmock_errmsg.argtypes = [ctypes.c_int]
    L.EZmockB200_set_option.restype = ctypes.c_int
    L.EZmockB200_set_option.argtypes = [_vp, ctypes.c_int, ctypes.c_long, _ip]
    L.EZmockB200_stage_times.restype = ctypes.c_int
    L.EZmockB200_stage_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.EZmockB200_copy_field.restype = ctypes.c_int
    L.EZmockB200_copy_field.argtypes = [_vp, ctypes.c_int, _vp, _ip]
    L.EZmockB200_populate_device.restype = ctypes.c_int
    L.EZmockB200_populate_device.argtypes = [_vp, _vp, ctypes.c_size_t, _sp, _ip]
    L.EZmockB200_copy_catalog.restype = ctypes.c_int
    L.EZmockB200_copy_catalog.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, _ip]
    L.EZmockB200_select_counts.restype = ctypes.c_int
    L.EZmockB200_select_counts.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_int, _sp, _sp, _vp, _ip]
    L.EZmockB200_rng_raw.restype = ctypes.c_int
    L.EZmockB200_rng_raw.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                     ctypes.c_uint64, _vp]
    L.EZmockB200_mt19937_fill_noalloc.restype = ctypes.c_int
    L.EZmockB200_mt19937_fill_noalloc.argtypes = [ctypes.c_uint64, ctypes.c_uint64,
                                                  ctypes.c_uint64, _vp, _vp]
    dp = ctypes.POINTER(ctypes.c_double)
    L.EZmockB200_powspec.restype = ctypes.c_int
    L.EZmockB200_powspec.argtypes = [_vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, _ip]
    L.EZmockB200_cic_pdf.restype = ctypes.c_int
    L.EZmockB200_cic_pdf.argtypes = [_vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, dp, _ip]
    L.EZmockB200_sync.restype = ctypes.c_int
    L.EZmockB200_sync.argtypes = [_vp]
    L.EZmockB200_real_size.restype = ctypes.c_int
    L.EZmockB200_real_size.argtypes = []
    L.EZmockB200_launch_count.restype = ctypes.c_longlong
    L.EZmockB200_launch_count.argtypes = []
    L.EZmockB200_select_path.restype = ctypes.c_int
    L.EZmockB200_select_path.argtypes = [ctypes.c_void_p]
    L.EZmockB200_mark.restype = ctypes.c_int
    L.EZmockB200_mark.argtypes = [_vp, ctypes.c_int]
    L.EZmockB200_elapsed.restype = ctypes.c_int
    L.EZmockB200_elapsed.argtypes = [_vp, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]
    L._rt = rt
    _cache[prec] = L
    return L


def header_symbols():
    """Function names declared in include/*.h."""
    import re
    names = []
    for fn in sorted(os.listdir(INCLUDE)):
        if fn.endswith(".h"):
            src = open(os.path.join(INCLUDE, fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(EZmock\w*)\s*\(", src)
    return sorted(set(names))
