"""ctypes binding of libjk.so, the J/K engine's C-ABI (include/byteqc_jk.h).

Mirrors the reference's ``byteqc.cuobc.lib.load_library``
(``cuobc/lib/__init__.py:39-42``).  There is no fallback: if the library was
not built, or no CUDA device is present, the J/K path raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.normpath(os.path.join(_HERE, '..', '..', 'csrc'))
LIBJK_PATH = os.path.join(CSRC, 'libjk.so')

JK_OK = 0


class JKOpts(ctypes.Structure):
    _fields_ = [('direct_scf_tol', ctypes.c_double),
                ('nbins', ctypes.c_int),
                ('prescreen', ctypes.c_int),
                ('fp32_cutoff', ctypes.c_double),
                ('shard', ctypes.c_int),
                ('nshards', ctypes.c_int),
                ('reserved', ctypes.c_int * 6)]


_LIB = None

_SIGNATURES = {
    'jk_basis_create': [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                        ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                        ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                        ctypes.c_int, ctypes.c_void_p],
    'jk_basis_destroy': [ctypes.c_void_p],
    'jk_basis_info': [ctypes.c_void_p, ctypes.c_void_p],
    'jk_basis_pairs': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_void_p],
    'jk_build_class_pair': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    'jk_fill_int2e': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                      ctypes.c_int, ctypes.c_void_p],
    'jk_build_class_pair_noalloc': [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p],
    'jk_build': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                 ctypes.c_void_p],
    'jk_get_jk': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    'jk_rys_roots_host': [ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                          ctypes.c_void_p],
    'jk_rys_roots_device': [ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_void_p],
    'jk_basis_cq_info': [ctypes.c_void_p, ctypes.c_void_p],
    'jk_last_counts': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    'jk_fma_peak': [ctypes.c_int, ctypes.c_void_p],
    'jk_int1e_cart': [ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                      ctypes.c_void_p],
    'jk_batch_create': [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    'jk_batch_create_ex': [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong,
                           ctypes.c_void_p],
    'jk_batch_nsolo': [ctypes.c_void_p, ctypes.c_void_p],
    'jk_class_pair_tasks': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                            ctypes.c_void_p],
    'jk_batch_destroy': [ctypes.c_void_p],
    'jk_batch_build': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                       ctypes.c_void_p],
    'jk_batch_get_jk': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p],
    'jk_batch_tune': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                      ctypes.c_char_p, ctypes.c_void_p],
    'jk_batch_info': [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    'jk_shard_plan': [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                      ctypes.c_void_p],
    'jk_last_error': [],
}


def load_library(path=LIBJK_PATH):
    """Load libjk.so (built in-tree by ``__graft_entry__.build()``)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError('libjk.so not built at %s: run '
                          '`python -c "import __graft_entry__ as g; g.build()"`'
                          % path)
    lib = ctypes.CDLL(path)
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    lib.jk_last_error.restype = ctypes.c_char_p
    _LIB = lib
    return lib


def check(rc, what):
    if rc != JK_OK:
        msg = load_library().jk_last_error().decode()
        raise RuntimeError('%s failed (status %d): %s' % (what, rc, msg))
