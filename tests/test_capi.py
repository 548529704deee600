"""The C-ABI library loads without a GPU, exports every symbol the header
declares, and rejects invalid arguments with a status (no process exit)."""
import ctypes
import os
import re

import numpy as np

from byteqc_b200.cuobc import lib as jklib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, 'include', 'byteqc_jk.h')).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(jk_[a-z0-9_]+)\s*\(', src)))


def test_exports_every_declared_symbol():
    lib = jklib.load_library()
    names = _declared()
    assert 'jk_build' in names and 'jk_get_jk' in names
    for n in names:
        assert hasattr(lib, n), n


def test_invalid_arguments_return_status():
    lib = jklib.load_library()
    out = ctypes.c_void_p()
    rc = lib.jk_basis_create(None, 0, None, 0, None, 0, None, 0, 1e-13, 0,
                             ctypes.byref(out))
    assert rc == 3
    assert b'invalid' in lib.jk_last_error()
    s = np.zeros(2)
    assert lib.jk_rys_roots_host(0, 1.0, s.ctypes.data, s.ctypes.data) == 3
    # the per-class-pair entries check their arguments before any CUDA call
    bins = np.zeros(2, dtype=np.int32)
    st = np.ones(4, dtype=np.int32)
    assert lib.jk_fill_int2e(None, None, 0, st.ctypes.data, st.ctypes.data,
                             bins.ctypes.data, bins.ctypes.data, 1, 0, 0,
                             None) == 3
    assert b'invalid' in lib.jk_last_error()
    assert lib.jk_build_class_pair(None, None, None, None, 0, 1,
                                   bins.ctypes.data, bins.ctypes.data, 1, 0,
                                   0, None) == 3


def test_product_tables_match_oracle_tables():
    import oracle
    lib = jklib.load_library()
    rng = np.random.default_rng(0)
    for n in range(1, 14):
        for x in np.concatenate([[0., 1e-12, 2., 39.999, 98.0, 150.],
                                 rng.uniform(0, 110, 40)]):
            s = np.zeros(n)
            w = np.zeros(n)
            assert lib.jk_rys_roots_host(n, x, s.ctypes.data,
                                         w.ctypes.data) == 0
            so, wo = oracle.rys_roots(n, x)
            np.testing.assert_allclose(s, so, rtol=5e-14, atol=0)
            np.testing.assert_allclose(w, wo, rtol=0, atol=5e-15 * w.sum())


def test_shard_plan_balances_and_is_deterministic():
    """jk_shard_plan (host code): every task gets one owner in range, the
    plan is the longest-processing-time rule (restated here), identical on
    repeated calls, and no owner exceeds the mean load by more than the
    largest task."""
    lib = jklib.load_library()
    rng = np.random.default_rng(3)
    for n, k in ((1, 1), (5, 8), (300, 2), (666, 4), (1000, 8)):
        cost = np.ascontiguousarray(rng.lognormal(0., 2., n))
        own = np.zeros(n, dtype=np.int32)
        assert lib.jk_shard_plan(cost.ctypes.data, n, k, own.ctypes.data) == 0
        own2 = np.zeros(n, dtype=np.int32)
        assert lib.jk_shard_plan(cost.ctypes.data, n, k, own2.ctypes.data) == 0
        np.testing.assert_array_equal(own, own2)
        assert own.min() >= 0 and own.max() < k
        ref = np.zeros(n, dtype=np.int32)
        load = np.zeros(k)
        for i in sorted(range(n), key=lambda i: (-cost[i], i)):
            r = int(np.argmin(load))
            ref[i] = r
            load[r] += cost[i]
        np.testing.assert_array_equal(own, ref)
        loads = np.bincount(own, weights=cost, minlength=k)
        assert loads.max() <= cost.sum() / k + cost.max() + 1e-9
    bad = np.zeros(1, dtype=np.int32)
    assert lib.jk_shard_plan(None, 1, 2, bad.ctypes.data) == 3
    assert lib.jk_shard_plan(np.ones(1).ctypes.data, 1, 0, bad.ctypes.data) == 3
