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


def _ref_bin_loop_count(bins_ij, bins_kl, nbins, diag):
    """The reference's bin loop (gvhf/nr_jk_driver.cu:252-280): kl bin b
    pairs with the ij rows [bins_ij[0], bins_ij[nbins - b]); a diagonal
    class pair keeps kl <= ij.  Returns the quartet count and the per-row
    counts."""
    rows = {}
    n = 0
    for b in range(nbins):
        kl0, kl1 = bins_kl[b], bins_kl[b + 1]
        for ij in range(bins_ij[0], bins_ij[nbins - b]):
            c = sum(1 for kl in range(kl0, kl1) if not (diag and kl > ij))
            rows[ij] = rows.get(ij, 0) + c
            n += c
    return n, rows


def test_class_pair_tasks_follow_the_reference_bin_loop():
    """The row prefix the per-class-pair entries build on the device (the
    same code, run here on the host) counts exactly the quartets of the
    reference's bin loop, on bins of seeded log-Schwarz values."""
    from oracle import hf_oracle
    lib = jklib.load_library()
    rng = np.random.default_rng(3)
    for it in range(60):
        n_ij = int(rng.integers(1, 120))
        diag = bool(it % 2)
        n_kl = n_ij if diag else int(rng.integers(1, 120))
        nbins = int(rng.integers(1, 16))
        cutoff = 10.0 ** -rng.uniform(6, 14)
        lq_ij = np.sort(rng.uniform(-30, 0, n_ij))[::-1]
        lq_kl = np.sort(rng.uniform(-30, 0, n_kl))[::-1]
        bij = hf_oracle.make_s_index_offsets(lq_ij, nbins, cutoff)
        bkl = bij if diag else hf_oracle.make_s_index_offsets(lq_kl, nbins, cutoff)
        qoff = np.zeros(n_ij + 1, dtype=np.int64)
        tot = ctypes.c_longlong()
        assert lib.jk_class_pair_tasks(bij.ctypes.data, bkl.ctypes.data, nbins, n_ij,
                                       int(diag), qoff.ctypes.data, ctypes.byref(tot)) == 0
        n, rows = _ref_bin_loop_count(bij, bkl, nbins, diag)
        assert tot.value == n
        per_row = np.diff(qoff)
        for ij in range(n_ij):
            assert per_row[ij] == rows.get(ij, 0), (it, ij)
    # decreasing bins are refused
    bad = np.array([0, 5, 3], dtype=np.int32)
    tot = ctypes.c_longlong()
    assert lib.jk_class_pair_tasks(bad.ctypes.data, bad.ctypes.data, 2, 5, 0, None,
                                   ctypes.byref(tot)) == 3
