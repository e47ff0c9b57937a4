"""DavidLongRangeClassYk in the oracle against a numpy restatement
(PIMC++/src/Actions/DavidLongRangeClassYk.cc:38-389): the uk / duk / Vlong_k
construction of both branches (RPA with tan and tanh, and the
multiple-species form), the k-vector matching, and the slice ranges of
SingleAction (interior of a window, or [0, M - skip] for the whole path) and
of d_dBeta / V (every slice, 1/2 at the ends).  No GPU.
"""
import numpy as np

import oracle as O

N, M, BOX, TAU, LAM = 16, 8, 10.0, 0.1, 0.5


def _system(seed=3):
    rng = np.random.default_rng(seed)
    o = O.System(N, M + 1, [BOX] * 3, TAU, LAM, 0)
    base = rng.uniform(0, BOX, (N, 3))
    path = base[None] + rng.normal(0, 0.3, (M + 1, N, 3))
    o.set_path(path, 0)
    new = path.copy()
    new[1:-1, 5] += rng.normal(0, 0.4, (M - 1, 3))
    o.set_path(new, 1)
    o.setup_kvecs(2.0)
    kv, _ = o.kvecs()
    return o, path, new, kv


def _table(kv):
    kmag = np.sqrt((kv ** 2).sum(1))
    kvals = np.unique(np.round(kmag, 12))
    kvals = np.array([kmag[np.argmin(np.abs(kmag - k))] for k in kvals])  # exact |k| values
    uk_long = np.where(kvals < 1.2, 40.0 / kvals ** 2, -60.0 * kvals ** 2)  # tanh and tan branches
    return np.concatenate([[0.0], kvals]), np.concatenate([[1.0], uk_long]), kmag


def _numpy_tables(kvals, uk_long, kmag, rpa):
    vol = BOX ** 3
    u, du, v = np.empty(len(kmag)), np.empty(len(kmag)), np.empty(len(kmag))
    for j, k in enumerate(kmag):
        i = int(np.argmin(np.abs(kvals - k)))
        ul = uk_long[i]
        v[j] = ul / vol
        if not rpa:
            u[j], du[j] = v[j] * TAU, v[j]
            continue
        arg = 1.0 + N * 2.0 * ul / (LAM * k * k * vol)
        theta = 0.5 * k * k * LAM * TAU
        if arg < 0:
            q = np.sqrt(-arg)
            t = np.tan(q * theta)
            s = q * (1 - q * t) / (q + t)
        else:
            q = np.sqrt(arg)
            t = np.tanh(theta * q)
            s = q * (1 + q * t) / (q + t)
        u[j] = (s - 1.0) / N
        du[j] = ul / vol - LAM * k * k * u[j] * (1.0 + 0.5 * N * u[j])
    return u, du, v


def _rhok(pos, kv):
    return np.exp(1j * pos @ kv.T).sum(0)


def test_yk_tables_both_branches():
    o, _, _, kv = _system()
    kvals, uk_long, kmag = _table(kv)
    for rpa in (True, False):
        assert o.set_yk(kvals, uk_long, rpa)
        got = o.yk_tables()
        ref = _numpy_tables(kvals, uk_long, kmag, rpa)
        for g, r in zip(got, ref):
            np.testing.assert_allclose(g, r, rtol=1e-13, atol=0)
    # both RPA branches occur in this table
    arg = 1.0 + N * 2.0 * uk_long[1:] / (LAM * kvals[1:] ** 2 * BOX ** 3)
    assert (arg < 0).any() and (arg > 0).any()


def test_yk_unmatched_kvector_is_an_error():
    o, _, _, kv = _system()
    kvals, uk_long, _ = _table(kv)
    assert not o.set_yk(kvals[:-1], uk_long[:-1], True)


def test_yk_single_action_slice_ranges():
    o, path, new, kv = _system()
    kvals, uk_long, kmag = _table(kv)
    assert o.set_yk(kvals, uk_long, True)
    u, du, v = _numpy_tables(kvals, uk_long, kmag, True)
    o.calc_rhok_all()
    for (s1, s2, level) in [(0, 4, 1), (2, 6, 0), (0, M, 0), (0, M, 1), (4, 8, 2)]:
        skip = 1 << level
        whole = s1 == 0 and s2 == M
        first = s1 if whole else s1 + skip
        for copy, p in ((0, path), (1, new)):
            ref = sum((np.abs(_rhok(p[s], kv)) ** 2 * u).sum() for s in range(first, s2 - skip + 1, skip))
            got = o.yk_single(s1, s2, [5], level, copy=copy)
            assert abs(got - ref) <= 1e-11 * max(1.0, abs(ref)), (s1, s2, level, copy, got, ref)
        assert o.yk_single(s1, s2, [], level, copy=0) == 0.0
    for w, fn in ((du, o.yk_dbeta), (v, o.yk_v)):
        ref = sum((0.5 if s in (1, 7) else 1.0) * (np.abs(_rhok(path[s], kv)) ** 2 * w).sum() for s in range(1, 8))
        got = fn(1, 7)
        assert abs(got - ref) <= 1e-11 * max(1.0, abs(ref))
