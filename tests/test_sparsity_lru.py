"""Sparsity cache for changing (contact) patterns: reuse, insertion, aging,
budget eviction and hard expiration."""
import numpy as np
import pytest

from meshfemsparse_b200.sparsity_lru import EXPIRED, STATIC_ENTRY_AGE, SparsityLRU


def csc(n, entries):
    """Upper CSC from (row, col) pairs."""
    cols = [[] for _ in range(n)]
    for i, j in entries:
        cols[j].append(i)
    Ap, Ai = [0], []
    for j in range(n):
        Ai.extend(sorted(set(cols[j])))
        Ap.append(len(Ai))
    return np.array(Ap), np.array(Ai)


N = 6
STATIC = [(j, j) for j in range(N)] + [(j, j + 1) for j in range(N - 1)]


def entries(lru):
    cols = np.repeat(np.arange(lru.n), np.diff(lru.Ap))
    return set(zip(lru.Ai.tolist(), cols.tolist()))


def test_reuse_insert_and_ages():
    lru = SparsityLRU(N, *csc(N, STATIC), budget_ratio=1.0)
    assert lru.update(N, *csc(N, [])) == 0
    assert lru.update(N, *csc(N, [(0, 3), (1, 5)])) == 2
    assert {(0, 3), (1, 5)} <= entries(lru)
    assert (lru.entryAges() == STATIC_ENTRY_AGE).sum() == len(STATIC)
    assert lru.update(N, *csc(N, [(0, 3), (1, 5)])) == 0
    assert lru.update(N, *csc(N, [(0, 3)])) == 0          # (1, 5) lingers within the budget
    ages = dict(zip(zip(lru.Ai.tolist(), np.repeat(np.arange(N), np.diff(lru.Ap)).tolist()), lru.entryAges()))
    assert ages[(1, 5)] == 1 and ages[(0, 3)] == 0


def test_expired_entries_leave_at_the_next_rebuild():
    lru = SparsityLRU(N, *csc(N, STATIC), budget_ratio=1.0, expiration_age=3, hard_expiration_age=100)
    lru.update(N, *csc(N, [(1, 5)]))
    assert lru.update(N, *csc(N, [(0, 2)])) == 1          # (0, 2) new; (1, 5) absent, age 1
    assert [lru.update(N, *csc(N, [(0, 2)])) for _ in range(3)] == [0, 0, 0]
    assert (1, 5) in entries(lru)                         # aged 4 (>= 3) but no rebuild yet
    assert lru.update(N, *csc(N, [(0, 2), (2, 4)])) == 1  # a new entry forces a rebuild
    assert (1, 5) not in entries(lru) and {(0, 2), (2, 4)} <= entries(lru)


def test_budget_eviction_returns_expired():
    lru = SparsityLRU(N, *csc(N, STATIC), budget_ratio=0.0)
    assert lru.update(N, *csc(N, [(0, 4)])) == 1
    assert lru.update(N, *csc(N, [(1, 3)])) == EXPIRED     # (0, 4) is old and the budget is 0
    assert (0, 4) not in entries(lru) and (1, 3) in entries(lru)
    assert set(STATIC) <= entries(lru)


def test_hard_expiration_and_static_entries_survive():
    lru = SparsityLRU(N, *csc(N, STATIC), budget_ratio=1.0, expiration_age=2, hard_expiration_age=4)
    lru.update(N, *csc(N, [(2, 5), (0, 1)]))               # (0, 1) is static
    results = [lru.update(N, *csc(N, [(0, 1)])) for _ in range(4)]
    assert results[:3] == [0, 0, 0] and results[3] == EXPIRED
    assert (2, 5) not in entries(lru) and set(STATIC) <= entries(lru)


def test_missing_diagonal_is_rejected():
    Ap, Ai = csc(N, [(j, j + 1) for j in range(N - 1)] + [(0, 0)])
    lru = SparsityLRU(N, Ap, Ai)
    with pytest.raises(RuntimeError):
        lru.update(N, *csc(N, [(0, 2)]))
