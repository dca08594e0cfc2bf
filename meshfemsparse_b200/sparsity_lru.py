"""Sparsity cache for patterns that change now and then (contact): keeps recently
seen dynamic entries so that a reappearing entry needs no new symbolic
factorization (the reference's SparsityLRU, SparsityLRU.hh:26-320).

The cached pattern is the static pattern plus dynamic entries. Static entries
have age -1 and never expire. A dynamic entry's age resets to 0 whenever it is
in the current dynamic pattern and grows by one at every update that lacks it.
`update(S_dynamic)` returns
  0        the cached pattern covers static + dynamic and can be reused as is
           (entries older than `expirationAge` may linger while the old entries
           fit the budget);
  k > 0    k entries were new: the cache was rebuilt (ages >= expirationAge and
           old entries beyond the budget dropped) and needs a symbolic factorization;
  EXPIRED  old entries were evicted (budget exceeded or an age reached
           `hardExpirationAge`): rebuilt, and a fresh ordering is advisable.
The budget is `entryCacheBudgetRatio` times the number of entries in the current
static + dynamic pattern; when it is exceeded, the oldest old entries go first.
Patterns are scalar or block upper-triangular CSC (n, Ap, Ai) with rows sorted
and the diagonal present in every column.
"""
from __future__ import annotations

import numpy as np

STATIC_ENTRY_AGE = -1
EXPIRED = np.iinfo(np.int64).max


class SparsityLRU:
    def __init__(self, n: int, Ap, Ai, budget_ratio: float = 0.01, expiration_age: int = 25,
                 hard_expiration_age: int = 250):
        self.n = int(n)
        self.Ap = np.asarray(Ap, dtype=np.int64).copy()
        self.Ai = np.asarray(Ai, dtype=np.int64).copy()
        self.age = np.full(self.Ai.size, STATIC_ENTRY_AGE, dtype=np.int64)
        self.num_static = int(self.Ai.size)
        self.entryCacheBudgetRatio = float(budget_ratio)
        self.expirationAge = int(expiration_age)
        self.hardExpirationAge = int(hard_expiration_age)

    # -- helpers
    def _rebuild(self, keep: np.ndarray, add_cols=None, add_rows=None) -> None:
        """Keep the flagged cache entries and insert new (row, col) entries with age 0."""
        cols = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(self.Ap))[keep]
        rows, ages = self.Ai[keep], self.age[keep]
        if add_cols is not None and add_cols.size:
            cols = np.concatenate([cols, add_cols])
            rows = np.concatenate([rows, add_rows])
            ages = np.concatenate([ages, np.zeros(add_cols.size, dtype=np.int64)])
        order = np.lexsort((rows, cols))
        cols, rows, ages = cols[order], rows[order], ages[order]
        self.Ap = np.zeros(self.n + 1, dtype=np.int64)
        np.add.at(self.Ap, cols + 1, 1)
        self.Ap = np.cumsum(self.Ap)
        self.Ai, self.age = rows, ages
        last = self.Ap[1:] - 1
        if self.n and (np.any(np.diff(self.Ap) <= 0) or np.any(self.Ai[last] != np.arange(self.n))):
            raise RuntimeError("SparsityLRU: missing diagonal entry in new sparsity pattern")

    def _match(self, Dp, Di):
        """For every cache entry: is it in D; for every D entry: is it in the cache."""
        ccols = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(self.Ap))
        dcols = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(Dp))
        ckey = ccols * (self.n + 1) + self.Ai
        dkey = dcols * (self.n + 1) + Di
        return np.isin(ckey, dkey), np.isin(dkey, ckey, invert=True), dcols

    def increaseAgeOfOldEntries(self, threshold: int = 0) -> bool:
        """Age the entries older than `threshold`; prune and return True on hard expiration."""
        old = self.age > threshold
        if not old.any():
            return False
        self.age[old] += 1
        if self.age.max() >= self.hardExpirationAge:
            self._rebuild(self.age < self.expirationAge)
            return True
        return False

    def update(self, n: int, Dp, Di) -> int:
        """Merge the current dynamic pattern (n, Dp, Di); see the module docstring."""
        if int(n) != self.n:
            raise RuntimeError("SparsityLRU: S_dynamic size mismatch")
        Dp = np.asarray(Dp, dtype=np.int64)
        Di = np.asarray(Di, dtype=np.int64)
        nonstatic = self.age != STATIC_ENTRY_AGE
        if Di.size == 0 and self.age.size <= self.entryCacheBudgetRatio * self.num_static:
            return EXPIRED if self.increaseAgeOfOldEntries(STATIC_ENTRY_AGE) else 0
        in_d, new_in_d, dcols = self._match(Dp, Di)
        # present dynamic entries get age 0, absent ones age by one
        self.age[nonstatic & in_d] = 0
        absent = nonstatic & ~in_d
        self.age[absent] += 1
        n_new = int(new_in_d.sum())
        n_current = int((~nonstatic).sum() + (nonstatic & in_d).sum()) + n_new
        n_old = int(absent.sum())
        budget = int(n_current * self.entryCacheBudgetRatio)
        if n_new == 0:
            if absent.any() and self.age[absent].max() >= self.hardExpirationAge:
                self._rebuild(self.age < self.expirationAge)
                return EXPIRED
            if n_old <= budget:
                return 0
        keep = self.age < self.expirationAge
        result = n_new
        if n_old > budget:
            # keep only the `budget` youngest old entries (stable: earlier entries first on ties)
            old_idx = np.nonzero(absent)[0]
            order = old_idx[np.argsort(self.age[old_idx], kind="stable")]
            keep[order[budget:]] = False
            result = EXPIRED
        self._rebuild(keep, dcols[new_in_d], Di[new_in_d])
        return result

    def entryAges(self) -> np.ndarray:
        return self.age
