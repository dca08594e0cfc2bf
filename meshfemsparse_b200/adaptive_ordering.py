"""Adaptive choice between two orderings from the factorization history.

Restates the reference's heuristic (Solvers/AdaptiveOrderingSelection.hh:34-250, with the
choices of Solvers/CatamariFactorizer.hh:156-167): start with the costly, high-quality
primary ordering (nested dissection); when the pattern changes so often that symbolic
analyses dominate, switch to the cheap alternate (minimum degree) for the next analysis,
and back when the balance turns again. Per method it keeps exponential moving averages
(weight 0.2) of the symbolic, numeric and solve times; over a window of the last five
symbolic analyses it estimates what each method would have cost for the analyses,
factorizations and solves done in that window (a method without data borrows the active
one's averages times an optimistic multiplier) and switches at the next analysis when the
active method's estimate exceeds the other's by 5 %. It asks for an early analysis
(`should_trigger_recompute`) only when the other method is known to factor faster, the
estimates differ by 10 % and the current analysis has served more than 25 factorizations.
The first two analyses always use the primary method; a factor that shrinks by 15 % since
the last switch discards the inactive method's history.
"""
from __future__ import annotations

from collections import deque
from dataclasses import dataclass, field


@dataclass
class _Average:
    """Exponential moving average (weight `alpha` on the newest sample) and a count."""
    alpha: float = 0.2
    value: float = 0.0
    count: int = 0

    def add(self, t: float) -> None:
        self.value = t if self.count == 0 else (1.0 - self.alpha) * self.value + self.alpha * t
        self.count += 1

    def known(self) -> bool:
        return self.count > 0

    def average(self, default: float = 0.0) -> float:
        return self.value if self.count else default


@dataclass
class _MethodTimes:
    symbolic: _Average = field(default_factory=_Average)
    numeric: _Average = field(default_factory=_Average)
    solve: _Average = field(default_factory=_Average)


class AdaptiveOrderingSelection:
    def __init__(self, primary, alternate, num_multipliers=(0.5, 1.35), sym_multipliers=(5.0, 0.10)):
        self.methods = (primary, alternate)
        # optimistic estimates of a method's time relative to the active one's, used until
        # the method has data of its own (index 0: primary, 1: alternate)
        self.num_multipliers = tuple(num_multipliers)
        self.sym_multipliers = tuple(sym_multipliers)
        self.window_size = 5
        self.warmup_sym_count = 2
        self.switch_threshold_soft = 1.05
        self.switch_threshold_hard = 1.10
        self.factorizations_before_hard_switch = 25
        self.nnz_reduction_for_reset = 0.15
        self.current = 0
        self.times = [_MethodTimes(), _MethodTimes()]
        self.nnz_at_last_switch = 0
        self.numeric_per_symbolic: deque[int] = deque()
        self.solves_per_symbolic: deque[int] = deque()

    # ----------------------------------------------------------------- state
    def current_method(self):
        return self.methods[self.current]

    def total_symbolic(self) -> int:
        return self.times[0].symbolic.count + self.times[1].symbolic.count

    def numeric_in_window(self) -> int:
        return sum(self.numeric_per_symbolic)

    def solves_in_window(self) -> int:
        return sum(self.solves_per_symbolic)

    # ------------------------------------------------------------- recording
    def record_symbolic(self, seconds: float, factor_nnz: int = 0) -> None:
        self.times[self.current].symbolic.add(seconds)
        for window in (self.numeric_per_symbolic, self.solves_per_symbolic):
            window.append(0)
            if len(window) > self.window_size:
                window.popleft()
        if self.nnz_at_last_switch == 0:
            self.nnz_at_last_switch = factor_nnz
        if factor_nnz < self.nnz_at_last_switch * (1.0 - self.nnz_reduction_for_reset):
            # the problem changed: the inactive method's timings no longer describe it
            self.times[1 - self.current] = _MethodTimes()

    def record_numeric(self, seconds: float) -> None:
        if self.times[self.current].symbolic.count == 0 or not self.numeric_per_symbolic:
            raise RuntimeError("adaptive ordering: a numeric factorization before any symbolic analysis")
        self.times[self.current].numeric.add(seconds)
        self.numeric_per_symbolic[-1] += 1

    def record_solve(self, seconds: float) -> None:
        if self.times[self.current].symbolic.count == 0 or not self.solves_per_symbolic:
            raise RuntimeError("adaptive ordering: a solve before any symbolic analysis")
        self.times[self.current].solve.add(seconds)
        self.solves_per_symbolic[-1] += 1

    # -------------------------------------------------------------- decisions
    def time_estimate(self, method: int) -> float:
        """What `method` would have cost for the window's analyses, factorizations and solves."""
        if self.numeric_in_window() == 0:
            raise RuntimeError("no numeric factorizations yet")
        cur = self.times[self.current]
        if not (cur.symbolic.known() and cur.numeric.known() and cur.solve.known()):
            raise RuntimeError("no times recorded for the current method")
        t = self.times[method]
        sym = t.symbolic.average(self.sym_multipliers[method] * cur.symbolic.average())
        num = t.numeric.average(self.num_multipliers[method] * cur.numeric.average())
        sol = t.solve.average(self.num_multipliers[method] * cur.solve.average())
        return (sym * len(self.numeric_per_symbolic) + num * self.numeric_in_window()
                + sol * self.solves_in_window())

    def _should_switch(self, threshold: float) -> bool:
        if self.total_symbolic() < self.warmup_sym_count:
            return False
        return self.time_estimate(self.current) / self.time_estimate(1 - self.current) > threshold

    def _switch_pays(self, threshold: float) -> bool:
        # without a factorization and a solve in the window there is nothing to compare
        # (the reference raises there); keep the active method
        try:
            return self._should_switch(threshold)
        except RuntimeError:
            return False

    def update_selection(self):
        """The method the next symbolic analysis uses (switching when it pays off)."""
        if self._switch_pays(self.switch_threshold_soft):
            self.current = 1 - self.current
            self.nnz_at_last_switch = 0
        return self.current_method()

    def should_trigger_recompute(self) -> bool:
        """Whether to redo the symbolic analysis now, with the other method."""
        cur, other = self.times[self.current].numeric, self.times[1 - self.current].numeric
        if not other.known() or other.average() > cur.average():
            return False
        return (self._switch_pays(self.switch_threshold_hard)
                and self.numeric_per_symbolic[-1] > self.factorizations_before_hard_switch)
