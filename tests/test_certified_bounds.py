"""The bound behind the level kernel's certified control steps, checked in
double arithmetic on the host: the sequential sum Q of N terms (the
reference's order) and any other order's sum P of the same terms differ by
at most 2 gamma_{N-1} sum|t| (recursive summation bound); the kernel widens
P by B = 3 N u A + 2^-50 |P| (A the computed sum of magnitudes, u = 2^-53),
which also covers the rounding of A and of the bounds.  Here Q comes from a
sequential cumulative sum, P from pairwise and blocked orders, on terms
chosen to make the orders disagree (cancellation, wide exponent ranges,
sums that cross zero)."""
import numpy as np
import pytest

U = 2.0 ** -53


def bounds(P, A, N):
    B = A * (3.0 * N * U) + abs(P) * 2.0 ** -50
    return P - B, P + B


def orders(t):
    """Sums of t in three parallel-style orders: pairwise, 64-term blocks
    added in order, and 512-term blocks added pairwise."""
    yield float(np.sum(t))   # numpy: pairwise
    blocks = np.add.reduceat(t, np.arange(0, t.size, 64))
    acc = 0.0
    for b in blocks:
        acc += b
    yield acc
    yield float(np.sum(np.add.reduceat(t, np.arange(0, t.size, 512))))


def cases(rng):
    n = 20000
    yield rng.normal(size=n)                                   # crosses zero repeatedly
    yield rng.normal(size=n) * 10.0 ** rng.integers(-12, 12, n)  # wide exponents
    x = rng.normal(size=n // 2)
    yield np.concatenate([x, -x[::-1]]) + rng.normal(size=n) * 1e-12   # near-total cancellation
    yield np.abs(rng.normal(size=n)) ** 2                       # positive (E_data-like)
    yield (rng.random(n) - 0.5) * 2.0 ** 40 + rng.random(n)     # large terms, small signal


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_ordered_sum_lies_in_the_certified_interval(seed):
    rng = np.random.default_rng(seed)
    for t in cases(rng):
        t = np.ascontiguousarray(t, dtype=np.float64)
        Q = float(np.cumsum(t)[-1])         # 0 + t0 + t1 + ... in order
        A = float(np.sum(np.abs(t)))
        for P in orders(t):
            lo, hi = bounds(P, A, t.size)
            assert lo <= Q <= hi, (P, Q, lo, hi)


def test_the_interval_is_tight_enough_to_decide_armijo_tests():
    """On a sum the size of a 513^2 energy pass the interval is ~1e-10 of the
    magnitude sum: far below the energy differences the Armijo tests compare
    except near convergence."""
    rng = np.random.default_rng(7)
    t = np.abs(rng.normal(size=513 * 513)) * 1e-6
    P, A = float(np.sum(t)), float(np.sum(np.abs(t)))
    lo, hi = bounds(P, A, t.size)
    assert (hi - lo) / A < 2e-10
