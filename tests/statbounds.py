"""Bounds for the statistical image tests.

A pixel channel whose two estimates agree in distribution lands beyond 3 combined
standard errors with probability p (0.0027 for normal means; more for standard errors
estimated from few samples: the t distribution's tail). Over n channels the count of such
channels is binomial(n, p); the tests allow its mean plus 4 standard deviations, so a
correct renderer fails about once in 30,000 runs, while a bias confined to a fraction of
the pixels well above p is caught."""
import math

from scipy import stats

P_NORMAL_3SIGMA = math.erfc(3.0 / math.sqrt(2.0))   # 0.0026998


def binomial_bound(n, p, k=4.0):
    """Largest count allowed: n p + k sqrt(n p (1 - p)), rounded up."""
    return int(math.ceil(n * p + k * math.sqrt(n * p * (1.0 - p))))


def t_tail(x, nu):
    """P(|T| > x) for Student's t with nu degrees of freedom."""
    return float(2.0 * stats.t.sf(x, nu))
