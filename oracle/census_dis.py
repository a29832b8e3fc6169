"""Operation census of the nested DIS qqbar-g integrands -- test and measurement infrastructure.

The roofline of the nested I2/I3 kernels needs the work one outer sample costs, counted on
the algorithm, not on a build's instructions.  This module runs the DIS oracle's FP64 numpy
restatement of the nested terms (``oracle.dis.qg_integrand`` with 'I2n' / 'I3n': the 48-node
inner rule of custom_kernels/dis/i2_i3/extension.py:21-35 with dis/observables.py:253-331 and
the G functions of dis/transverse.py and dis/longitudinal.py) on arrays that count the
element-wise operations applied to them:

* arithmetic = add, subtract, multiply, divide, reciprocal, square, negative is not counted;
* special = exp, log, log1p, expm1, sqrt, power, trigonometric functions and the special
  functions the oracle calls from scipy (the Bessel functions K0/K1, the dilogarithm), one
  each;
* selects, comparisons, absolute values, min/max and array bookkeeping are not counted, and
  neither is arithmetic on constants only (it is hoisted out of the sample loop).

Counts are per outer sample, for one kinematic point of the DIS workload (light quark
m = 0.14 GeV) with the GBW dipole (the BK table's lookups are a few arithmetic operations per
amplitude and are not part of the inner loop).  ``tests/test_census.py`` checks that
``bench.py``'s DIS census constants are what ``workload_census()`` returns.

    python -m oracle.census_dis
"""

from __future__ import annotations

import numpy as np

ARITHMETIC = {"add", "subtract", "multiply", "true_divide", "divide", "reciprocal", "square"}
NOT_COUNTED = {"negative", "positive", "absolute", "fabs", "maximum", "minimum", "fmax", "fmin", "greater",
               "greater_equal", "less", "less_equal", "equal", "not_equal", "logical_and", "logical_or",
               "logical_not", "isfinite", "isnan", "isinf", "sign", "floor", "ceil", "rint", "trunc", "copysign",
               "bitwise_and", "bitwise_or"}


class Tally:
    arithmetic = 0
    special = 0
    names: dict = {}

    @classmethod
    def reset(cls) -> None:
        cls.arithmetic = 0
        cls.special = 0
        cls.names = {}


def _unwrap(value):
    if isinstance(value, Counted):
        return value.view(np.ndarray)
    if isinstance(value, (list, tuple)):
        return type(value)(_unwrap(v) for v in value)
    if isinstance(value, dict):
        return {k: _unwrap(v) for k, v in value.items()}
    return value


def _wrap(value):
    if isinstance(value, np.ndarray) and not isinstance(value, Counted):
        return value.view(Counted)
    if isinstance(value, tuple):
        return tuple(_wrap(v) for v in value)
    if isinstance(value, list):
        return [_wrap(v) for v in value]
    return value


class Counted(np.ndarray):
    """An array that adds the element-wise operations applied to it to ``Tally``."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        result = getattr(ufunc, method)(*_unwrap(inputs), **_unwrap(kwargs))
        if method == "__call__":
            name = ufunc.__name__
            size = int(np.size(result[0] if isinstance(result, tuple) else result))
            if name in ARITHMETIC:
                Tally.arithmetic += size
            elif name not in NOT_COUNTED:
                Tally.special += size
                Tally.names[name] = Tally.names.get(name, 0) + size
        return _wrap(result)

    def __array_function__(self, func, types, args, kwargs):
        return _wrap(func(*_unwrap(args), **_unwrap(kwargs)))


def census(contribution: str, transverse: bool, samples: int = 64, Q2: float = 10.0, xbj: float = 1e-3) -> dict:
    """Mean arithmetic and special operations per outer sample of a nested term."""
    from oracle import dis as odis

    kin = odis.Kinematics(Q2=Q2, xbj=xbj, mf=0.14, transverse=transverse, active_flavors=3)
    dipole = odis.GBWDipole(qs0sqr=0.25, lam=0.29)
    x = np.random.default_rng(7).uniform(0.02, 0.98, (samples, 5))
    Tally.reset()
    odis.qg_integrand(x.view(Counted), kin, contribution, dipole)
    return {"arithmetic": Tally.arithmetic / samples, "special": Tally.special / samples,
            "special_by_name": {k: v / samples for k, v in sorted(Tally.names.items())}}


def workload_census() -> dict:
    """Whole operations per outer sample of nested I2 and I3, averaged over the two
    polarisations (the DIS workload integrates both)."""
    out = {}
    for term in ("I2n", "I3n"):
        c = [census(term, t) for t in (True, False)]
        out[term] = {"arithmetic": int(round(sum(v["arithmetic"] for v in c) / 2)),
                     "special": int(round(sum(v["special"] for v in c) / 2))}
    return out


if __name__ == "__main__":
    import json

    print(json.dumps(workload_census()))
    print(json.dumps(census("I3n", True)["special_by_name"]))
