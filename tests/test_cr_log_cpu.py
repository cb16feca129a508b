"""The distance epilogue's logarithm (csharp_b200/csrc/swg_log.cuh) on the CPU: the same source the
Kimura2 / JukesCantor epilogues run on the device, compiled for the host.

Tolerance: exact.  Every result must equal the correctly rounded natural logarithm, taken from
Python's decimal module at 50 significant digits (its ln is correctly rounded at that precision),
on the arguments the distances produce -- JukesCantor's 1 - (4/3)(diff / columns) and Kimura2's
1 - 2P - Q and 1 - 2Q for small column counts, in the reference's binary64 operation order
(Alignment.cs:254-348) -- and on random arguments over the whole exponent range and near 1.  The
C library's log (what the oracle uses) is off by one unit in the last place on a fraction of these
arguments; none of those changes an Int16 distance here.
"""
import ctypes as C
import shutil
import subprocess
from decimal import Decimal, getcontext
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def crlog(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ is missing")
    so = tmp_path_factory.mktemp("crlog") / "libcrlog.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so),
                    str(HERE / "cr_log_host.cpp")], check=True)
    lib = C.CDLL(str(so))

    def run(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        lib.cr_log_many(C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), C.c_long(len(x)))
        return y
    return run


def _jc_args(max_cols):
    xs = set()
    for ng in range(1, max_cols + 1):
        for diff in range(ng + 1):
            d = 1.0 - (4.0 / 3.0) * (diff / ng)
            if d > 5e-324:
                xs.add(d)
    return np.array(sorted(xs))


def _kimura_args(max_cols):
    a_l, b_l = [], []
    for ng in range(1, max_cols + 1):
        for ts in range(ng + 1):
            tv = np.arange(ng + 1 - ts)
            P, Q = ts / ng, tv / ng
            a, b = 1.0 - 2.0 * P - Q, 1.0 - 2.0 * Q
            ok = (a > 5e-324) & (b > 5e-324)
            a_l.append(a[ok])
            b_l.append(b[ok])
    return np.concatenate(a_l), np.concatenate(b_l)


def _correct(xs):
    getcontext().prec = 50
    return np.array([float(Decimal(float(v)).ln()) for v in xs])


def test_correctly_rounded_on_distance_arguments_and_random_inputs(crlog):
    rng = np.random.default_rng(1)
    a, b = _kimura_args(60)
    xs = np.unique(np.concatenate([_jc_args(250), a, b, np.exp(rng.uniform(-700, 700, 5000)),
                                   1.0 + rng.uniform(-1e-6, 1e-6, 2000), [1.0, 0.5, 2.0, 5e-324, 1.7e308]]))
    got = crlog(xs)
    want = _correct(xs)
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, (xs[bad][:5], got[bad][:5], want[bad][:5])


def test_special_values(crlog):
    y = crlog(np.array([0.0, -1.0, np.inf, np.nan]))
    assert y[0] == -np.inf and np.isnan(y[1]) and y[2] == np.inf and np.isnan(y[3])


def test_int16_distances_equal_the_c_library_logs(crlog):
    """Over every JukesCantor argument with up to 600 non-gap columns and every Kimura2 pair with
    up to 120, the Int16 distance is the same with either logarithm."""
    i16 = lambda v: np.trunc(v * 32767.0)
    d = _jc_args(600)
    assert np.array_equal(i16(-0.75 * crlog(d)), i16(-0.75 * np.log(d)))
    a, b = _kimura_args(120)
    assert np.array_equal(i16(-0.5 * crlog(a) - 0.25 * crlog(b)), i16(-0.5 * np.log(a) - 0.25 * np.log(b)))
