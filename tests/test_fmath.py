"""The deterministic elementary functions (falcor_b200/csrc/fmath.h) that the
kernels and the CPU oracle share.

CPU: within 3 ulp of the correctly rounded value (numpy float64 rounded to
float32) over seeded sweeps of the ranges the path uses.  GPU: the device
evaluation is bit-identical to the host's, and within 8 ulp of CUDA's own
sinf/cosf/... (whose documented errors are up to 4 ulp).
"""
import numpy as np
import pytest

from oracle import ffi as O

RNG = np.random.default_rng(2024)
N = 400_000


def _cases():
    u = lambda lo, hi: RNG.uniform(lo, hi, N).astype(np.float32)  # noqa: E731
    return {
        "sin": (u(-7.0, 7.0), None, lambda x, y: np.sin(x)),
        "cos": (u(-7.0, 7.0), None, lambda x, y: np.cos(x)),
        "atan2": (u(-3.0, 3.0), u(-3.0, 3.0), lambda x, y: np.arctan2(x, y)),
        "acos": (u(-1.0, 1.0), None, lambda x, y: np.arccos(x)),
        "exp": (u(-100.0, 88.0), None, lambda x, y: np.exp(x)),
        "log": (np.exp2(u(-140.0, 127.0)).astype(np.float32), None, lambda x, y: np.log(x)),
        "log2": (np.exp2(u(-140.0, 127.0)).astype(np.float32), None, lambda x, y: np.log2(x)),
        "exp2": (u(-126.0, 127.0), None, lambda x, y: np.exp2(x)),
        "pow": (u(0.001, 100.0), u(-3.0, 3.0), lambda x, y: np.power(x, y)),
    }


CASES = _cases()


def _ulp_diff(a, b):
    """|a - b| in units in the last place of float32 (sign-magnitude order)."""
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-(2 ** 31)) - ia, ia)
    ib = np.where(ib < 0, np.int64(-(2 ** 31)) - ib, ib)
    return np.abs(ia - ib)


@pytest.mark.parametrize("fn", list(CASES))
def test_fmath_within_3_ulp_of_correctly_rounded(oracle, fn):
    x, y, ref = CASES[fn]
    got = O.fmath(fn, x, y)
    exact = ref(x.astype(np.float64), None if y is None else y.astype(np.float64)).astype(np.float32)
    d = _ulp_diff(got, exact)
    assert d.max() <= 3, f"{fn}: max {d.max()} ulp at x={x[d.argmax()]!r}"


def test_fmath_special_values(oracle):
    f = lambda fn, a, b=None: float(O.fmath(fn, np.array([a], np.float32), None if b is None else np.array([b], np.float32))[0])  # noqa: E731
    assert f("atan2", 0.0, -0.0) == pytest.approx(np.pi)
    assert f("atan2", -0.0, -1.0) == pytest.approx(-np.pi)
    assert f("atan2", 1.0, 0.0) == pytest.approx(np.pi / 2)
    assert f("acos", -1.0) == pytest.approx(np.pi)
    assert f("acos", 1.0) == 0.0
    assert np.isnan(f("acos", 1.5))
    assert f("log", 0.0) == -np.inf and np.isnan(f("log", -1.0))
    assert f("exp", -200.0) == 0.0 and f("exp", 100.0) == np.inf
    assert f("exp2", -149.0) == np.float32(2.0 ** -149)
    assert f("pow", 2.0, 0.0) == 1.0 and f("pow", 0.0, 2.5) == 0.0
    assert f("pow", 0.5, 5.0) == np.float32(0.5) ** 5
    assert f("pow", -2.0, 3.0) == -8.0


@pytest.mark.gpu
@pytest.mark.parametrize("fn", list(CASES))
def test_fmath_device_bit_identical_to_host(fpt, oracle, fn):
    import ctypes as C
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200 import _ffi
    x, y, ref = CASES[fn]
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda() if y is not None else None
    out = torch.empty_like(dx)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    k = O.FMATH[fn]
    _ffi.check(fpt.fpt_fmath_eval(k, 0, x.size, dx.data_ptr(), dy.data_ptr() if dy is not None else None, out.data_ptr(), stream))
    dev = out.cpu().numpy()
    host = O.fmath(fn, x, y)
    same = dev.view(np.uint32) == host.view(np.uint32)
    assert same.all(), f"{fn}: {(~same).sum()} of {x.size} differ, first x={x[~same][0]!r}"
    _ffi.check(fpt.fpt_fmath_eval(k, 1, x.size, dx.data_ptr(), dy.data_ptr() if dy is not None else None, out.data_ptr(), stream))
    cuda = out.cpu().numpy()
    d = _ulp_diff(dev, cuda)
    assert d.max() <= 8, f"{fn}: {d.max()} ulp from CUDA's function at x={x[d.argmax()]!r}"
