"""The drop-in through NumPP's own front end.

oracle/_ref/dropin/libnumpp_dropin.so is NumPP's unmodified portable sources
built with this repository's GpuVTable header, numpp_b200/csrc/vtable.cpp in
place of gpu_null.cpp, and numpp_b200/frontend/linalg_dispatch.cpp defining
numpp::linalg::{solve, inv, det, slogdet, matrix_power} over the vtable's
batched slots (the reference's own definitions, compiled under ref_* names,
serve what the device does not). It is called here through the same extern
"C" shim as the reference library, i.e. the way a NumPP user calls
numpp::linalg::solve and friends.

Without a device (the CPU tests) the vtable is null and every call must give
the reference's own bits. On a B200 the calls must reach the device
(last_backend() == Cuda), for stacks and for 2-D arrays, and agree with the
oracle at the parity bar: solutions within 1e-12 * cond(A), det / slogdet
signs bit-exact, values within the same bound; singular matrices raise the
reference's linalg_error for solve / inv and give det 0, slogdet (0, -inf).
"""
import os

import numpy as np
import pytest


@pytest.fixture(scope="module")
def dropin():
    from oracle.oracle import DROPIN_SO, RefLib
    if not os.path.exists(DROPIN_SO):
        pytest.skip("oracle/_ref/dropin (the drop-in build of the reference) is not present here")
    return RefLib(DROPIN_SO)


def _cases(seed=0):
    rng = np.random.default_rng(seed)
    A3 = rng.standard_normal((4, 48, 48)) + 48 * np.eye(48)
    A4 = rng.standard_normal((2, 3, 20, 20))
    A2 = rng.standard_normal((70, 70))
    return rng, A3, A4, A2


def test_without_a_device_the_dropin_is_the_reference(dropin, ref):
    from numpp_b200 import _lib
    if _lib.load().nppb_device_available() == 1:
        pytest.skip("a device is present: the GPU tests cover the drop-in")
    rng, A3, A4, A2 = _cases()
    B3 = rng.standard_normal((4, 48, 2))
    calls = ((lambda L: L.solve(A3, B3)), (lambda L: L.solve(A2, A2[:, 0].copy())), (lambda L: L.inv(A4)),
             (lambda L: L.det(A4)), (lambda L: L.slogdet(A2)), (lambda L: L.matrix_power(A3, -3)))
    for f in calls:
        got, want = f(dropin), f(ref)
        for g, w in zip(got if isinstance(got, tuple) else (got,), want if isinstance(want, tuple) else (want,)):
            assert np.array_equal(g, w)
    assert dropin.last_backend() != dropin.BACKEND_CUDA


@pytest.mark.gpu
def test_stacks_and_2d_reach_the_device(lib, dropin, oracle):
    from test_gpu_parity import check_solution
    rng, A3, A4, A2 = _cases(1)
    cond = lambda A: np.linalg.cond(A).max()  # noqa: E731

    def on_device(fn, *a):
        dropin.clear_last_backend()
        r = fn(*a)
        assert dropin.last_backend() == dropin.BACKEND_CUDA, fn
        return r

    # solve: stacked with matrix and vector right-hand sides, 2-D with both
    B3 = rng.standard_normal((4, 48, 3))
    check_solution(on_device(dropin.solve, A3, B3), oracle.solve(A3, B3)[0], A3)
    b3 = rng.standard_normal((4, 48))
    x3 = on_device(dropin.solve, A3, b3)
    assert x3.shape == (4, 48)
    check_solution(x3[..., None], oracle.solve(A3, b3[..., None])[0], A3)
    for B2 in (rng.standard_normal(70), rng.standard_normal((70, 5))):
        x2 = on_device(dropin.solve, A2, B2)
        assert x2.shape == B2.shape
        check_solution(x2.reshape(1, 70, -1), oracle.solve(A2[None], B2.reshape(1, 70, -1))[0], A2[None])
    # inv, det, slogdet on a 4-D stack and a 2-D array
    A4f = A4.reshape(6, 20, 20)
    check_solution(on_device(dropin.inv, A4).reshape(6, 20, 20), oracle.inv(A4f)[0], A4f)
    d4 = on_device(dropin.det, A4)
    assert d4.shape == (2, 3)
    do = oracle.det(A4f)
    assert np.array_equal(np.sign(d4.ravel()), np.sign(do))
    np.testing.assert_allclose(d4.ravel(), do, rtol=1e-12 * cond(A4f))
    s2, l2 = on_device(dropin.slogdet, A2)
    so, lo = oracle.slogdet(A2[None])
    assert s2.shape == () and s2 == so[0]
    assert abs(l2 - lo[0]) <= 1e-12 * cond(A2[None]) * max(1.0, abs(lo[0]))
    check_solution(on_device(dropin.inv, A2)[None], oracle.inv(A2[None])[0], A2[None])
    # matrix_power, 2-D and stacked, negative powers through the inverse
    for A, p in ((A2, 3), (A3, -2), (A3, 0)):
        got = on_device(dropin.matrix_power, A, p)
        want, ok = oracle.matrix_power(A.reshape(-1, A.shape[-1], A.shape[-1]), p)
        assert ok.all()
        np.testing.assert_allclose(got.reshape(want.shape), want, rtol=1e-10, atol=1e-10 * np.abs(want).max())


@pytest.mark.gpu
def test_dtype_policy_and_errors_through_the_front_end(lib, dropin, ref):
    from oracle.oracle import RefError
    rng = np.random.default_rng(2)
    A = (rng.standard_normal((3, 30, 30)) + 30 * np.eye(30)).astype(np.float32)
    B = rng.standard_normal((3, 30, 2)).astype(np.float32)
    dropin.clear_last_backend()
    x = dropin.solve(A, B)
    assert x.dtype == np.float32 and dropin.last_backend() == dropin.BACKEND_CUDA
    np.testing.assert_allclose(x, ref.solve(A, B), rtol=1e-5, atol=1e-6)
    # singular stacks: solve / inv raise the reference's error, det 0, slogdet (0, -inf)
    S = rng.standard_normal((2, 16, 16))
    S[1, 3] = 0.0
    for fn in (lambda: dropin.solve(S, np.ones((2, 16, 1))), lambda: dropin.inv(S)):
        with pytest.raises(RefError, match="Singular matrix"):
            fn()
    d = dropin.det(S)
    assert d[1] == 0.0 and d[0] != 0.0
    s, la = dropin.slogdet(S)
    assert s[1] == 0.0 and np.isneginf(la[1])
    # non-square: the reference's own error, from its own code
    with pytest.raises(RefError, match="square"):
        dropin.inv(rng.standard_normal((2, 4, 5)))
