"""Host-side logic of numpp_b200.linalg (the numpp::linalg mirror) with the device
calls replaced by the C oracle, in the way NumPP's refgpu backend stands in for a
device (src/backend/refgpu_backend.cpp): shapes, the vector-RHS rule, the dtype
policy and the error behaviour, checked against the reference's own outputs."""
import numpy as np
import pytest

from numpp_b200 import linalg as la


class OracleBackend:
    def __init__(self, o):
        self.o = o
        self.calls = []

    def solve(self, A, B):
        self.calls.append(("solve", A.shape, B.shape))
        X, ok = self.o.solve(A, B)
        return X, (ok == 0).astype(np.int32)

    def inv(self, A):
        self.calls.append(("inv", A.shape))
        out, ok = self.o.inv(A)
        return out, (ok == 0).astype(np.int32)

    def det(self, A):
        self.calls.append(("det", A.shape))
        return self.o.det(A)

    def slogdet(self, A):
        self.calls.append(("slogdet", A.shape))
        return self.o.slogdet(A)

    def gemm(self, A, B):
        self.calls.append(("gemm", A.shape, B.shape))
        return self.o.matmul(A, B).astype(A.dtype)


@pytest.fixture()
def be(oracle):
    return OracleBackend(oracle)


def test_2d_calls(golden, be):
    M, b = golden["spd3_A"], golden["spd3_b"]
    x = la.solve(M, b, backend=be)
    assert x.shape == (3,) and np.array_equal(x, golden["spd3_x"])
    assert np.array_equal(la.inv(M, backend=be), golden["spd3_inv"])
    d = la.det(M, backend=be)
    assert d.shape == () and d == golden["spd3_det"]
    s, l = la.slogdet(M, backend=be)
    assert s == golden["spd3_sign"] and l == golden["spd3_logabs"]
    # M @ x == b (test_linalg.cpp:44-45)
    np.testing.assert_allclose(M @ x, b, rtol=1e-9, atol=1e-9)


def test_stacked_vector_and_matrix_rhs(golden, be):
    S = golden["stack_A"]
    xv = la.solve(S, golden["stack_bvec"], backend=be)
    assert xv.shape == (3, 2) and np.array_equal(xv, golden["stack_xvec"])
    xm = la.solve(S, golden["stack_bmat"], backend=be)
    assert xm.shape == (3, 2, 2) and np.array_equal(xm, golden["stack_xmat"])
    assert la.det(S, backend=be).shape == (3,)
    D = la.det(golden["det4d_A"], backend=be)
    assert D.shape == (2, 2) and np.array_equal(D, golden["det4d_det"])
    assert la.inv(S, backend=be).shape == (3, 2, 2)


def test_bvec_rule_is_numpy1(be):
    # b.ndim == a.ndim - 1 -> stack of vectors, even when b has matrix-like shape
    A = np.stack([np.eye(3) * 2] * 3)
    b = np.arange(9.0).reshape(3, 3)
    x = la.solve(A, b, backend=be)
    assert x.shape == (3, 3)
    np.testing.assert_array_equal(x, b / 2)


def test_dtype_policy(golden, be):
    x = la.solve(golden["f32_A"], golden["f32_A"], backend=be)
    assert x.dtype == np.float32 and np.array_equal(x, golden["f32_x"])
    assert la.det(np.eye(2, dtype=np.int64), backend=be).dtype == np.float64
    assert la.inv(np.eye(2, dtype=np.float16), backend=be).dtype == np.float64
    with pytest.raises(la.Declined):
        la.det(np.eye(2, dtype=np.complex128), backend=be)


def test_errors(golden, be):
    with pytest.raises(la.LinAlgError, match="^Singular matrix$"):
        la.inv(np.zeros((2, 2)), backend=be)
    with pytest.raises(la.LinAlgError, match="^Singular matrix$"):
        la.solve(golden["sing_A"], np.ones(2), backend=be)
    with pytest.raises(la.LinAlgError, match="Last 2 dimensions of the array must be square"):
        la.det(np.zeros((2, 3)), backend=be)
    with pytest.raises(la.LinAlgError, match="Last 2 dimensions"):
        la.solve(np.zeros(3), np.zeros(3), backend=be)
    with pytest.raises(la.LinAlgError, match="Last 2 dimensions"):
        la.inv(np.zeros((4, 2, 3)), backend=be)
    # one singular matrix fails the whole stacked call, as the reference loop does
    A = np.stack([np.eye(2), np.zeros((2, 2))])
    with pytest.raises(la.LinAlgError):
        la.solve(A, np.ones((2, 2)), backend=be)
    with pytest.raises(ValueError):
        la.solve(np.eye(3), np.ones(4), backend=be)
    with pytest.raises(ValueError, match="2-D"):
        la.matmul(np.ones(3), np.ones(3), backend=be)
    with pytest.raises(ValueError, match="shape mismatch"):
        la.matmul(np.ones((2, 3)), np.ones((2, 3)), backend=be)


def test_singular_det_slogdet(golden, be):
    assert la.det(golden["sing_A"], backend=be) == 0.0
    s, l = la.slogdet(golden["sing_A"], backend=be)
    assert s == 0.0 and l == -np.inf


def test_empty_and_tiny(golden, be):
    assert la.det(np.zeros((0, 0)), backend=be) == 1.0
    assert la.inv(np.zeros((0, 0)), backend=be).shape == (0, 0)
    assert la.solve(np.zeros((0, 4, 4)), np.zeros((0, 4)), backend=be).shape == (0, 4)
    assert la.det(np.zeros((0, 3, 3)), backend=be).shape == (0,)
    assert la.inv(golden["one_A"], backend=be)[0, 0] == golden["one_inv"][0, 0]


def test_matmul(golden, be):
    C = la.matmul(golden["gemm_A"], golden["gemm_B"], backend=be)
    np.testing.assert_array_equal(C, golden["gemm_C"])
    with pytest.raises(la.Declined):
        la.matmul(np.ones((2, 2), np.int64), np.ones((2, 2), np.int64), backend=be)


def test_stack_is_passed_as_one_batch(be):
    A = np.stack([np.eye(4) * (i + 1) for i in range(6)]).reshape(2, 3, 4, 4)
    la.det(A, backend=be)
    assert be.calls[-1] == ("det", (6, 4, 4))
