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

    def gemm_batched(self, A, B):
        self.calls.append(("gemm_batched", A.shape, B.shape))
        return np.stack([self.o.matmul(A[i], B[i]) for i in range(A.shape[0])])

    def cholesky(self, A):
        self.calls.append(("cholesky", A.shape))
        Lm, ok = self.o.cholesky(A)
        return Lm, (ok == 0).astype(np.int32)

    def lstsq(self, A, B, rcond):
        self.calls.append(("lstsq", A.shape, B.shape))
        x, res, rk, sv = self.o.lstsq(A[0], B[0], rcond)
        has = np.array([1 if res.size else 0], np.int32)
        r = np.zeros((1, B.shape[-1]))
        if res.size:
            r[0] = res
        return x[None], sv[None], np.array([rk], np.int32), r, has

    def svdvals(self, A):
        self.calls.append(("svdvals", A.shape))
        return np.stack([self.o.lstsq(A[i], np.zeros((A.shape[1], 1)))[3] for i in range(A.shape[0])])

    def matrix_power(self, A, p):
        self.calls.append(("matrix_power", A.shape, p))
        R, ok = self.o.matrix_power(A, p)
        return R, (ok == 0).astype(np.int32)


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


def test_matrix_power(golden, be):
    """linalg.cpp:440-454 through the mirror: same values, dtype and errors as the reference."""
    for p in (0, 1, 2, 7, -1, -3):
        R = la.matrix_power(golden["mp2_A"], p, backend=be)
        assert R.shape == (2, 2) and np.array_equal(R, golden[f"mp2_p{p}"]), p
    R = la.matrix_power(golden["mp2_A"].astype(np.float32), 0, backend=be)
    assert R.dtype == golden["mp2_f32_p0"].dtype and np.array_equal(R, golden["mp2_f32_p0"])
    for p in (3, 8, -2, -4):
        assert np.array_equal(la.matrix_power(golden["mp9_A"], p, backend=be), golden[f"mp9_p{p}"])
    with pytest.raises(la.LinAlgError, match=str(golden["mp_sing_err"])):
        la.matrix_power(golden["sing_A"], -1, backend=be)
    with pytest.raises(la.LinAlgError, match="square"):
        la.matrix_power(np.zeros((2, 3)), 2, backend=be)
    assert la.matrix_power(np.zeros((0, 4, 4)), 3, backend=be).shape == (0, 4, 4)
    # one batched call for the whole stack (batched.cpp:83-84 maps one matrix at a time)
    be.calls.clear()
    la.matrix_power(np.ones((2, 3, 5, 5)), 2, backend=be)
    assert be.calls == [("matrix_power", (6, 5, 5), 2)]


def test_tensorsolve_tensorinv(golden, be):
    """tensor_solve.cpp:10-49 semantics against the reference's own outputs."""
    T, b = golden["tens_A"], golden["tens_b"]
    x = la.tensorsolve(T, b, backend=be)
    assert x.shape == (2, 2) and np.array_equal(x, golden["tens_x"])
    assert np.array_equal(la.tensorsolve(T, b, axes=(0,), backend=be), golden["tens_x_ax0"])
    ti = la.tensorinv(T, 2, backend=be)
    assert ti.shape == (2, 2, 2, 2) and np.array_equal(ti, golden["tens_inv"])
    x3 = la.tensorsolve(golden["tens3_A"], golden["tens3_b"], backend=be)
    assert x3.shape == (12,) and np.array_equal(x3, golden["tens3_x"])
    t4 = la.tensorinv(golden["tens4_A"], 2, backend=be)
    assert t4.shape == (8, 3, 4, 6) and np.array_equal(t4, golden["tens4_inv"])
    np.testing.assert_allclose(x3, np.linalg.tensorsolve(golden["tens3_A"], golden["tens3_b"]), rtol=1e-10)
    with pytest.raises(ValueError, match=str(golden["tensinv_ind0_err"])):
        la.tensorinv(T, 0, backend=be)
    with pytest.raises(ValueError, match="Invalid ind"):
        la.tensorinv(T, 5, backend=be)
    with pytest.raises(la.LinAlgError, match="must equal"):
        la.tensorsolve(np.ones((2, 3, 5)), np.ones((2, 3)), backend=be)


def test_matmul_batched(golden, be):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((2, 3, 4, 5))
    B = rng.standard_normal((3, 5, 6))          # broadcasts over the leading 2
    Cm = la.matmul_batched(A, B, backend=be)
    assert Cm.shape == (2, 3, 4, 6)
    np.testing.assert_allclose(Cm, A @ B, rtol=1e-13, atol=1e-13)
    assert be.calls[-1] == ("gemm_batched", (6, 4, 5), (6, 5, 6))
    assert la.matmul_batched(A.astype(np.float32), B.astype(np.float32), backend=be).dtype == np.float32
    assert la.matmul_batched(np.zeros((0, 2, 3)), np.zeros((0, 3, 4)), backend=be).shape == (0, 2, 4)
    with pytest.raises(ValueError, match="shape mismatch"):
        la.matmul_batched(A, A, backend=be)
    with pytest.raises(la.Declined):
        la.matmul_batched(A.astype(np.complex128), B, backend=be)


def test_cond(be):
    rng = np.random.default_rng(6)
    A = rng.standard_normal((3, 7, 7)) + 3 * np.eye(7)
    for p in (1, -1, np.inf, -np.inf, "fro"):
        c = la.cond(A, p, backend=be)
        np.testing.assert_allclose(c, np.linalg.cond(A, p), rtol=1e-12)
        assert isinstance(la.cond(A[0], p, backend=be), np.floating)
    S = np.stack([A[0], np.zeros((7, 7))])
    c = la.cond(S, 1, backend=be)
    assert np.isfinite(c[0]) and c[1] == np.inf   # singular -> inf (tensor.cpp:361-368)
    for p in (None, 2, -2):  # from the singular values
        np.testing.assert_allclose(la.cond(A, p, backend=be), np.linalg.cond(A, p), rtol=1e-11)
    with pytest.raises(ValueError):
        la.cond(A, "nuc", backend=be)


def test_device_mirror_declines_host_tensors():
    """numpp_b200.device serves CUDA tensors only; host tensors go to the host mirror."""
    torch = pytest.importorskip("torch")
    from numpp_b200 import device as dev
    with pytest.raises(la.Declined):
        dev.det(torch.eye(3, dtype=torch.float64))
    with pytest.raises(la.Declined):
        dev.solve(torch.eye(3, dtype=torch.float64), torch.ones(3, dtype=torch.float64))
    with pytest.raises(la.Declined):       # numpy speaks DLPack too, from the host
        dev.inv(np.eye(3))
    with pytest.raises(TypeError):
        dev.inv([[1.0, 0.0], [0.0, 1.0]])


def test_cholesky(golden, be):
    """linalg.cpp:117-136 through the mirror, against the reference's outputs."""
    assert np.array_equal(la.cholesky(golden["spd3_A"], backend=be), golden["chol_spd3"])
    assert np.array_equal(la.cholesky(golden["chol_stack_A"], backend=be), golden["chol_stack_L"])
    assert np.array_equal(la.cholesky(golden["chol40_A"], backend=be), golden["chol40_L"])
    with pytest.raises(la.LinAlgError, match=str(golden["chol_notpd_err"])):
        la.cholesky(np.array([[-1.0, 0], [0, -1]]), backend=be)
    with pytest.raises(la.LinAlgError, match="square"):
        la.cholesky(np.ones((2, 3)), backend=be)
    assert la.cholesky(np.eye(3, dtype=np.float32), backend=be).dtype == np.float32
    assert la.cholesky(np.zeros((0, 5, 5)), backend=be).shape == (0, 5, 5)
    be.calls.clear()
    la.cholesky(np.stack([np.eye(4)] * 6).reshape(2, 3, 4, 4), backend=be)
    assert be.calls == [("cholesky", (6, 4, 4))]


def test_step_update_bytes_counts():
    """The algorithmic-bytes model behind the bench's HBM roofline of the
    trailing update, on one system counted by hand."""
    from numpp_b200 import workloads
    sys_ = {"n": np.array([64, 20]), "nrhs": np.array([1, 3]), "inv_off": np.array([-1, 0])}
    # n = 64, one right-hand side, no inverse: step 0 has 32 rows below and
    # 32 + 1 trailing columns (one strip), step 32 only the row-move pass on 1 column;
    # the order-20 system takes the warp kernel and adds nothing
    want = (16 * 32 * 33 + 8 * 32 * 32 * 1 + 16 * 32 * 33) + (16 * 32 * 1)
    assert workloads.step_update_bytes(sys_) == want


def test_lstsq_mirror(golden, be):
    """linalg.cpp:755-784 semantics through the mirror, against the reference's outputs."""
    for key in ("R", "W", "tall", "wide", "sq", "def"):
        x, res, rk, sv = la.lstsq(golden[f"lsq_{key}_A"], golden[f"lsq_{key}_b"], backend=be)
        assert np.array_equal(x, golden[f"lsq_{key}_x"]), key
        assert np.array_equal(res, golden[f"lsq_{key}_res"]), key
        assert rk == int(golden[f"lsq_{key}_rank"]) and np.array_equal(sv, golden[f"lsq_{key}_s"]), key
    assert la.lstsq(golden["lsq_R_A"], golden["lsq_R_b"], backend=be)[0].shape == (3,)
    with pytest.raises(la.LinAlgError):
        la.lstsq(np.ones((2, 3, 4)), np.ones((2, 3)), backend=be)
    x, res, rk, sv = la.lstsq(np.zeros((0, 3)), np.zeros(0), backend=be)
    assert x.shape == (3,) and rk == 0
    np.testing.assert_allclose(la.svdvals(golden["lsq_tall_A"], backend=be), golden["lsq_tall_s"], rtol=1e-14)
