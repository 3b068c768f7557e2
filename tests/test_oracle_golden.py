"""The C oracle pinned against outputs of the reference itself (tests/golden/),
and, where oracle/_ref is present, against live reference calls on random inputs."""
import numpy as np
import pytest

from numpp_b200 import workloads


def bits_equal(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def test_known_answers(golden, oracle):
    # test_linalg.cpp:40-59: 3x3 SPD
    x, ok = oracle.solve(golden["spd3_A"][None], golden["spd3_b"][None, :, None])
    assert ok.all() and bits_equal(x[0, :, 0], golden["spd3_x"])
    inv, _ = oracle.inv(golden["spd3_A"][None])
    assert bits_equal(inv[0], golden["spd3_inv"])
    assert bits_equal(oracle.det(golden["spd3_A"][None])[0], golden["spd3_det"])
    s, la = oracle.slogdet(golden["spd3_A"][None])
    assert bits_equal(s[0], golden["spd3_sign"]) and bits_equal(la[0], golden["spd3_logabs"])
    # test_batched_linalg.cpp: arange stack, every det is -2 (to rounding)
    S = golden["stack_A"]
    assert bits_equal(oracle.det(S), golden["stack_det"])
    np.testing.assert_allclose(golden["stack_det"], [-2.0, -2.0, -2.0], rtol=1e-13)
    assert bits_equal(oracle.inv(S)[0], golden["stack_inv"])
    s, la = oracle.slogdet(S)
    assert bits_equal(s, golden["stack_sign"]) and bits_equal(la, golden["stack_logabs"])
    xv, _ = oracle.solve(S, golden["stack_bvec"][..., None])
    assert bits_equal(xv[..., 0], golden["stack_xvec"])
    xm, _ = oracle.solve(S, golden["stack_bmat"])
    assert bits_equal(xm, golden["stack_xmat"])
    assert bits_equal(oracle.det(golden["det4d_A"].reshape(4, 3, 3)).reshape(2, 2), golden["det4d_det"])


def test_edge_cases(golden, oracle):
    assert bits_equal(oracle.inv(golden["one_A"][None])[0][0], golden["one_inv"])
    assert bits_equal(oracle.det(golden["one_A"][None])[0], golden["one_det"])
    assert oracle.det(np.zeros((1, 0, 0)))[0] == golden["empty_det"] == 1.0
    # singular: det 0, slogdet (0, -inf), solve/inv report failure
    Sg = golden["sing_A"][None]
    assert oracle.det(Sg)[0] == golden["sing_det"] == 0.0
    s, la = oracle.slogdet(Sg)
    assert s[0] == golden["sing_sign"] == 0.0 and la[0] == golden["sing_logabs"] == -np.inf
    assert oracle.inv(np.zeros((1, 2, 2)))[1][0] == 0 and str(golden["zeros_inv_err"]) == "Singular matrix"
    assert oracle.solve(Sg, np.ones((1, 2, 1)))[1][0] == 0
    assert str(golden["nonsquare_err"]) == "Last 2 dimensions of the array must be square"


def test_nodal_and_gemm(golden, oracle):
    G, I = golden["nodal_G"], golden["nodal_I"]
    x, _ = oracle.solve(G[None], I[None, :, None])
    assert bits_equal(x[0, :, 0], golden["nodal_v"])
    assert bits_equal(oracle.det(G[None])[0], golden["nodal_det"])
    assert bits_equal(oracle.inv(G[None])[0][0], golden["nodal_inv"])
    assert bits_equal(oracle.matmul(golden["gemm_A"], golden["gemm_B"]), golden["gemm_C"])


def test_seeded_batches(golden, oracle):
    A, B = golden["u16_A"], golden["u16_B"]
    x, ok = oracle.solve(A, B)
    assert ok.all() and bits_equal(x, golden["u16_x"])
    assert bits_equal(oracle.det(A), golden["u16_det"])
    s, la = oracle.slogdet(A)
    assert bits_equal(s, golden["u16_sign"]) and bits_equal(la, golden["u16_logabs"])
    assert bits_equal(oracle.inv(A)[0], golden["u16_inv"])
    sys_ = {k[len("uneven_"):]: golden[k] for k in golden if k.startswith("uneven_")}
    sys_["inv_size"] = int(sys_["inv_size"])
    X, s, la, inv, ok = oracle.solve_grouped(sys_)
    assert bits_equal(X, golden["uneven_x"]) and bits_equal(s, golden["uneven_sign"])
    assert bits_equal(la, golden["uneven_logabs"]) and bits_equal(inv, golden["uneven_inv"])
    assert np.array_equal(ok, golden["uneven_ok"])


def test_generator_matches_reference_rng(golden):
    """numpy's default_rng draws are the reference generator's (PCG64 + ziggurat)."""
    for seed in (12345, 7):
        g = np.random.default_rng(seed)
        assert bits_equal(g.standard_normal(64), golden[f"rng{seed}_normal_a"])
        assert bits_equal(g.standard_normal(16), golden[f"rng{seed}_normal_b"])
        u = np.random.default_rng(seed).uniform(np.log(4.0), np.log(513.0), 32)
        assert bits_equal(u, golden[f"rng{seed}_uniform"])
    A1, B1 = workloads.uniform_batch(seed=12345, count=16, n=32, nrhs=1)
    assert bits_equal(A1, golden["u16_A"]) and bits_equal(B1, golden["u16_B"])


def test_pivots_follow_reference_rule(oracle):
    """Ties go to the first maximum in position order (strict '>' scan)."""
    A = np.array([[[1.0, 2.0], [-1.0, 3.0]]])  # |a00| == |a10|: no swap
    _, piv, sgn, ok = oracle.lu(A)
    assert ok[0] == 1 and list(piv[0]) == [0, 1] and sgn[0] == 1.0
    A = np.array([[[1.0, 2.0], [-2.0, 3.0]]])
    _, piv, sgn, _ = oracle.lu(A)
    assert list(piv[0]) == [1, 0] and sgn[0] == -1.0


@pytest.mark.parametrize("n", [1, 2, 5, 17, 33, 64])
def test_oracle_vs_live_reference(ref, oracle, n):
    rng = np.random.default_rng(100 + n)
    A = rng.standard_normal((6, n, n))
    B = rng.standard_normal((6, n, 3))
    x, ok = oracle.solve(A, B)
    assert ok.all() and bits_equal(x, ref.solve(A, B))
    assert bits_equal(oracle.det(A), ref.det(A))
    s, la = oracle.slogdet(A)
    rs, rla = ref.slogdet(A)
    assert bits_equal(s, rs) and bits_equal(la, rla)
    assert bits_equal(oracle.inv(A)[0], ref.inv(A))


def test_oracle_vs_numpy_tolerance(oracle):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((8, 20, 20)) + 20 * np.eye(20)
    B = rng.standard_normal((8, 20, 2))
    x, _ = oracle.solve(A, B)
    np.testing.assert_allclose(x, np.linalg.solve(A, B), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(oracle.det(A), np.linalg.det(A), rtol=1e-12)


def test_matrix_power_known_answers(golden, oracle):
    """test_linalg_mined3.cpp:29-40 and a seeded stack: the restatement of
    linalg.cpp:440-454 reproduces the reference bit for bit."""
    P = golden["mp2_A"][None]
    for p in (0, 1, 2, 7, -1, -3):
        R, ok = oracle.matrix_power(P, p)
        assert ok.all() and bits_equal(R[0], golden[f"mp2_p{p}"]), p
    np.testing.assert_allclose(golden["mp2_p-3"], np.linalg.matrix_power(golden["mp2_A"], -3), rtol=1e-12)
    for p in (3, 8, -2, -4):
        R, ok = oracle.matrix_power(golden["mp9_A"], p)
        assert ok.all() and bits_equal(R, golden[f"mp9_p{p}"]), p
    _, ok = oracle.matrix_power(golden["sing_A"][None], -1)
    assert ok[0] == 0 and str(golden["mp_sing_err"]) == "Singular matrix"
    assert golden["mp2_f32_p0"].dtype == np.float32


def test_tensor_solve_known_answers(golden, oracle):
    """tensor_solve.cpp:10-49 is a reshape around solve / inv: the oracle's solve
    and inv on the reshaped matrices give the reference's tensorsolve / tensorinv."""
    T, b = golden["tens_A"], golden["tens_b"]
    x, ok = oracle.solve(T.reshape(1, 4, 4), b.reshape(1, 4, 1))
    assert ok.all() and bits_equal(x.reshape(2, 2), golden["tens_x"])
    Tm = np.ascontiguousarray(np.transpose(T, (1, 2, 3, 0))).reshape(1, 4, 4)
    x, _ = oracle.solve(Tm, b.reshape(1, 4, 1))
    assert bits_equal(x.reshape(2, 2), golden["tens_x_ax0"])
    inv, _ = oracle.inv(T.reshape(1, 4, 4))
    assert bits_equal(inv.reshape(2, 2, 2, 2), golden["tens_inv"])
    x, _ = oracle.solve(golden["tens3_A"].reshape(1, 12, 12), golden["tens3_b"].reshape(1, 12, 1))
    assert bits_equal(x.reshape(12), golden["tens3_x"])
    inv, _ = oracle.inv(golden["tens4_A"].reshape(1, 24, 24))
    assert bits_equal(inv.reshape(8, 3, 4, 6), golden["tens4_inv"])
    assert str(golden["tensinv_ind0_err"]) == "Invalid ind argument"


def test_cholesky_known_answers(golden, oracle):
    """test_linalg.cpp:61-69 and test_batched_linalg.cpp:53-58 plus a seeded
    stack: the restatement of linalg.cpp:117-136 is bit-exact with the reference."""
    L, ok = oracle.cholesky(golden["spd3_A"][None])
    assert ok.all() and bits_equal(L[0], golden["chol_spd3"])
    L, ok = oracle.cholesky(golden["chol_stack_A"])
    assert ok.all() and bits_equal(L, golden["chol_stack_L"])
    L, ok = oracle.cholesky(golden["chol40_A"])
    assert ok.all() and bits_equal(L, golden["chol40_L"])
    _, ok = oracle.cholesky(np.array([[[-1.0, 0], [0, -1]]]))
    assert ok[0] == 0 and str(golden["chol_notpd_err"]) == "Matrix is not positive definite"


LSQ_CASES = ("R", "W", "tall", "wide", "sq", "def")


def test_lstsq_known_answers(golden, oracle):
    """test_linalg3.cpp:70-77 and seeded tall / wide / square / rank-deficient
    problems: the restatement of the reference's Jacobi SVD and lstsq
    (linalg.cpp:620-712, 755-784) reproduces its solution, residuals, rank and
    singular values bit for bit."""
    for key in LSQ_CASES:
        x, res, rk, sv = oracle.lstsq(golden[f"lsq_{key}_A"], golden[f"lsq_{key}_b"])
        assert bits_equal(x, golden[f"lsq_{key}_x"]), key
        assert bits_equal(sv, golden[f"lsq_{key}_s"]), key
        assert rk == int(golden[f"lsq_{key}_rank"]), key
        assert bits_equal(res, golden[f"lsq_{key}_res"]), key
    assert int(golden["lsq_def_rank"]) == 4 and golden["lsq_def_res"].size == 0
    np.testing.assert_allclose(golden["lsq_R_x"], np.linalg.lstsq(golden["lsq_R_A"], golden["lsq_R_b"], rcond=None)[0],
                               rtol=1e-12)
