"""Regenerate tests/golden/*.npz from the reference itself.

Runs NumPP's own CPU path (oracle/_ref/libnumpp_ref.so, built by
``make -C oracle ref`` from the reference sources) on the known-answer cases of
NumPP's tests and on small seeded workloads, and stores inputs + outputs:

* tests/test_linalg.cpp:13-20,40-59       3x3 SPD solve / inv / det / slogdet, singular inv
* tests/test_batched_linalg.cpp:14-75,125-136   (3,2,2) arange stack, (2,2,3,3) det
* tests/test_linalg_mined.cpp:82-112,191-196    0x0, 1x1, float32 dtype preservation
* tests/test_linalg_mined3.cpp:129-136           singular det / slogdet
* examples/ee02_nodal_analysis.cpp:44-69         nodal conductance solve / det / inv
* tests/test_gpu.cpp:56-69                        the 40x50 @ 50x30 GEMM
* seeded uniform batch (16 x 32x32 + 32 I) and a seeded uneven batch (n in 1..80)
* numpp::random::default_rng draws (PCG64 + ziggurat) for seeds 12345 / 7
* tests/test_linalg_mined3.cpp:29-40             matrix_power of [[1,2],[3,4]] for 0, 1, 2, 7, -1, -3
* tests/test_tensor_solve.cpp:9-71                tensorsolve / tensorinv of the (2,2,2,2) tridiagonal
* a seeded (6, 9, 9) stack to the powers 3, 8, -2, -4 (src/linalg/batched.cpp:83-84)
* tests/test_linalg3.cpp:12-25,70-77        lstsq of the 4x3 and 3x4 matrices, plus seeded tall,
  wide, square and rank-deficient problems (solution, residuals, rank, singular values)
* tests/test_linalg.cpp:61-69, tests/test_batched_linalg.cpp:53-58   cholesky of the 3x3 SPD
  matrix, of the (2,2,2) stack, the not-positive-definite error, and a seeded (5, 40, 40) stack

Usage: python tests/golden/make_golden.py   (needs oracle/_ref; run where it was built)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import load_ref  # noqa: E402
from oracle.oracle import RefError  # noqa: E402
from numpp_b200 import workloads  # noqa: E402


def err_of(fn, *a):
    try:
        fn(*a)
    except RefError as e:
        return str(e)
    return ""


def main():
    r = load_ref()
    g = {}
    M = np.array([[4.0, 2, 1], [2, 5, 3], [1, 3, 6]])
    b3 = np.array([1.0, 2, 3])
    g["spd3_A"], g["spd3_b"] = M, b3
    g["spd3_x"] = r.solve(M, b3)
    g["spd3_inv"] = r.inv(M)
    g["spd3_det"] = r.det(M)
    g["spd3_sign"], g["spd3_logabs"] = r.slogdet(M)

    S = np.arange(12.0).reshape(3, 2, 2)
    g["stack_A"] = S
    g["stack_det"] = r.det(S)
    g["stack_inv"] = r.inv(S)
    g["stack_sign"], g["stack_logabs"] = r.slogdet(S)
    g["stack_bvec"] = np.arange(1.0, 7.0).reshape(3, 2)
    g["stack_xvec"] = r.solve(S, g["stack_bvec"])
    g["stack_bmat"] = np.arange(1.0, 13.0).reshape(3, 2, 2)
    g["stack_xmat"] = r.solve(S, g["stack_bmat"])
    D4 = np.arange(36.0).reshape(2, 2, 3, 3)
    g["det4d_A"], g["det4d_det"] = D4, r.det(D4)

    g["one_A"] = np.array([[5.0]])
    g["one_inv"], g["one_det"] = r.inv(g["one_A"]), r.det(g["one_A"])
    g["empty_det"] = r.det(np.zeros((0, 0)))
    g["empty_inv_shape"] = np.array(r.inv(np.zeros((0, 0))).shape)

    Sg = np.array([[1.0, 2], [2, 4]])
    g["sing_A"] = Sg
    g["sing_det"] = r.det(Sg)
    g["sing_sign"], g["sing_logabs"] = r.slogdet(Sg)
    g["zeros_inv_err"] = np.array(err_of(r.inv, np.zeros((2, 2))))
    g["sing_solve_err"] = np.array(err_of(r.solve, Sg, np.array([1.0, 1.0])))
    g["nonsquare_err"] = np.array(err_of(r.det, np.zeros((2, 3))))

    F = np.array([[1, 0.5], [0.5, 1]], np.float32)
    g["f32_A"] = F
    g["f32_x"] = r.solve(F, F)

    G = np.array([[3.5, -1.0, -2.0, 0.0], [-1.0, 3.0, -0.5, -1.5], [-2.0, -0.5, 3.5, -1.0],
                  [0.0, -1.5, -1.0, 4.5]])
    I = np.array([2.0, 0.0, -1.0, 3.0])
    g["nodal_G"], g["nodal_I"] = G, I
    g["nodal_v"], g["nodal_det"], g["nodal_inv"] = r.solve(G, I), r.det(G), r.inv(G)

    A = np.arange(0.0, 2000.0).reshape(40, 50)
    B = np.arange(0.0, 1500.0).reshape(50, 30) * 0.001
    g["gemm_A"], g["gemm_B"], g["gemm_C"] = A, B, r.matmul(A, B)

    A1, B1 = workloads.uniform_batch(seed=12345, count=16, n=32, nrhs=1)
    g["u16_A"], g["u16_B"] = A1, B1
    g["u16_x"] = r.solve(A1, B1)
    g["u16_det"] = r.det(A1)
    g["u16_sign"], g["u16_logabs"] = r.slogdet(A1)
    g["u16_inv"] = r.inv(A1)

    sysu = workloads.uneven_batch(seed=7, count=40, n_lo=1, n_hi=80, nrhs_choices=(1, 3, 8),
                                  inv_fraction=0.25)
    X, s, la, inv, ok = r.solve_grouped(sysu)
    for k in ("n", "nrhs", "a_off", "b_off", "inv_off", "A", "B"):
        g["uneven_" + k] = sysu[k]
    g["uneven_inv_size"] = np.array(sysu["inv_size"])
    g["uneven_x"], g["uneven_sign"], g["uneven_logabs"], g["uneven_inv"], g["uneven_ok"] = X, s, la, inv, ok

    P = np.array([[1.0, 2], [3, 4]])
    g["mp2_A"] = P
    for p in (0, 1, 2, 7, -1, -3):
        g[f"mp2_p{p}"] = r.matrix_power(P, p)
    g["mp2_f32_p0"] = r.matrix_power(P.astype(np.float32), 0)
    g["mp_sing_err"] = np.array(err_of(r.matrix_power, Sg, -1))
    rng = np.random.default_rng(2024)
    Ms = rng.standard_normal((6, 9, 9)) / 3.0 + 0.5 * np.eye(9)
    g["mp9_A"] = Ms
    for p in (3, 8, -2, -4):
        g[f"mp9_p{p}"] = r.matrix_power(Ms, p)

    g["chol_spd3"] = r.cholesky(M)
    S2 = np.array([[[2.0, 0], [0, 3]], [[4, 1], [1, 3]]])
    g["chol_stack_A"], g["chol_stack_L"] = S2, r.cholesky(S2)
    g["chol_notpd_err"] = np.array(err_of(r.cholesky, np.array([[-1.0, 0], [0, -1]])))
    Xc = np.random.default_rng(77).standard_normal((5, 40, 40))
    Ac = Xc @ Xc.transpose(0, 2, 1) + 40 * np.eye(40)
    Ac[:, 0, 39] = 7.0  # the upper triangle is never read
    g["chol40_A"], g["chol40_L"] = Ac, r.cholesky(Ac)

    rl = np.random.default_rng(99)
    Rm = np.array([[1.0, 2, 3], [4, 5, 6], [7, 8, 10], [1, 0, 2]])
    lcases = {"R": (Rm, np.array([1.0, 2, 3, 4])),
              "W": (np.array([[1.0, 4, 7, 1], [2, 5, 8, 0], [3, 6, 10, 2]]), np.array([1.0, 2, 3])),
              "tall": (rl.standard_normal((30, 8)), rl.standard_normal((30, 3))),
              "wide": (rl.standard_normal((7, 19)), rl.standard_normal((7, 2))),
              "sq": (rl.standard_normal((24, 24)), rl.standard_normal(24)),
              "def": (np.hstack([rl.standard_normal((16, 4))] * 2), rl.standard_normal((16, 2)))}
    for key, (Al, Bl) in lcases.items():
        x, res, rk, sv = r.lstsq(Al, Bl)
        g[f"lsq_{key}_A"], g[f"lsq_{key}_b"] = Al, Bl
        g[f"lsq_{key}_x"], g[f"lsq_{key}_res"] = x, res
        g[f"lsq_{key}_rank"], g[f"lsq_{key}_s"] = np.array(rk), sv

    T = np.array([4.0, 1, 0, 0, 1, 4, 1, 0, 0, 1, 4, 1, 0, 0, 1, 4]).reshape(2, 2, 2, 2)
    bt = np.array([1.0, 2, 3, 4]).reshape(2, 2)
    g["tens_A"], g["tens_b"] = T, bt
    g["tens_x"] = r.tensorsolve(T, bt).reshape(2, 2)
    g["tens_x_ax0"] = r.tensorsolve(T, bt, (0,)).reshape(2, 2)
    g["tens_inv"] = r.tensorinv(T, 2).reshape(2, 2, 2, 2)
    T3 = rng.standard_normal((3, 4, 12))
    b3r = rng.standard_normal((3, 4))
    g["tens3_A"], g["tens3_b"] = T3, b3r
    g["tens3_x"] = r.tensorsolve(T3, b3r).reshape(12)
    T4 = rng.standard_normal((4, 6, 8, 3))
    g["tens4_A"] = T4
    g["tens4_inv"] = r.tensorinv(T4, 2).reshape(8, 3, 4, 6)
    g["tensinv_ind0_err"] = np.array(err_of(r.tensorinv, T, 0))
    g["tenssolve_shape_err"] = np.array(err_of(r.tensorsolve, rng.standard_normal((2, 3, 5)), b3r[:2, :3]))

    for seed in (12345, 7):
        a, b = r.standard_normal2(seed, 64, 16)
        g[f"rng{seed}_normal_a"], g[f"rng{seed}_normal_b"] = a, b
        g[f"rng{seed}_uniform"] = r.uniform(seed, np.log(4.0), np.log(513.0), 32)

    out = os.path.join(HERE, "reference_cases.npz")
    np.savez_compressed(out, **g)
    print(out, os.path.getsize(out), "bytes,", len(g), "arrays")


if __name__ == "__main__":
    main()
