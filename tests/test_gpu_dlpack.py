"""DLPack device handoff: device-resident stacks in, device results out, through
nppb_dl_linalg / nppb_dl_matmul, against the oracle (same bar as the host path:
x within 1e-12 * cond(A), det / slogdet within 1e-12 * cond(A) relative)."""
import numpy as np
import pytest

from numpp_b200 import _lib
from numpp_b200 import device as dev
from numpp_b200 import linalg as la

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


class Foreign:
    """A non-torch DLPack producer (what CuPy or JAX would hand over)."""

    def __init__(self, t):
        self.t = t

    def __dlpack__(self, stream=None):
        return self.t.__dlpack__(stream=stream)

    def __dlpack_device__(self):
        return self.t.__dlpack_device__()


def _stack(seed, count, n):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((count, n, n)) + np.sqrt(n) * np.eye(n)


@pytest.mark.parametrize("count,n,k", [(7, 5, 3), (64, 40, 1), (16, 100, 8), (3, 600, 2)])
def test_solve_on_device_matches_oracle(lib, oracle, count, n, k):
    A = _stack(count + n, count, n)
    B = np.random.default_rng(n).standard_normal((count, n, k))
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    X = dev.solve(dA, dB)
    assert X.is_cuda and X.dtype == torch.float64 and tuple(X.shape) == (count, n, k)
    Xo, ok = oracle.solve(A, B)
    cond = np.linalg.cond(A)
    err = np.linalg.norm((X.cpu().numpy() - Xo).reshape(count, -1), axis=1)
    assert np.all(err <= 1e-12 * cond * np.linalg.norm(Xo.reshape(count, -1), axis=1))


def test_vector_rhs_inv_det_slogdet(lib, oracle):
    A = _stack(3, 9, 48)
    b = np.random.default_rng(4).standard_normal((9, 48))
    dA = torch.from_numpy(A).cuda()
    x = dev.solve(dA, torch.from_numpy(b).cuda())
    assert tuple(x.shape) == (9, 48)
    xo, _ = oracle.solve(A, b[..., None])
    np.testing.assert_allclose(x.cpu().numpy(), xo[..., 0], rtol=1e-10, atol=1e-12)
    inv = dev.inv(dA).cpu().numpy()
    io, _ = oracle.inv(A)
    np.testing.assert_allclose(inv, io, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(dev.det(dA).cpu().numpy(), oracle.det(A), rtol=1e-11)
    s, l = dev.slogdet(dA)
    so, lo = oracle.slogdet(A)
    assert np.array_equal(s.cpu().numpy(), so)
    np.testing.assert_allclose(l.cpu().numpy(), lo, rtol=1e-12)


def test_leading_axes_dtype_and_foreign_producer(lib):
    A = _stack(5, 6, 12).reshape(2, 3, 12, 12)
    dA = torch.from_numpy(A).cuda()
    d = dev.det(Foreign(dA))
    assert tuple(d.shape) == (2, 3)
    np.testing.assert_allclose(d.cpu().numpy(), np.linalg.det(A), rtol=1e-11)
    f = dev.inv(dA.float())
    assert f.dtype == torch.float32
    np.testing.assert_allclose(f.cpu().numpy(), np.linalg.inv(A.astype(np.float32).astype(np.float64)),
                               rtol=1e-4, atol=1e-5)


def test_singular_and_check_false(lib):
    A = torch.stack([torch.eye(4, dtype=torch.float64), torch.zeros(4, 4, dtype=torch.float64)]).cuda()
    with pytest.raises(la.LinAlgError, match="Singular matrix"):
        dev.inv(A)
    r, info = dev.solve(A, torch.ones(2, 4, dtype=torch.float64, device="cuda"), check=False)
    assert info.is_cuda and int(info[0]) == 0 and int(info[1]) != 0
    assert float(dev.det(A)[1]) == 0.0
    s, l = dev.slogdet(A)
    assert float(s[1]) == 0.0 and float(l[1]) == -np.inf


def test_matmul_batched_on_device(lib):
    rng = np.random.default_rng(8)
    A = rng.standard_normal((5, 2, 33, 70))
    B = rng.standard_normal((5, 2, 70, 19))
    Cm = dev.matmul_batched(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda())
    assert Cm.is_cuda and tuple(Cm.shape) == (5, 2, 33, 19)
    assert np.all(np.abs(Cm.cpu().numpy() - A @ B) <= 1e-13 * (np.abs(A) @ np.abs(B)))


def test_abi_checks_each_tensor(lib):
    """Host tensors and other float widths are declined; bad shapes / strides are errors."""
    st = torch.cuda.current_stream().cuda_stream
    A = torch.from_numpy(_stack(1, 2, 8)).cuda()
    x = torch.empty(2, 8, 3, dtype=torch.float64, device="cuda")
    b = torch.ones(2, 8, 3, dtype=torch.float64, device="cuda")
    info = torch.zeros(2, dtype=torch.int32, device="cuda")
    W = _lib.WANT_SOLVE

    def call(a, bb, xx, inf=info):
        h = dev._Handoff(st)
        return lib.nppb_dl_linalg(W, h.ptr(a), h.ptr(bb), h.ptr(xx), None, None, None, None, h.ptr(inf), st)

    assert call(A, b, x) == _lib.OK
    torch.cuda.synchronize()
    assert call(A.cpu(), b, x) == _lib.DECLINED
    assert call(A.float(), b, x) == _lib.DECLINED
    assert call(A.transpose(1, 2), b, x) == _lib.E_ARG          # not C-contiguous
    assert "contiguous" in _lib.last_error()
    assert call(A, b[:, :4], x) == _lib.E_ARG                   # wrong order
    assert call(A, b, x[..., :2]) == _lib.E_ARG                 # x does not match b
    assert call(A, b, x, info.to(torch.int64)) == _lib.E_ARG    # info must be int32
    assert call(A[:, :, :7], b, x) == _lib.E_ARG                # not square
    h = dev._Handoff(st)
    assert lib.nppb_dl_linalg(_lib.WANT_LU, h.ptr(A), None, None, None, None, None, None, None, st) == _lib.E_ARG
    assert lib.nppb_dl_matmul(h.ptr(A), h.ptr(b), h.ptr(x), st) == _lib.OK
    torch.cuda.synchronize()
    np.testing.assert_allclose(x.cpu().numpy(), A.cpu().numpy() @ b.cpu().numpy(), rtol=1e-13)
    assert lib.nppb_dl_matmul(h.ptr(A), h.ptr(A), h.ptr(x), st) == _lib.E_ARG


def test_cholesky_on_device(lib, oracle):
    rng = np.random.default_rng(9)
    X = rng.standard_normal((2, 3, 70, 70))
    A = X @ X.transpose(0, 1, 3, 2) / 70 + np.eye(70)
    Lt = dev.cholesky(Foreign(torch.from_numpy(A).cuda()))
    assert Lt.is_cuda and tuple(Lt.shape) == (2, 3, 70, 70)
    Lo, ok = oracle.cholesky(A.reshape(6, 70, 70))
    assert ok.all()
    np.testing.assert_allclose(Lt.cpu().numpy().reshape(6, 70, 70), Lo, rtol=1e-11, atol=1e-13)
    bad = torch.from_numpy(-np.eye(5)[None].repeat(2, 0)).cuda()
    with pytest.raises(la.LinAlgError, match="positive definite"):
        dev.cholesky(bad)
    _, info = dev.cholesky(bad, check=False)
    assert bool((info > 0).all())
