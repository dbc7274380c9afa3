"""The 3D 7-point heat operator's FP64 Jacobi-PCG (ops_b200_heat_solve3d)
against numpy: the operator through the initial residual ||u0 - A u||, the
solution against a sparse direct solve, and the iteration count against a
numpy restatement of the same preconditioned CG with TeaLeaf's stopping rule
(the sums differ in order, so the count may differ by one at the threshold)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def apply3d(Kx, Ky, Kz, u, rx, ry, rz):
    """A u on the interior of padded (nz + 2, ny + 2, nx + 2) arrays."""
    c = (slice(1, -1),) * 3
    kx0, kx1 = Kx[c], Kx[1:-1, 1:-1, 2:]
    ky0, ky1 = Ky[c], Ky[1:-1, 2:, 1:-1]
    kz0, kz1 = Kz[c], Kz[2:, 1:-1, 1:-1]
    out = np.zeros_like(u)
    out[c] = ((1.0 + rz * (kz1 + kz0) + ry * (ky1 + ky0) + rx * (kx1 + kx0)) * u[c]
              - rz * (kz1 * u[2:, 1:-1, 1:-1] + kz0 * u[:-2, 1:-1, 1:-1])
              - ry * (ky1 * u[1:-1, 2:, 1:-1] + ky0 * u[1:-1, :-2, 1:-1])
              - rx * (kx1 * u[1:-1, 1:-1, 2:] + kx0 * u[1:-1, 1:-1, :-2]))
    return out


def pcg_numpy(Kx, Ky, Kz, u0, rx, ry, rz, eps):
    """Jacobi-PCG from u = u0 with TeaLeaf's stop sqrt|r.z| < eps ||r0||;
    returns (u, iterations as TeaLeaf reports them)."""
    c = (slice(1, -1),) * 3
    d = np.zeros_like(u0)
    d[c] = 1.0 + rz * (Kz[2:, 1:-1, 1:-1] + Kz[c]) + ry * (Ky[1:-1, 2:, 1:-1] + Ky[c]) + \
        rx * (Kx[1:-1, 1:-1, 2:] + Kx[c])
    Mi = np.zeros_like(u0)
    Mi[c] = 1.0 / d[c]
    u = u0.copy()
    r = u0 - apply3d(Kx, Ky, Kz, u, rx, ry, rz)
    r[~np.pad(np.ones(tuple(s - 2 for s in u0.shape), bool), 1)] = 0.0
    stop = eps * np.sqrt(np.sum(r * r))
    z = Mi * r
    p = z.copy()
    rro = np.sum(r * z)
    for it in range(1, 100000):
        w = apply3d(Kx, Ky, Kz, p, rx, ry, rz)
        alpha = rro / np.sum(p * w)
        u += alpha * p
        r -= alpha * w
        z = Mi * r
        rrn = np.sum(r * z)
        beta = rrn / rro
        rro = rrn
        if np.sqrt(abs(rrn)) < stop:
            return u, it - 1
        p = beta * p + z
    raise AssertionError("numpy PCG did not converge")


def problem(nx, ny, nz, seed):
    from ops_b200 import lmg
    rng = np.random.default_rng(seed)
    rho = np.exp(rng.uniform(np.log(0.1), np.log(100.0), (nz, ny, nx)))
    Kx, Ky, Kz = lmg.faces3d(rho)
    u0 = np.zeros((nz + 2, ny + 2, nx + 2))
    u0[1:-1, 1:-1, 1:-1] = rng.uniform(0.0, 1.0, (nz, ny, nx)) * rho
    return Kx, Ky, Kz, u0


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", [(24, 20, 16), (1, 7, 5), (33, 1, 2)])
def test_operator_matches_numpy(gpu_runtime, shape):
    from ops_b200 import lmg
    nx, ny, nz = shape
    Kx, Ky, Kz, u0 = problem(nx, ny, nz, 11)
    rng = np.random.default_rng(12)
    u = np.zeros_like(u0)
    u[1:-1, 1:-1, 1:-1] = rng.standard_normal((nz, ny, nx))
    rx, ry, rz = 3.0, 5.0, 7.0
    st = lmg.solve3d(cuda(Kx), cuda(Ky), cuda(Kz), cuda(u0), cuda(u), rx, ry, rz, method=lmg.PCG, max_iters=0)
    ref = u0 - apply3d(Kx, Ky, Kz, u, rx, ry, rz)
    ref = np.sqrt(np.sum(ref[1:-1, 1:-1, 1:-1] ** 2))
    assert abs(st["initial_residual"] - ref) <= 1e-12 * ref


@pytest.mark.parametrize("shape,rxyz", [((24, 20, 16), (10.0, 10.0, 10.0)), ((17, 9, 31), (4.0, 30.0, 2.0))])
def test_pcg_matches_numpy(gpu_runtime, shape, rxyz):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    from ops_b200 import lmg
    nx, ny, nz = shape
    rx, ry, rz = rxyz
    Kx, Ky, Kz, u0 = problem(nx, ny, nz, 21)
    # the TeaLeaf stopping rule: iteration count against the numpy restatement
    u = cuda(u0)
    st = lmg.solve3d(cuda(Kx), cuda(Ky), cuda(Kz), cuda(u0), u, rx, ry, rz, method=lmg.PCG, eps=1e-10)
    un, itn = pcg_numpy(Kx, Ky, Kz, u0, rx, ry, rz, 1e-10)
    assert st["converged"]
    assert abs(st["iterations"] - itn) <= 1, (st["iterations"], itn)
    # the true-residual rule: ||u0 - A u|| < 1e-10 ||r0||, and the sparse direct solution
    u2 = cuda(u0)
    st2 = lmg.solve3d(cuda(Kx), cuda(Ky), cuda(Kz), cuda(u0), u2, rx, ry, rz, method=lmg.PCG_TRUE, eps=1e-10)
    assert st2["converged"] and st2["final_residual"] < 1.5e-10 * st2["initial_residual"]
    n = nx * ny * nz
    cols = []
    for k in range(n):
        e = np.zeros_like(u0)
        idx = np.unravel_index(k, (nz, ny, nx))
        e[idx[0] + 1, idx[1] + 1, idx[2] + 1] = 1.0
        cols.append(sp.csc_matrix(apply3d(Kx, Ky, Kz, e, rx, ry, rz)[1:-1, 1:-1, 1:-1].reshape(-1, 1)))
    A = sp.hstack(cols).tocsc()
    exact = spla.spsolve(A, u0[1:-1, 1:-1, 1:-1].reshape(-1))
    got = u2.cpu().numpy()[1:-1, 1:-1, 1:-1].reshape(-1)
    assert np.linalg.norm(got - exact) <= 1e-8 * np.linalg.norm(exact)
    # the restatement stops on TeaLeaf's weaker sqrt|r.z| rule: a looser bound
    assert np.linalg.norm(un[1:-1, 1:-1, 1:-1].reshape(-1) - exact) <= 1e-6 * np.linalg.norm(exact)


@pytest.mark.parametrize("shape", [(24, 20, 16), (40, 8, 3)])
def test_mixed_precision_reaches_the_fp64_residual(gpu_runtime, shape):
    """FP32 inner PCG under FP64 reliable updates: the FP64 residual reaches
    1e-10 and the solution agrees with the FP64 PCG solution."""
    from ops_b200 import lmg
    nx, ny, nz = shape
    Kx, Ky, Kz, u0 = problem(nx, ny, nz, 31)
    k = [cuda(a) for a in (Kx, Ky, Kz, u0)]
    u64, u32 = cuda(u0), cuda(u0)
    s64 = lmg.solve3d(*k, u64, 10.0, 10.0, 10.0, method=lmg.PCG_TRUE, eps=1e-10)
    s32 = lmg.solve3d(*k, u32, 10.0, 10.0, 10.0, method=lmg.MIXED, eps=1e-10)
    assert s64["converged"] and s32["converged"] and s32["updates"] >= 1
    assert s32["final_residual"] < 1e-10 * s32["initial_residual"]
    a, b = u64.cpu().numpy(), u32.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(a)
    assert s32["iterations"] <= 1.3 * s64["iterations"] + 10


def test_bad_shapes_are_refused(gpu_runtime):
    import ctypes

    from ops_b200 import lmg
    from ops_b200._lib import HeatStats, HeatSystem3D, lib
    Kx, Ky, Kz, u0 = problem(4, 4, 4, 1)
    t = [cuda(a) for a in (Kx, Ky, Kz, u0, u0)]
    ptr = [ctypes.c_void_p(x.data_ptr()) for x in t]
    st = HeatStats()
    bad = HeatSystem3D(4, 4, 4, 6, 35, *ptr, 1.0, 1.0, 1.0)  # plane != pitch * (ny + 2)
    assert lib().ops_b200_heat_solve3d(ctypes.byref(bad), lmg.PCG, 1e-10, 10, ctypes.byref(st), None) < 0
    ok = HeatSystem3D(4, 4, 4, 6, 36, *ptr, 1.0, 1.0, 1.0)
    assert lib().ops_b200_heat_solve3d(ctypes.byref(ok), 3, 1e-10, 10, ctypes.byref(st), None) < 0  # method (0-2)
