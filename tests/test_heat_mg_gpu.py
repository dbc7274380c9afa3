"""Native multigrid preconditioner of the heat solve (method OPS_B200_HEAT_FCG_MG;
no reference counterpart: the reference's TeaLeaf solvers are Jacobi, CG,
Chebyshev and PPCG, and its mgrid app only moves data between levels).

1. One V-cycle z = M r through ops_b200_heat_mg_apply against an FP64 numpy
   statement of the same cycle (written below from the algorithm the header
   documents: 2 x 2 aggregation, coarse mass = sum, coarse faces = half the
   covered fine faces, two damped-Jacobi sweeps with omega 0.8 on each side,
   64 sweeps on the <= 16 x 16 coarsest level). The kernels run the cycle in
   FP32, so the check is relative L2 within 1e-4 (a wrong level, face or
   sweep is off by O(1)).
2. Flexible CG with that preconditioner reaches the FP64 residual 1e-10 on
   the seeded heat problems, on square, odd and degenerate shapes, in a small
   fraction of Jacobi-PCG's iterations, and agrees with the PCG solution.
3. Two solves give bit-identical results (no atomics, fixed sum orders)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OMEGA, FACE_SCALE, COARSEST, SWEEPS, COARSE_SWEEPS = 0.8, 0.5, 16, 2, 64


# ---- FP64 statement of the V-cycle ---------------------------------------
class Level:
    def __init__(self, m, ax, ay):
        self.m, self.ax, self.ay = m, ax, ay       # m (ny, nx); ax (ny, nx+1); ay (ny+1, nx)
        self.ny, self.nx = m.shape
        self.c = m + ax[:, :-1] + ax[:, 1:] + ay[:-1, :] + ay[1:, :]

    def resid(self, r, z):
        s = r - self.c * z
        s[:, 1:] += self.ax[:, 1:-1] * z[:, :-1]
        s[:, :-1] += self.ax[:, 1:-1] * z[:, 1:]
        s[1:, :] += self.ay[1:-1, :] * z[:-1, :]
        s[:-1, :] += self.ay[1:-1, :] * z[1:, :]
        return s


def hierarchy(Kx, Ky, rx, ry):
    ny, nx = Kx.shape[0] - 2, Kx.shape[1] - 2
    levels = [Level(np.ones((ny, nx)), rx * Kx[1:-1, 1:nx + 2], ry * Ky[1:ny + 2, 1:-1])]
    while not (levels[-1].nx <= COARSEST and levels[-1].ny <= COARSEST):
        F = levels[-1]
        cny, cnx = (F.ny + 1) // 2, (F.nx + 1) // 2
        yi, xi = np.arange(F.ny) // 2, np.arange(F.nx) // 2
        m = np.zeros((cny, cnx))
        np.add.at(m, (yi[:, None], xi[None, :]), F.m)
        ax = np.zeros((cny, cnx + 1))
        np.add.at(ax, (yi,), F.ax[:, np.minimum(2 * np.arange(cnx + 1), F.nx)])
        ay = np.zeros((cny + 1, cnx))
        np.add.at(ay, (slice(None), xi), F.ay[np.minimum(2 * np.arange(cny + 1), F.ny), :])
        levels.append(Level(m, FACE_SCALE * ax, FACE_SCALE * ay))
    return levels


def vcycle(levels, r, l=0):
    L = levels[l]
    z = OMEGA * r / L.c
    if l == len(levels) - 1:
        for _ in range(COARSE_SWEEPS - 1):
            z = z + OMEGA * L.resid(r, z) / L.c
        return z
    for _ in range(SWEEPS - 1):
        z = z + OMEGA * L.resid(r, z) / L.c
    s = L.resid(r, z)
    rc = np.zeros(((L.ny + 1) // 2, (L.nx + 1) // 2))
    np.add.at(rc, (np.arange(L.ny)[:, None] // 2, np.arange(L.nx)[None, :] // 2), s)
    e = vcycle(levels, rc, l + 1)
    z = z + e[np.arange(L.ny)[:, None] // 2, np.arange(L.nx)[None, :] // 2]
    for _ in range(SWEEPS):
        z = z + OMEGA * L.resid(r, z) / L.c
    return z


# ---- problems ----------------------------------------------------------------
def random_problem(ny, nx, seed):
    rng = np.random.default_rng(seed)
    Kx = np.zeros((ny + 2, nx + 2))
    Ky = np.zeros((ny + 2, nx + 2))
    Kx[1:-1, 2:-1] = 10.0 ** rng.uniform(-2, 1, (ny, nx - 1))
    Ky[2:-1, 1:-1] = 10.0 ** rng.uniform(-2, 1, (ny - 1, nx))
    r = np.zeros((ny + 2, nx + 2))
    r[1:-1, 1:-1] = rng.standard_normal((ny, nx))
    return Kx, Ky, r


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("ny,nx,rx,seed", [(64, 64, 40.0, 1), (37, 53, 400.0, 2), (9, 13, 5.0, 3),
                                           (1, 1, 2.0, 4), (3, 70, 30.0, 5), (130, 17, 900.0, 6)])
def test_vcycle_matches_fp64_statement(gpu_runtime, ny, nx, rx, seed):
    from ops_b200 import lmg
    Kx, Ky, r = random_problem(ny, nx, seed)
    z = cuda(np.zeros_like(r))
    nlev = lmg.mg_apply(cuda(Kx), cuda(Ky), cuda(r), z, rx, 0.7 * rx)
    levels = hierarchy(Kx, Ky, rx, 0.7 * rx)
    assert nlev == len(levels)
    want = vcycle(levels, r[1:-1, 1:-1])
    got = z.cpu().numpy()
    assert np.all(got[0, :] == 0) and np.all(got[:, 0] == 0)       # the ring is not written
    got = got[1:-1, 1:-1]
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-4


def seeded_problem(n, seed=4):
    from ops_b200 import lmg
    rho, en = lmg.density_field(n, seed)
    return lmg.padded_problem(rho, en)


@pytest.mark.parametrize("n,rx", [(256, 0.004 / (10.0 / 256) ** 2), (128, 400.0), (512, 0.004 / (10.0 / 512) ** 2)])
def test_fcg_mg_converges_in_few_iterations(gpu_runtime, n, rx):
    import torch
    from ops_b200 import lmg
    Kx, Ky, u0 = (cuda(a) for a in seeded_problem(n))
    u_mg = u0.clone()
    st = lmg.solve(Kx, Ky, u0, u_mg, rx, rx, method=lmg.FCG_MG, eps=1e-10, window=40, max_iters=2000)
    u_cg = u0.clone()
    sp = lmg.solve(Kx, Ky, u0, u_cg, rx, rx, method=lmg.PCG_TRUE, eps=1e-12, max_iters=100000)
    assert st["converged"] == 1 and st["fallbacks"] == 0
    assert st["final_residual"] < 1e-10 * st["initial_residual"]
    assert st["iterations"] * 5 < sp["iterations"], (st["iterations"], sp["iterations"])
    assert float(torch.linalg.norm(u_mg - u_cg) / torch.linalg.norm(u_cg)) < 1e-8


@pytest.mark.parametrize("ny,nx", [(1, 1), (1, 40), (33, 1), (17, 16), (100, 37), (65, 129)])
def test_fcg_mg_odd_shapes(gpu_runtime, ny, nx):
    from ops_b200 import lmg
    rng = np.random.default_rng(ny * 1000 + nx)
    Kx, Ky, _ = random_problem(max(ny, 2), max(nx, 2), 7)
    Kx, Ky = Kx[:ny + 2, :nx + 2].copy(), Ky[:ny + 2, :nx + 2].copy()
    Kx[:, nx + 1] = 0.0                      # boundary faces zero, as TeaLeaf's
    Ky[ny + 1, :] = 0.0
    Kx[:, 1] = 0.0
    Ky[1, :] = 0.0
    u0 = np.zeros((ny + 2, nx + 2))
    u0[1:-1, 1:-1] = rng.uniform(0.5, 2.0, (ny, nx))
    k, ky, b = cuda(Kx), cuda(Ky), cuda(u0)
    u = b.clone()
    st = lmg.solve(k, ky, b, u, 50.0, 50.0, method=lmg.FCG_MG, eps=1e-10, window=40, max_iters=500)
    assert st["converged"] == 1
    assert st["final_residual"] <= 1e-10 * st["initial_residual"] or st["final_residual"] < 1e-13


def test_fcg_mg_is_deterministic(gpu_runtime):
    import torch
    from ops_b200 import lmg
    Kx, Ky, u0 = (cuda(a) for a in seeded_problem(192, seed=11))
    outs = []
    for _ in range(2):
        u = u0.clone()
        st = lmg.solve(Kx, Ky, u0, u, 200.0, 200.0, method=lmg.FCG_MG, eps=1e-10, window=40)
        outs.append((u, st["iterations"]))
    assert outs[0][1] == outs[1][1]
    assert torch.equal(outs[0][0], outs[1][0])
