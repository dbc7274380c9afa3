"""Learned multigrid preconditioner for the TeaLeaf heat solve (no reference
counterpart; the reference's solvers are Jacobi, CG, Chebyshev and PPCG).

Pipeline, all arithmetic on the GPU through the library's C-ABI:
  1. seeded coefficient fields (16 density rectangles, rho log-uniform in
     [0.1, 100] over rho = 1; TeaLeaf's CONDUCTIVITY face coefficients),
  2. residual/error pairs from Jacobi-PCG: a converged FP64 solve gives u*,
     truncated solves from the same start give u_k, r_k = u0 - A u_k and
     e_k = u* - u_k,
  3. training of the network (tcgen05 forward and input-gradient
     convolutions, CUDA-core weight gradients, Adam) on the A-norm error
     ||M(r) - e||_A / ||e||_A, then rounds of on-policy pairs taken along the
     learned FCG's own iterates and retraining (a network trained only on
     PCG residuals stalls FCG once the residuals leave that distribution),
  4. flexible CG with the trained network as preconditioner, falling back to
     Jacobi-PCG when the network stops helping.
FCG_MG runs the same flexible CG with the library's native (non-learned)
aggregation-multigrid V-cycle as preconditioner, the baseline the learned one
is measured against; `mg_apply` applies that V-cycle once. FCG_LEARNED_MG
puts the two together: M(r) = V-cycle(r) + s y, the network trained (`fit`
with base="mg") on the error the V-cycle leaves, e - V-cycle(r).
Device buffers are torch CUDA tensors (allocation only)."""
import ctypes

import numpy as np

from . import seeded
from ._lib import HeatBatch, HeatStats, HeatSystem, HeatSystem3D, check, lib

PCG, PCG_TRUE, MIXED, FCG_LEARNED, FCG_JACOBI, FCG_MG, FCG_LEARNED_MG = 0, 1, 2, 3, 4, 5, 6


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def density_field(n, seed, nrect=16):
    """Cell densities and energies of the seeded heat problem on an n x n grid
    over [0, 10]^2 (cell centres inside a rectangle take its state)."""
    st = seeded.tea_config4_states(n, n, seed, n=nrect)
    rho = np.full((n, n), st[0]["density"])
    en = np.full((n, n), st[0]["energy"])
    xc = (np.arange(n) + 0.5) * (10.0 / n)
    for s in st[1:]:
        mx = (xc >= s["xmin"]) & (xc < s["xmax"])
        my = (xc >= s["ymin"]) & (xc < s["ymax"])
        m = my[:, None] & mx[None, :]
        rho[m] = s["density"]
        en[m] = s["energy"]
    return rho, en


def padded_problem(rho, en):
    """Kx, Ky (tea_leaf_common_init_Kx_Ky_kernel with CONDUCTIVITY: face value
    (w- + w) / (2 w- w), zero on the domain boundary) and u0 = energy * density,
    as (ny + 2) x (nx + 2) arrays with a one-cell ring."""
    ny, nx = rho.shape
    Kx = np.zeros((ny + 2, nx + 2))
    Ky = np.zeros((ny + 2, nx + 2))
    w = rho
    Kx[1:-1, 2:-1] = (w[:, :-1] + w[:, 1:]) / (2.0 * w[:, :-1] * w[:, 1:])
    Ky[2:-1, 1:-1] = (w[:-1, :] + w[1:, :]) / (2.0 * w[:-1, :] * w[1:, :])
    u0 = np.zeros((ny + 2, nx + 2))
    u0[1:-1, 1:-1] = en * rho
    return Kx, Ky, u0


def interior(t, pitch):
    """Pointer to the first interior cell of a padded field tensor."""
    return ctypes.c_void_p(t.data_ptr() + (pitch + 1) * t.element_size())


def solve(Kx, Ky, u0, u, rx, ry, method=PCG_TRUE, net=-1, eps=1e-10, max_iters=100000, window=40, r_out=None,
          stream=None):
    """Heat solve on padded (ny + 2, nx + 2) FP64 CUDA tensors; u is updated.
    Returns the solve statistics as a dict."""
    ny, nx = Kx.shape[0] - 2, Kx.shape[1] - 2
    pitch = nx + 2
    sysd = HeatSystem(nx, ny, pitch, interior(Kx, pitch), interior(Ky, pitch), interior(u0, pitch),
                      interior(u, pitch), rx, ry)
    st = HeatStats()
    check(lib().ops_b200_heat_solve(ctypes.byref(sysd), method, net, eps, max_iters, window,
                                    None if r_out is None else interior(r_out, pitch), ctypes.byref(st),
                                    None if stream is None else ctypes.c_void_p(stream)))
    return {k: getattr(st, k) for k, _ in HeatStats._fields_}


def solve3d(Kx, Ky, Kz, u0, u, rx, ry, rz, method=PCG_TRUE, eps=1e-10, max_iters=100000, stream=None):
    """3D 7-point heat solve (FP64 Jacobi-PCG) on padded (nz + 2, ny + 2,
    nx + 2) FP64 CUDA tensors; u is updated. Returns the solve statistics."""
    import torch
    nz, ny, nx = Kx.shape[0] - 2, Kx.shape[1] - 2, Kx.shape[2] - 2
    for t in (Kx, Ky, Kz, u0, u):
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and tuple(t.shape) == tuple(Kx.shape)
    pitch, plane = nx + 2, (nx + 2) * (ny + 2)

    def first(t):
        return ctypes.c_void_p(t.data_ptr() + 8 * (plane + pitch + 1))

    sysd = HeatSystem3D(nx, ny, nz, pitch, plane, first(Kx), first(Ky), first(Kz), first(u0), first(u), rx, ry, rz)
    st = HeatStats()
    check(lib().ops_b200_heat_solve3d(ctypes.byref(sysd), method, eps, max_iters, ctypes.byref(st),
                                      None if stream is None else ctypes.c_void_p(stream)))
    return {k: getattr(st, k) for k, _ in HeatStats._fields_}


def faces3d(rho):
    """Face conductivities of a 3D density field, as padded_problem's in 2D:
    (w- + w) / (2 w- w) on the faces between two interior cells, zero on the
    domain's boundary faces; Kx, Ky, Kz as (nz + 2, ny + 2, nx + 2) arrays."""
    nz, ny, nx = rho.shape
    w = rho
    Kx = np.zeros((nz + 2, ny + 2, nx + 2))
    Ky = np.zeros_like(Kx)
    Kz = np.zeros_like(Kx)
    Kx[1:-1, 1:-1, 2:-1] = (w[:, :, :-1] + w[:, :, 1:]) / (2.0 * w[:, :, :-1] * w[:, :, 1:])
    Ky[1:-1, 2:-1, 1:-1] = (w[:, :-1, :] + w[:, 1:, :]) / (2.0 * w[:, :-1, :] * w[:, 1:, :])
    Kz[2:-1, 1:-1, 1:-1] = (w[:-1, :, :] + w[1:, :, :]) / (2.0 * w[:-1, :, :] * w[1:, :, :])
    return Kx, Ky, Kz


def mg_apply(Kx, Ky, r, z, rx, ry, stream=None):
    """z = M r with the library's native multigrid preconditioner (one V-cycle
    of the hierarchy built from Kx, Ky, rx, ry); padded (ny + 2, nx + 2) FP64
    CUDA tensors. Returns the number of levels."""
    ny, nx = Kx.shape[0] - 2, Kx.shape[1] - 2
    pitch = nx + 2
    sysd = HeatSystem(nx, ny, pitch, interior(Kx, pitch), interior(Ky, pitch), interior(r, pitch),
                      interior(z, pitch), rx, ry)
    levels = ctypes.c_int(0)
    check(lib().ops_b200_heat_mg_apply(ctypes.byref(sysd), interior(r, pitch), interior(z, pitch),
                                       ctypes.byref(levels), None if stream is None else ctypes.c_void_p(stream)))
    return levels.value


class Net:
    """Handle on a learned-preconditioner network held by the library."""

    def __init__(self, seed=5):
        self.h = lib().ops_b200_lmg_create(seed)
        check(self.h)

    def close(self):
        if self.h >= 0:
            lib().ops_b200_lmg_destroy(self.h)
            self.h = -1

    @staticmethod
    def num_params():
        return lib().ops_b200_lmg_num_params()

    def params(self):
        out = np.zeros(self.num_params(), dtype=np.float32)
        check(lib().ops_b200_lmg_get_params(self.h, out.ctypes.data))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        check(lib().ops_b200_lmg_set_params(self.h, p.ctypes.data))

    def grads(self):
        out = np.zeros(self.num_params(), dtype=np.float32)
        check(lib().ops_b200_lmg_get_grads(self.h, out.ctypes.data))
        return out

    @staticmethod
    def _batch(r, Kx, Ky, rx, ry):
        n, hp, wp = r.shape
        return HeatBatch(n, hp - 2, wp - 2, wp, hp * wp, interior(r[0], wp), interior(Kx[0], wp),
                         interior(Ky[0], wp), rx, ry)

    def apply(self, r, Kx, Ky, rx, ry, out):
        """out = M(r) for a batch of padded (n, h + 2, w + 2) FP64 CUDA tensors."""
        b = self._batch(r, Kx, Ky, rx, ry)
        check(lib().ops_b200_lmg_apply(self.h, ctypes.byref(b), interior(out[0], r.shape[2]), None))

    def train_step(self, r, Kx, Ky, e, rx, ry, lr, loss="anorm"):
        """One forward/backward (and Adam step when lr > 0); returns the loss
        ("l2": ||M(r) - e||^2 / ||e||^2, "anorm": the same in the A-norm)."""
        b = self._batch(r, Kx, Ky, rx, ry)
        out = ctypes.c_double(0.0)
        check(lib().ops_b200_lmg_train_step(self.h, ctypes.byref(b), interior(e[0], r.shape[2]),
                                            {"l2": 0, "anorm": 1}[loss], lr, ctypes.byref(out), None))
        return out.value


def generate_pairs(nfields, n, seed0=1000, snaps=(2, 8, 32), rx_range=(100.0, 1000.0), device="cuda"):
    """Residual/error pairs from Jacobi-PCG on `nfields` seeded n x n problems.
    Field i uses seed seed0 + i and rx = ry log-uniform in rx_range (folded
    into the coefficients, so the pairs are for rx = ry = 1). Returns padded
    CUDA tensors r, e, Kx, Ky of shape (nfields * len(snaps), n + 2, n + 2)."""
    import torch
    m = nfields * len(snaps)
    R = torch.zeros((m, n + 2, n + 2), dtype=torch.float64, device=device)
    E = torch.zeros_like(R)
    KX = torch.zeros_like(R)
    KY = torch.zeros_like(R)
    kx = torch.zeros((n + 2, n + 2), dtype=torch.float64, device=device)
    ky, b, u, ustar, r = (torch.zeros_like(kx) for _ in range(5))
    j = 0
    for i in range(nfields):
        rho, en = density_field(n, seed0 + i)
        Kx, Ky, u0 = padded_problem(rho, en)
        rx = float(rx_range[0] * (rx_range[1] / rx_range[0]) ** seeded.u01(seed0 + i, np.array([7], np.uint64))[0])
        kx.copy_(torch.from_numpy(Kx * rx))
        ky.copy_(torch.from_numpy(Ky * rx))
        b.copy_(torch.from_numpy(u0))
        ustar.copy_(b)
        solve(kx, ky, b, ustar, 1.0, 1.0, method=PCG_TRUE, eps=1e-12, max_iters=100000)
        for k in snaps:
            u.copy_(b)
            solve(kx, ky, b, u, 1.0, 1.0, method=PCG, eps=1e-30, max_iters=k, r_out=r)
            R[j].copy_(r)
            E[j].copy_(ustar - u)
            KX[j].copy_(kx)
            KY[j].copy_(ky)
            j += 1
    # the ring of r and e is not part of the pairs
    for t in (R, E):
        t[:, 0, :] = 0
        t[:, -1, :] = 0
        t[:, :, 0] = 0
        t[:, :, -1] = 0
    return R, E, KX, KY


def generate_on_policy(net, nfields, n, seed0, snaps=(2, 4, 8, 16, 32, 64), rx_range=(100.0, 1000.0),
                       device="cuda", method=FCG_LEARNED):
    """Residual/error pairs along the learned FCG's own trajectory: like
    generate_pairs, but u_k comes from k iterations of flexible CG with the
    current network, so the pairs are the residuals the network meets when
    it is used as a preconditioner."""
    import torch
    m = nfields * len(snaps)
    R = torch.zeros((m, n + 2, n + 2), dtype=torch.float64, device=device)
    E, KX, KY = (torch.zeros_like(R) for _ in range(3))
    kx = torch.zeros((n + 2, n + 2), dtype=torch.float64, device=device)
    ky, b, u, ustar, r = (torch.zeros_like(kx) for _ in range(5))
    j = 0
    for i in range(nfields):
        rho, en = density_field(n, seed0 + i)
        Kx, Ky, u0 = padded_problem(rho, en)
        rx = float(rx_range[0] * (rx_range[1] / rx_range[0]) ** seeded.u01(seed0 + i, np.array([7], np.uint64))[0])
        kx.copy_(torch.from_numpy(Kx * rx))
        ky.copy_(torch.from_numpy(Ky * rx))
        b.copy_(torch.from_numpy(u0))
        ustar.copy_(b)
        solve(kx, ky, b, ustar, 1.0, 1.0, method=PCG_TRUE, eps=1e-12, max_iters=100000)
        for k in snaps:
            u.copy_(b)
            solve(kx, ky, b, u, 1.0, 1.0, method=method, net=net.h, eps=1e-30, window=0, max_iters=k, r_out=r)
            R[j].copy_(r)
            E[j].copy_(ustar - u)
            KX[j].copy_(kx)
            KY[j].copy_(ky)
            j += 1
    for t in (R, E):
        t[:, 0, :] = 0
        t[:, -1, :] = 0
        t[:, :, 0] = 0
        t[:, :, -1] = 0
    return R, E, KX, KY


def mg_targets(data):
    """Targets that train the network as a correction to the multigrid
    V-cycle: the network's output is r / D + s y (D = diag(A)), and method
    FCG_LEARNED_MG applies V-cycle(r) + s y, so the pair (r, e) becomes
    (r, e - V-cycle(r) + r / D). Pairs are for rx = ry = 1."""
    import torch
    R, E, KX, KY = data
    E2 = E.clone()
    z = torch.zeros_like(R[0])
    for j in range(R.shape[0]):
        z.zero_()
        mg_apply(KX[j], KY[j], R[j], z, 1.0, 1.0)
        kx, ky = KX[j], KY[j]
        D = 1.0 + kx[1:-1, 1:-1] + kx[1:-1, 2:] + ky[1:-1, 1:-1] + ky[2:, 1:-1]
        E2[j, 1:-1, 1:-1] = E[j, 1:-1, 1:-1] - z[1:-1, 1:-1] + R[j, 1:-1, 1:-1] / D
    return R, E2, KX, KY


def fit(net, n=64, nfields=300, steps=1500, rounds=3, lr=2e-3, batch=16, seed0=1000, log=None, base="jacobi"):
    """The training recipe: PCG pairs, then `rounds` rounds of on-policy pairs
    (half as many fields each, new seeds) added to the set, training after
    each. Returns the loss history of every round. base="mg" trains the
    network as the correction of FCG_LEARNED_MG (targets by mg_targets,
    on-policy pairs along that method's own iterates)."""
    import torch
    retarget = mg_targets if base == "mg" else (lambda d: d)
    method = FCG_LEARNED_MG if base == "mg" else FCG_LEARNED
    data = retarget(generate_pairs(nfields, n, seed0=seed0))
    hists = [train(net, data, steps=steps, batch=batch, lr=lr, seed=0)]
    for rd in range(rounds):
        extra = retarget(generate_on_policy(net, max(1, nfields // 2), n, seed0 + 100000 * (rd + 1), method=method))
        data = tuple(torch.cat([a, b]) for a, b in zip(data, extra))
        hists.append(train(net, data, steps=steps, batch=batch, lr=0.5 * lr, seed=rd + 1))
        if log:
            log(f"round {rd + 1}: {data[0].shape[0]} pairs, loss {np.mean(hists[-1][-50:]):.4f}")
    return hists


def train(net, data, steps=1000, batch=16, lr=1e-3, seed=0, log=None, loss="anorm"):
    """Adam on random batches of the pairs; returns the loss history."""
    import torch
    R, E, KX, KY = data
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    for it in range(steps):
        idx = torch.randint(0, R.shape[0], (batch,), generator=g).to(R.device)
        lr_t = lr * (0.1 if it > 0.8 * steps else 1.0)
        L = net.train_step(R[idx].contiguous(), KX[idx].contiguous(), KY[idx].contiguous(), E[idx].contiguous(),
                           1.0, 1.0, lr_t, loss)
        hist.append(L)
        if log and (it % 100 == 0 or it == steps - 1):
            log(f"step {it} loss {L:.4f}")
    return hist
