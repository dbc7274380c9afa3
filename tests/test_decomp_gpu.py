"""Blocks partitioned across processes, on the GPU: each test runs ranks as
separate processes (gloo process group on 127.0.0.1, the host transport of
ops_b200.dist) that share GPU 0. Their halo exchanges go through host memory
and complete before either process launches the loops that read them, so no
kernel waits on another process.

The bar is the single-rank result the reference's own build produced:
* CloverLeaf 2D 64^2, 30 steps (tests/golden/clover_64x64_s30.npz), split in 2
  and 3 slabs along y: dt of every step exactly (min reductions combine
  exactly), field summaries to 1e-12 relative (the ranks' partial sums are
  added in rank order, another order than one GPU's), and every field,
  reassembled from the ranks' owned parts, bit for bit.
* Laplace 2D (the oracle, bit for bit): every iteration's max |delta| and the
  final field.
* CloverLeaf 3D 24x20x16, 40 steps, split in 2 slabs along z: the same bars.
* TeaLeaf CG with the diagonal preconditioner (tests/golden/tea_cg_jacdiag_64):
  iteration counts exactly, summaries to 1e-12, density bit for bit and u,
  energy1 to 1e-10 of their maximum (dot products sum in another order).
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
FIELDS = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0", "xvel1",
          "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y"]
pytestmark = pytest.mark.gpu
FIELDS3D = ["density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0"]

RANK_SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r})
import torch.distributed as dist
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:{port}", rank={rank}, world_size={world})
from ops_b200 import apps, seeded
from ops_b200 import dist as D
from ops_b200 import ops as O
D.use_host_transport()
O.ops_init(0, 0)
case, out = {case!r}, {out!r}
res = {{}}
if case == "clover":
    deck = apps.clover_deck(x_cells=64, y_cells=64, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0,
                            initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=30,
                            summary_frequency=1, states=seeded.clover_config2_states(64, 64, 2))
    summ, _ = apps.cloverleaf(deck, dump_dir=out)
    np.save(out + "/summaries.npy", summ)
elif case == "clover3d":
    deck = apps.clover3d_deck(x_cells=24, y_cells=20, z_cells=16, xmax=10.0, ymax=10.0, zmax=10.0,
                              initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=40,
                              summary_frequency=1, states=seeded.clover3d_states(24, 20, 16, 6))
    summ, _ = apps.cloverleaf3d(deck, dump_dir=out)
    np.save(out + "/summaries.npy", summ)
elif case == "laplace":
    init = seeded.laplace_field(96, 64, 7)
    A, errs, _ = apps.laplace2d(init, 25)
    np.save(out + "/A.npy", A)
    np.save(out + "/errs.npy", errs)
elif case == "tea":
    deck = apps.tea_deck(x_cells=64, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=2,
                         max_iters=5000, eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
                         states=seeded.tea_config4_states(64, 64, 4))
    summ, solves, _ = apps.tealeaf(deck, dump_dir=out)
    np.save(out + "/summaries.npy", summ)
    np.save(out + "/solves.npy", solves)
res["rank_info"] = D.rank_info()
dist.barrier()
dist.destroy_process_group()
print("RESULT " + json.dumps(res))
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(case, world, tmp_path, timeout=600):
    port = free_port()
    procs, dirs = [], []
    for r in range(world):
        d = tmp_path / f"rank{r}"
        d.mkdir()
        dirs.append(str(d))
        code = RANK_SCRIPT.format(root=ROOT, port=port, rank=r, world=world, case=case, out=str(d))
        procs.append(subprocess.Popen([sys.executable, "-c", code], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    infos = []
    for p in procs:
        o, e = p.communicate(timeout=timeout)
        assert p.returncode == 0, o[-2000:] + e[-4000:]
        infos.append(json.loads([l for l in o.splitlines() if l.startswith("RESULT ")][-1][len("RESULT "):]))
    for r, info in enumerate(infos):
        rank, nranks, exchanges = info["rank_info"]
        assert (rank, nranks) == (r, world)
        assert exchanges > 0, "no halo exchange was made"
    return dirs


def reassemble(dirs, name, shape):
    """A dat's whole extent from the ranks' owned parts (slabs along the
    outermost dimension, in rank order)."""
    parts = [np.fromfile(os.path.join(d, name + ".bin")) for d in dirs]
    full = np.concatenate([p.reshape((-1,) + tuple(shape[1:])) for p in parts], axis=0)
    assert full.shape == shape, (name, full.shape, shape)
    return full


def reference_columns(s):
    return np.stack([s[:, 0], s[:, 2], s[:, 3], s[:, 3] / s[:, 2], s[:, 6] / s[:, 2], s[:, 4], s[:, 5],
                     s[:, 4] + s[:, 5]], axis=1)


@pytest.mark.timeout(900)
@pytest.mark.parametrize("world", [2, 3])
def test_cloverleaf_split_matches_single_rank_golden(world, tmp_path):
    g = np.load(os.path.join(GOLDEN, "clover_64x64_s30.npz"))
    dirs = run_ranks("clover", world, tmp_path)
    summs = [np.load(os.path.join(d, "summaries.npy")) for d in dirs]
    for s in summs[1:]:
        assert np.array_equal(s, summs[0]), "ranks disagree on the combined reductions"
    summ = summs[0]
    ref = g["summaries"]
    ours = reference_columns(summ)
    assert ours.shape == ref.shape
    assert np.array_equal(ours[:, 0], ref[:, 0])
    np.testing.assert_allclose(ours[:, 1:], ref[:, 1:], rtol=1e-12, atol=0)
    assert np.array_equal(summ[1:31, 7], g["dts"])
    for f in FIELDS:
        ext = g["f_" + f]
        assert np.array_equal(reassemble(dirs, f, ext.shape), ext), f


@pytest.mark.timeout(900)
def test_cloverleaf3d_split_matches_single_rank_golden(tmp_path):
    """CloverLeaf 3D 24x20x16, 40 steps (tests/golden/clover3d_24x20x16_s40.npz),
    split in 2 slabs along z (whole xy planes per message)."""
    g = np.load(os.path.join(GOLDEN, "clover3d_24x20x16_s40.npz"))
    dirs = run_ranks("clover3d", 2, tmp_path)
    summ = np.load(os.path.join(dirs[0], "summaries.npy"))
    assert np.array_equal(summ, np.load(os.path.join(dirs[1], "summaries.npy")))
    ours = reference_columns(summ)
    assert ours.shape == g["summaries"].shape
    np.testing.assert_allclose(ours[:, 1:], g["summaries"][:, 1:], rtol=1e-12, atol=0)
    assert np.array_equal(summ[1:41, 7], g["dts"])
    for f in FIELDS3D:
        ext = g["f_" + f]
        assert np.array_equal(reassemble(dirs, f, ext.shape), ext), f


@pytest.mark.timeout(600)
def test_laplace_split_matches_oracle(tmp_path):
    import oracle
    from ops_b200 import dist as D
    from ops_b200 import seeded
    dirs = run_ranks("laplace", 2, tmp_path)
    init = seeded.laplace_field(96, 64, 7)
    ref = np.ascontiguousarray(init.copy())
    eo = np.zeros(25)
    oracle.lib().oracle_laplace_run(96, 64, 25, ref.ctypes.data, eo.ctypes.data)
    full = np.empty_like(ref)
    for r, d in enumerate(dirs):
        w = D.slab_window(64, 2, r, 1, -1, 65)
        lo, hi = w["own"]
        A = np.load(os.path.join(d, "A.npy"))
        full[lo + 1:hi + 1] = A[lo + 1:hi + 1]
        assert np.array_equal(np.load(os.path.join(d, "errs.npy")), eo)
    assert np.array_equal(full, ref)


@pytest.mark.timeout(900)
def test_tealeaf_cg_split_matches_single_rank_golden(tmp_path):
    g = np.load(os.path.join(GOLDEN, "tea_cg_jacdiag_64.npz"))
    dirs = run_ranks("tea", 2, tmp_path)
    summ = np.load(os.path.join(dirs[0], "summaries.npy"))
    solves = np.load(os.path.join(dirs[0], "solves.npy"))
    assert np.array_equal(solves[:, 0].astype(np.int64), g["iters"])
    ours = np.stack([summ[:, 0], summ[:, 2], summ[:, 3], summ[:, 3] / summ[:, 2], summ[:, 4], summ[:, 5]], axis=1)
    np.testing.assert_allclose(ours[:, 1:], g["summaries"][:, 1:], rtol=1e-12, atol=0)
    for f in ("density", "energy1", "u"):
        ext = g["f_" + f]
        got = reassemble(dirs, f, ext.shape)
        if f == "density":
            assert np.array_equal(got, ext), f
        else:
            np.testing.assert_allclose(got, ext, rtol=0, atol=1e-10 * np.abs(ext).max(), err_msg=f)
