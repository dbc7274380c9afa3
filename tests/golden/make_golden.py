"""Regenerates the golden fixtures in tests/golden from the reference itself.

Runs the reference's OpenMP apps built by oracle/build_ref.sh (oracle/_ref/bin,
this container only: it needs the reference tree to build) and stores their
outputs as small .npz files that travel with the tests. The fixtures pin the
oracle (oracle/src) and the B200 path to the reference's own results.

    python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

# (imax, jmax, iters, seed). The reference app itself fails on degenerate
# grids (1x1 segfaults, 2x1 does not terminate), so those edge cases are
# checked against the oracle only.
LAPLACE_CASES = [
    (37, 23, 25, 11),
    (64, 64, 50, 1),
    (130, 7, 9, 5),
]


def laplace():
    exe = oracle.reference_binary("laplace2d_seeded")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/laplace2d_seeded missing: run oracle/build_ref.sh")
    for imax, jmax, iters, seed in LAPLACE_CASES:
        with tempfile.TemporaryDirectory() as td:
            dump = os.path.join(td, "A.bin")
            r = subprocess.run([exe, str(imax), str(jmax), str(iters), str(seed), dump], cwd=td,
                               capture_output=True, text=True, check=True, timeout=120,
                               env=dict(os.environ, OMP_NUM_THREADS="1"))
            errs = [float(l.split()[3]) for l in r.stdout.splitlines() if l.startswith("iter ")]
            field = np.fromfile(dump, dtype=np.float64).reshape(jmax + 2, imax + 2)
        name = os.path.join(HERE, f"laplace_seeded_{imax}x{jmax}_it{iters}_s{seed}.npz")
        np.savez_compressed(name, field=field, errors=np.array(errs), imax=imax, jmax=jmax, iters=iters,
                            seed=seed)
        print("wrote", name)


if __name__ == "__main__" and len(sys.argv) == 1:
    laplace()


# CloverLeaf decks: (name, x_cells, y_cells, end_step, rectangle seed)
CLOVER_CASES = [
    ("clover_64x64_s30", 64, 64, 30, 2),
    ("clover_100x70_s25", 100, 70, 25, 5),
]
DUMP_FIELDS = ["density0", "density1", "energy0", "energy1", "pressure", "viscosity", "soundspeed", "xvel0",
               "xvel1", "yvel0", "yvel1", "vol_flux_x", "vol_flux_y", "mass_flux_x", "mass_flux_y"]


def run_reference_clover(deck_text, dump=False, threads=1, timeout=600):
    """Runs the reference CloverLeaf build on a deck; returns (summaries, dts, dumps)."""
    exe = oracle.reference_binary("cloverleaf")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/cloverleaf missing: run oracle/build_ref.sh")
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "clover.in"), "w") as f:
            f.write(deck_text)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        if dump:
            env["ORACLE_DUMP_DIR"] = td
        r = subprocess.run([exe], cwd=td, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
        out = open(os.path.join(td, "clover.out")).read()
        summ = []
        for line in out.splitlines():
            if line.strip().startswith("step:"):
                v = line.split()
                summ.append([float(x) for x in v[1:9]])
        dts = [float(l.split()[7]) for l in r.stdout.splitlines() if l.strip().startswith("Step ")]
        dumps = {}
        if dump:
            for name in DUMP_FIELDS:
                meta = open(os.path.join(td, name + ".meta")).read().split("\n")
                size = [int(x) for x in meta[1].split()[1:]]
                xpad = int(meta[4].split()[1])
                a = np.fromfile(os.path.join(td, name + ".bin"), dtype=np.float64).reshape(size[1], size[0])
                dumps[name] = a[:, :size[0] - xpad]
    # columns: step, vol, mass, density, pressure, ie, ke, total
    return np.array(summ), np.array(dts), dumps


def clover():
    from ops_b200 import apps, seeded
    for name, nx, ny, steps, seed in CLOVER_CASES:
        deck = apps.clover_deck(x_cells=nx, y_cells=ny, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0,
                                initial_timestep=0.04, timestep_rise=1.5, max_timestep=0.04, end_step=steps,
                                summary_frequency=1, states=seeded.clover_config2_states(nx, ny, seed))
        text = apps.clover_deck_text(deck)
        summ, dts, dumps = run_reference_clover(text, dump=True)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, deck=text, summaries=summ, dts=dts, **{"f_" + k: v for k, v in dumps.items()})
        print("wrote", path, summ.shape, len(dts))


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "clover":
    clover()


# CloverLeaf 3D decks: (name, x, y, z cells, end_step, cuboid seed,
# max_timestep); uneven extents so that an axis mix-up shows, and a large
# max_timestep in the second so that the CFL limit sets dt
CLOVER3D_CASES = [
    ("clover3d_24x20x16_s40", 24, 20, 16, 40, 6, 0.04),
    ("clover3d_18x14x22_s30", 18, 14, 22, 30, 9, 1.0),
]
DUMP3D_FIELDS = ["density0", "energy0", "pressure", "xvel0", "yvel0", "zvel0"]


def run_reference_clover3d(deck_text, dump=False, threads=1, timeout=600):
    """Runs the reference CloverLeaf 3D build on a deck; returns (summaries, dts, dumps)."""
    exe = oracle.reference_binary("cloverleaf3d")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/cloverleaf3d missing: run oracle/build_ref.sh")
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "clover.in"), "w") as f:
            f.write(deck_text)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        if dump:
            env["ORACLE_DUMP_DIR"] = td
        r = subprocess.run([exe], cwd=td, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
        out = open(os.path.join(td, "clover.out")).read()
        summ = [[float(x) for x in l.split()[1:9]] for l in out.splitlines() if l.strip().startswith("step:")]
        dts = [float(l.split()[7]) for l in r.stdout.splitlines() if l.strip().startswith("Step ")]
        dumps = {}
        if dump:
            for name in DUMP3D_FIELDS:
                meta = open(os.path.join(td, name + ".meta")).read().split("\n")
                size = [int(x) for x in meta[1].split()[1:]]
                xpad = int(meta[4].split()[1])
                a = np.fromfile(os.path.join(td, name + ".bin"), dtype=np.float64).reshape(size[2], size[1], size[0])
                dumps[name] = a[:, :, :size[0] - xpad]
    # columns: step, vol, mass, density, pressure, ie, ke, total
    return np.array(summ), np.array(dts), dumps


def clover3d():
    from ops_b200 import apps, seeded
    for name, nx, ny, nz, steps, seed, max_dt in CLOVER3D_CASES:
        deck = apps.clover3d_deck(x_cells=nx, y_cells=ny, z_cells=nz, xmax=10.0, ymax=10.0, zmax=10.0,
                                  initial_timestep=0.04, timestep_rise=1.5, max_timestep=max_dt, end_step=steps,
                                  summary_frequency=1, states=seeded.clover3d_states(nx, ny, nz, seed))
        text = apps.clover3d_deck_text(deck)
        summ, dts, dumps = run_reference_clover3d(text, dump=True)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, deck=text, summaries=summ, dts=dts, **{"f_" + k: v for k, v in dumps.items()})
        print("wrote", path, summ.shape, len(dts), os.path.getsize(path))


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "clover3d":
    clover3d()


# TeaLeaf decks: (name, deck keywords)
TEA_CASES = [
    ("tea_kat_jacobi", dict(x_cells=10, y_cells=10, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=10,
                            max_iters=1000, eps=1e-15, solver=0, summary_frequency=10,
                            states="tea.in")),
    ("tea_cg_jacdiag_64", dict(x_cells=64, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=2,
                               max_iters=5000, eps=1e-10, solver=1, preconditioner=1, summary_frequency=1,
                               states=("seeded", 64, 64, 4))),
    ("tea_cg_plain_100x70", dict(x_cells=100, y_cells=70, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=1,
                                 max_iters=5000, eps=1e-10, solver=1, preconditioner=0, summary_frequency=1,
                                 states=("seeded", 100, 70, 7))),
    # Chebyshev and PPCG after CG presteps (tea_solve.cpp:146-300); dt = 0.04
    # gives condition numbers near 100, so the polynomial phases run for
    # tens to hundreds of iterations, and later timesteps reuse the first
    # solve's eigenvalue estimate
    ("tea_cheby_plain_96", dict(x_cells=96, y_cells=96, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=3,
                                max_iters=5000, eps=1e-10, solver=2, preconditioner=0, summary_frequency=1,
                                states=("seeded", 96, 96, 4))),
    ("tea_cheby_jacdiag_80x64", dict(x_cells=80, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.04,
                                     end_step=2, max_iters=5000, eps=1e-10, solver=2, preconditioner=1,
                                     summary_frequency=1, states=("seeded", 80, 64, 11))),
    ("tea_ppcg_plain_96", dict(x_cells=96, y_cells=96, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=3,
                               max_iters=5000, eps=1e-10, solver=3, preconditioner=0, summary_frequency=1,
                               states=("seeded", 96, 96, 4))),
    ("tea_ppcg_jacdiag_64", dict(x_cells=64, y_cells=64, xmax=10.0, ymax=10.0, initial_timestep=0.04, end_step=2,
                                 max_iters=5000, eps=1e-10, solver=3, preconditioner=1, summary_frequency=1,
                                 ch_cg_presteps=10, ch_cg_epslim=0.5, ppcg_inner_steps=12,
                                 states=("seeded", 64, 64, 5))),
]
TEA_DUMP = ["u", "energy1", "density"]


def tea_states(spec):
    from ops_b200 import seeded
    if spec == "tea.in":  # apps/c/TeaLeaf/tea.in
        return [dict(density=100.0, energy=0.0001),
                dict(density=0.1, energy=25.0, geometry="rectangle", xmin=0.0, xmax=1.0, ymin=1.0, ymax=2.0),
                dict(density=0.1, energy=0.1, geometry="rectangle", xmin=1.0, xmax=6.0, ymin=1.0, ymax=2.0),
                dict(density=0.1, energy=0.1, geometry="rectangle", xmin=5.0, xmax=6.0, ymin=1.0, ymax=8.0),
                dict(density=0.1, energy=0.1, geometry="rectangle", xmin=5.0, xmax=10.0, ymin=7.0, ymax=8.0)]
    _, nx, ny, seed = spec
    return seeded.tea_config4_states(nx, ny, seed)


def run_reference_tea(deck_text, dump=False, threads=1, timeout=900):
    exe = oracle.reference_binary("tealeaf")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/tealeaf missing: run oracle/build_ref.sh")
    with tempfile.TemporaryDirectory() as td:
        with open(os.path.join(td, "tea.in"), "w") as f:
            f.write(deck_text)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        if dump:
            env["ORACLE_DUMP_DIR"] = td
        r = subprocess.run([exe], cwd=td, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0:
            raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
        out = open(os.path.join(td, "tea.out")).read()
        summ = [[float(x) for x in l.split()[1:7]] for l in out.splitlines() if l.strip().startswith("step:")]
        iters = [int(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Iteration count")]
        errs = [float(l.split()[-1]) for l in r.stdout.splitlines() if l.strip().startswith("Conduction error")]
        # Chebyshev / PPCG lines (tea_solve.cpp:228-231, tea_leaf_cheby.cpp:312-313, tea_solve.cpp:389-392)
        lines = r.stdout.splitlines()
        poly = dict(
            switch=[int(l.split()[2]) for l in lines if l.startswith("Switching after")],
            eig=[[float(l.split()[2]), float(l.split()[5])] for l in lines if l.startswith("Eigen min")],
            est_itc=[int(lines[i + 1]) for i, l in enumerate(lines) if l.strip() == "est itc"],
            ppcg=[int(l.split()[3]) for l in lines if l.startswith("PPCG Iteration count")])
        dumps = {}
        if dump:
            # the reference pads TeaLeaf dat names with blanks (build_field.cpp:55-73)
            files = {f[:-5].strip(): f[:-5] for f in os.listdir(td) if f.endswith(".meta")}
            for name in TEA_DUMP:
                fn = files[name]
                meta = open(os.path.join(td, fn + ".meta")).read().split("\n")
                size = [int(x) for x in meta[1].split()[1:]]
                xpad = int(meta[4].split()[1])
                a = np.fromfile(os.path.join(td, fn + ".bin"), dtype=np.float64).reshape(size[1], size[0])
                dumps[name] = a[:, :size[0] - xpad]
    # summary columns: step, vol, mass, density, ie, temp
    return np.array(summ), np.array(iters), np.array(errs), dumps, {k: np.array(v) for k, v in poly.items()}


def tea():
    from ops_b200 import apps
    for name, kw in TEA_CASES:
        kw = dict(kw)
        kw["states"] = tea_states(kw["states"])
        deck = apps.tea_deck(**kw)
        text = apps.tea_deck_text(deck)
        summ, iters, errs, dumps, poly = run_reference_tea(text, dump=True)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, deck=text, summaries=summ, iters=iters, errors=errs,
                            **{"f_" + k: v for k, v in dumps.items()}, **{"poly_" + k: v for k, v in poly.items()})
        print("wrote", path, summ.shape, iters, errs)


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "tea":
    tea()


# ---------------------------------------------------------------------------
# halo transfer cases from the reference library (oracle/ref_drivers/halo_cases.cpp)
# ---------------------------------------------------------------------------
def halo():
    exe = oracle.reference_binary("halo_cases")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/halo_cases missing: run oracle/build_ref.sh")
    out = {}
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([exe, td], check=True, capture_output=True, timeout=300)
        for c in range(6):
            for name, dt in (("a", np.float64), ("b", np.float64), ("bf", np.float32)):
                raw = open(os.path.join(td, f"case{c}_{name}.bin"), "rb").read()
                nx, ny = np.frombuffer(raw[:8], dtype=np.int32)
                out[f"case{c}_{name}"] = np.frombuffer(raw[8:], dtype=dt).reshape(ny, nx).copy()
    path = os.path.join(HERE, "halo_cases.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out))


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "halo":
    halo()


# ---------------------------------------------------------------------------
# Full-size configurations: the headline decks at their stated sizes. The
# fixtures hold every per-step scalar the reference prints (dt, field
# summaries, max|delta|, iteration counts) and a SHA-256 digest of each final
# field (the reference's host layout without its x padding, which is also the
# layout of ops_b200's dumps), so a GPU test checks the full-size fields bit
# for bit without carrying gigabytes of fixtures.
#
#     python tests/golden/make_golden.py fullsize
# ---------------------------------------------------------------------------
FULL_CLOVER = ("fullsize_clover_3840_s200", 3840, 200, 2)
FULL_TEA = ("fullsize_tea_4096_pcg", 4096, 4)
FULL_LAPLACE = ("fullsize_laplace_4096_it1000", 4096, 1000, 1)


def sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def fullsize_clover(threads):
    from ops_b200 import apps, seeded
    name, n, steps, seed = FULL_CLOVER
    deck = apps.clover_deck(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.04,
                            timestep_rise=1.5, max_timestep=0.04, end_step=steps, summary_frequency=1,
                            states=seeded.clover_config2_states(n, n, seed))
    text = apps.clover_deck_text(deck)
    summ, dts, dumps = run_reference_clover(text, dump=True, threads=threads, timeout=7200)
    digests = {k: sha256(v) for k, v in dumps.items()}
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, deck=text, summaries=summ, dts=dts, field_names=np.array(sorted(digests)),
                        field_sha256=np.array([digests[k] for k in sorted(digests)]),
                        field_shapes=np.array([dumps[k].shape for k in sorted(digests)]))
    print("wrote", path, summ.shape, len(dts))


def fullsize_tea(threads):
    from ops_b200 import apps
    name, n, seed = FULL_TEA
    kw = dict(x_cells=n, y_cells=n, xmin=0.0, ymin=0.0, xmax=10.0, ymax=10.0, initial_timestep=0.004, end_step=1,
              summary_frequency=1, max_iters=200000, eps=1e-10, solver=1, preconditioner=1,
              states=("seeded", n, n, seed))
    kw["states"] = tea_states(kw["states"])
    text = apps.tea_deck_text(apps.tea_deck(**kw))
    summ, iters, errs, _, _ = run_reference_tea(text, dump=False, threads=threads, timeout=7200)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, deck=text, summaries=summ, iters=iters, errors=errs)
    print("wrote", path, summ, iters, errs)


def fullsize_laplace(threads):
    exe = oracle.reference_binary("laplace2d_seeded")
    if exe is None:
        raise SystemExit("oracle/_ref/bin/laplace2d_seeded missing: run oracle/build_ref.sh")
    name, n, iters, seed = FULL_LAPLACE
    with tempfile.TemporaryDirectory() as td:
        dump = os.path.join(td, "A.bin")
        r = subprocess.run([exe, str(n), str(n), str(iters), str(seed), dump], cwd=td, capture_output=True,
                           text=True, check=True, timeout=7200, env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        errs = [float(l.split()[3]) for l in r.stdout.splitlines() if l.startswith("iter ")]
        field = np.fromfile(dump, dtype=np.float64).reshape(n + 2, n + 2)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, errors=np.array(errs), field_sha256=sha256(field), field_sum=float(field.sum()),
                        imax=n, jmax=n, iters=iters, seed=seed)
    print("wrote", path, len(errs))


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "fullsize":
    nthreads = os.cpu_count() or 1
    which = sys.argv[2:] or ["laplace", "clover", "tea"]
    for w in which:
        {"laplace": fullsize_laplace, "clover": fullsize_clover, "tea": fullsize_tea}[w](nthreads)
