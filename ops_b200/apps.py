"""Reference app drivers restated on the OPS-B200 runtime (C++ drivers in
ops_b200/csrc/apps_*.cpp, reached through the C-ABI)."""
import ctypes

import numpy as np

from ._lib import check, lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def laplace2d(field, iters, warmup=0, return_errors=True, out=None):
    """Laplace Jacobi (apps/c/laplace2d_tutorial/step7/laplace2d.cpp:113-124).

    field: (jmax+2, imax+2) float64 full extent (ring = boundary values).
    out: optional C-contiguous float64 array of the same shape that receives
    the final field (e.g. pinned host memory); a new array otherwise.
    Returns (final_field, errors_per_iteration, device_seconds)."""
    field = np.ascontiguousarray(field, dtype=np.float64)
    jmax, imax = field.shape[0] - 2, field.shape[1] - 2
    if out is None:
        out = np.empty_like(field)
    elif out.shape != field.shape or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
        raise ValueError("out must be a C-contiguous float64 array shaped like field")
    elif not out.flags["WRITEABLE"]:
        raise ValueError("out must be writeable (the final field is written into it)")
    errs = np.empty(max(warmup + iters, 1), dtype=np.float64) if return_errors else None
    secs = ctypes.c_double(0.0)
    check(lib().ops_b200_app_laplace2d(imax, jmax, warmup, iters, _ptr(field), _ptr(out), _ptr(errs),
                                       ctypes.byref(secs)))
    return out, (errs[:warmup + iters] if errs is not None else None), secs.value


# ---------------------------------------------------------------------------
# CloverLeaf
# ---------------------------------------------------------------------------
# read_input.cpp:46-68 defaults, overridden by the deck.
CLOVER_DEFAULTS = dict(x_cells=10, y_cells=10, xmin=0.0, ymin=0.0, xmax=100.0, ymax=100.0, initial_timestep=0.1,
                       timestep_rise=1.5, max_timestep=1.0, end_time=10.0, end_step=640000, summary_frequency=10)
GEOMETRY = {"rectangle": 1, "circle": 2, "point": 3}


def clover_deck(**kw):
    """Build a deck from keyword values; `states` is a list of dicts with
    density, energy and optionally xvel, yvel, geometry, xmin..ymax, radius."""
    from ._lib import CloverDeck
    d = CloverDeck()
    vals = dict(CLOVER_DEFAULTS)
    vals.update({k: v for k, v in kw.items() if k != "states"})
    for k, v in vals.items():
        setattr(d, k, v)
    states = kw["states"]
    d.number_of_states = len(states)
    for i, s in enumerate(states):
        st = d.states[i]
        st.density, st.energy = s["density"], s["energy"]
        st.xvel, st.yvel = s.get("xvel", 0.0), s.get("yvel", 0.0)
        g = s.get("geometry", 0)
        st.geometry = GEOMETRY.get(g, g) if isinstance(g, str) else g
        for k in ("xmin", "xmax", "ymin", "ymax", "radius"):
            setattr(st, k, s.get(k, 0.0))
    return d


def clover_deck_text(deck):
    """The same deck as clover.in text (17 significant digits, so the
    reference's atof reads back identical doubles)."""
    g = lambda v: repr(float(v))
    lines = ["*clover"]
    for i in range(deck.number_of_states):
        s = deck.states[i]
        line = f" state {i + 1} density={g(s.density)} energy={g(s.energy)}"
        if s.xvel != 0.0:
            line += f" xvel={g(s.xvel)}"
        if s.yvel != 0.0:
            line += f" yvel={g(s.yvel)}"
        if i > 0:
            geo = {1: "rectangle", 2: "circle", 3: "point"}[s.geometry]
            line += f" geometry={geo} xmin={g(s.xmin)} xmax={g(s.xmax)} ymin={g(s.ymin)} ymax={g(s.ymax)}"
            if s.geometry == 2:
                line += f" radius={g(s.radius)}"
        lines.append(line)
    lines += [f" x_cells={deck.x_cells}", f" y_cells={deck.y_cells}", f" xmin={g(deck.xmin)}", f" ymin={g(deck.ymin)}",
              f" xmax={g(deck.xmax)}", f" ymax={g(deck.ymax)}", f" initial_timestep={g(deck.initial_timestep)}",
              f" timestep_rise={g(deck.timestep_rise)}", f" max_timestep={g(deck.max_timestep)}",
              f" end_time={g(deck.end_time)}", f" end_step={deck.end_step}",
              f" summary_frequency={deck.summary_frequency}", "*endclover", ""]
    return "\n".join(lines)


def cloverleaf(deck, warmup_steps=0, dump_dir=None, max_summaries=100000):
    """Runs a CloverLeaf deck on the GPU. Returns (summaries[n, 8], device_seconds);
    columns: step, time, volume, mass, internal energy, kinetic energy, pressure sum, dt."""
    out = np.zeros((max_summaries, 8))
    n = ctypes.c_int(0)
    secs = ctypes.c_double(0.0)
    check(lib().ops_b200_app_cloverleaf(ctypes.byref(deck), warmup_steps, out.ctypes.data, max_summaries,
                                        ctypes.byref(n), ctypes.byref(secs),
                                        dump_dir.encode() if dump_dir else None))
    return out[:n.value].copy(), secs.value


# ---------------------------------------------------------------------------
# CloverLeaf 3D
# ---------------------------------------------------------------------------
# apps/c/CloverLeaf_3D/read_input.cpp:44-80 defaults, overridden by the deck.
CLOVER3D_DEFAULTS = dict(x_cells=10, y_cells=10, z_cells=10, xmin=0.0, ymin=0.0, zmin=0.0, xmax=100.0, ymax=100.0,
                         zmax=100.0, initial_timestep=0.1, timestep_rise=1.05, max_timestep=1.0, end_time=10.0,
                         end_step=640000, summary_frequency=10)
GEOMETRY3D = {"cuboid": 1, "sphere": 2, "point": 3}


def clover3d_deck(**kw):
    """A 3D deck from keyword values; `states` is a list of dicts with density,
    energy and optionally xvel, yvel, zvel, geometry, xmin..zmax, radius."""
    from ._lib import Clover3DDeck
    d = Clover3DDeck()
    vals = dict(CLOVER3D_DEFAULTS)
    vals.update({k: v for k, v in kw.items() if k != "states"})
    for k, v in vals.items():
        setattr(d, k, v)
    states = kw["states"]
    d.number_of_states = len(states)
    for i, s in enumerate(states):
        st = d.states[i]
        st.density, st.energy = s["density"], s["energy"]
        st.xvel, st.yvel, st.zvel = s.get("xvel", 0.0), s.get("yvel", 0.0), s.get("zvel", 0.0)
        g = s.get("geometry", 0)
        st.geometry = GEOMETRY3D.get(g, g) if isinstance(g, str) else g
        for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "radius"):
            setattr(st, k, s.get(k, 0.0))
    return d


def clover3d_deck_text(deck):
    """The 3D deck as clover.in text for the reference build. The reference
    reads checkpoint_frequency as a divisor every step (clover_leaf.cpp:204)
    and leaves it 0 when absent, so the text always sets it (its checkpoint
    hook does nothing in a build without HDF5)."""
    g = lambda v: repr(float(v))
    lines = ["*clover"]
    for i in range(deck.number_of_states):
        s = deck.states[i]
        line = f" state {i + 1} density={g(s.density)} energy={g(s.energy)}"
        for k in ("xvel", "yvel", "zvel"):
            if getattr(s, k) != 0.0:
                line += f" {k}={g(getattr(s, k))}"
        if i > 0:
            geo = {1: "cuboid", 2: "sphere", 3: "point"}[s.geometry]
            line += (f" geometry={geo} xmin={g(s.xmin)} xmax={g(s.xmax)} ymin={g(s.ymin)} ymax={g(s.ymax)}"
                     f" zmin={g(s.zmin)} zmax={g(s.zmax)}")
            if s.geometry == 2:
                line += f" radius={g(s.radius)}"
        lines.append(line)
    lines += [f" x_cells={deck.x_cells}", f" y_cells={deck.y_cells}", f" z_cells={deck.z_cells}",
              f" xmin={g(deck.xmin)}", f" ymin={g(deck.ymin)}", f" zmin={g(deck.zmin)}", f" xmax={g(deck.xmax)}",
              f" ymax={g(deck.ymax)}", f" zmax={g(deck.zmax)}", f" initial_timestep={g(deck.initial_timestep)}",
              f" timestep_rise={g(deck.timestep_rise)}", f" max_timestep={g(deck.max_timestep)}",
              f" end_time={g(deck.end_time)}", f" end_step={deck.end_step}",
              f" summary_frequency={deck.summary_frequency}", " checkpoint_frequency=10", "*endclover", ""]
    return "\n".join(lines)


def cloverleaf3d(deck, warmup_steps=0, dump_dir=None, max_summaries=100000):
    """Runs a CloverLeaf 3D deck on the GPU. Returns (summaries[n, 8], device_seconds);
    columns as cloverleaf()."""
    out = np.zeros((max_summaries, 8))
    n = ctypes.c_int(0)
    secs = ctypes.c_double(0.0)
    check(lib().ops_b200_app_cloverleaf3d(ctypes.byref(deck), warmup_steps, out.ctypes.data, max_summaries,
                                          ctypes.byref(n), ctypes.byref(secs),
                                          dump_dir.encode() if dump_dir else None))
    return out[:n.value].copy(), secs.value


# ---------------------------------------------------------------------------
# TeaLeaf
# ---------------------------------------------------------------------------
# read_input.cpp:70-103 defaults (Jacobi, no preconditioner, conductivity).
TEA_DEFAULTS = dict(x_cells=10, y_cells=10, xmin=0.0, ymin=0.0, xmax=100.0, ymax=100.0, initial_timestep=0.1,
                    end_time=10.0, end_step=640000, summary_frequency=10, max_iters=1000, eps=1e-10,
                    coefficient=1, preconditioner=0, solver=0, reflective_boundary=0, check_result=0,
                    fused=0, mixed=0, true_residual_stop=0, reliable_delta=0.1,
                    ch_cg_presteps=25, ch_cg_epslim=1.0, ppcg_inner_steps=-1)
TEA_SOLVERS = {0: "tl_use_jacobi", 1: "tl_use_cg", 2: "tl_use_chebyshev", 3: "tl_use_ppcg"}
# columns of a solve record (OPS_B200_TEA_SOLVE_COLS)
TEA_SOLVE_COLS = ("iterations", "initial_residual", "error_ratio", "exact_ratio", "true_ratio", "reliable_updates",
                  "seconds", "ppcg_inner_iterations", "switch_iteration", "eigmin", "eigmax", "est_itc")


def tea_deck(**kw):
    from ._lib import TeaDeck
    d = TeaDeck()
    vals = dict(TEA_DEFAULTS)
    vals.update({k: v for k, v in kw.items() if k != "states"})
    for k, v in vals.items():
        setattr(d, k, v)
    states = kw["states"]
    d.number_of_states = len(states)
    for i, s in enumerate(states):
        st = d.states[i]
        st.density, st.energy = s["density"], s["energy"]
        g = s.get("geometry", 0)
        st.geometry = GEOMETRY.get(g, g) if isinstance(g, str) else g
        for k in ("xmin", "xmax", "ymin", "ymax", "radius"):
            setattr(st, k, s.get(k, 0.0))
    return d


def tea_deck_text(deck):
    """The deck as tea.in text for the reference build."""
    g = lambda v: repr(float(v))
    lines = ["*tea"]
    for i in range(deck.number_of_states):
        s = deck.states[i]
        line = f" state {i + 1} density={g(s.density)} energy={g(s.energy)}"
        if i > 0:
            geo = {1: "rectangle", 2: "circle", 3: "point"}[s.geometry]
            line += f" geometry={geo} xmin={g(s.xmin)} xmax={g(s.xmax)} ymin={g(s.ymin)} ymax={g(s.ymax)}"
            if s.geometry == 2:
                line += f" radius={g(s.radius)}"
        lines.append(line)
    lines += [f" x_cells={deck.x_cells}", f" y_cells={deck.y_cells}", f" xmin={g(deck.xmin)}", f" ymin={g(deck.ymin)}",
              f" xmax={g(deck.xmax)}", f" ymax={g(deck.ymax)}", f" initial_timestep={g(deck.initial_timestep)}",
              f" end_time={g(deck.end_time)}", f" end_step={deck.end_step}",
              f" summary_frequency={deck.summary_frequency}", f" tl_max_iters={deck.max_iters}",
              f" tl_eps={deck.eps!r}"]
    lines.append(" " + TEA_SOLVERS[deck.solver])
    if deck.solver in (2, 3):
        lines += [f" tl_ch_cg_presteps={deck.ch_cg_presteps}", f" tl_ch_cg_epslim={g(deck.ch_cg_epslim)}",
                  f" tl_ppcg_inner_steps={deck.ppcg_inner_steps}"]
    if deck.preconditioner == 1:
        lines.append(" tl_preconditioner_type=jac_diag")
    lines.append(" tl_coefficient_inverse_density" if deck.coefficient == 2 else " tl_coefficient_density")
    if deck.reflective_boundary:
        lines.append(" reflective_boundary")
    if deck.check_result:
        lines.append(" tl_check_result=1")
    lines += ["*endtea", ""]
    return "\n".join(lines)


def tealeaf(deck, dump_dir=None, max_rows=100000):
    """Runs a TeaLeaf deck. Returns (summaries[n, 6], solves[m, 12], device_seconds):
    summaries: step, time, volume, mass, internal energy, temperature;
    solves: the TEA_SOLVE_COLS columns (iterations, initial residual, error
    ratio, exact residual ratio, true FP64 residual ratio (fused solves, else
    -1), reliable updates, solve device seconds, PPCG inner iterations, the
    iteration Chebyshev/PPCG took over (-1 if not), eigenvalue bounds,
    Chebyshev's estimated iteration count (-1 if none))."""
    out = np.zeros((max_rows, 6))
    sv = np.zeros((max_rows, len(TEA_SOLVE_COLS)))
    n, ns = ctypes.c_int(0), ctypes.c_int(0)
    secs = ctypes.c_double(0.0)
    check(lib().ops_b200_app_tealeaf(ctypes.byref(deck), out.ctypes.data, max_rows, ctypes.byref(n), sv.ctypes.data,
                                     max_rows, ctypes.byref(ns), ctypes.byref(secs),
                                     dump_dir.encode() if dump_dir else None))
    return out[:n.value].copy(), sv[:ns.value].copy(), secs.value
