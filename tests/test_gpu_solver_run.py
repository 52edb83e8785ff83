"""``solver.run(setup)``, the reference-facing entry point (src/solver.py:88-151),
on the device against the oracle's time loop.

* A viscous 3D Rayleigh-Taylor setup (reflecting / Neumann z walls, periodic
  x and y, MUSCL van Leer + HLL + rk3) and a 2D sharp Kelvin-Helmholtz setup
  (periodic, minmod + HLL + SSPRK3), float64, run by step count with snapshots
  every 10 steps. Every snapshot holds the state after its step (relative L2
  <= 1e-10 against the oracle after the same number of steps), is labelled with
  the time before that step (relative 1e-12), and stores the state's own time.
* With ``t_end`` and no step count, the run takes as many steps as the
  reference loop ``while t <= t_end`` takes with the oracle's time steps.
* A run restarted from a snapshot ends bitwise equal to the run it was
  taken from, in float64 and float32.
"""

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

BC_NAMES = {0: "periodic", 1: "neumann", 2: "reflecting", 3: "dirichlet"}
I3 = (slice(None),) + (slice(1, -1),) * 3


def _setup(kind, precision="fp64", n_steps=25):
    if kind == "rt":
        from multiphysics_fvm_b200.setups import rayleigh_taylor_3d as m
        s = m.get_setup(12, 10, 16, seed=3, n_steps=n_steps, precision=precision)
    else:
        from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as m
        s = m.get_setup(32, 24, 1, seed=1, n_steps=n_steps, precision=precision)
    return s


def _initial_state(s):
    from multiphysics_fvm_b200.grid.geometry import build_grid
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], build_grid(s["coordinate_system"],
                                           s["grid_config"]), s["initial_conditions"]["parameters"])
    return U


def _oracle_args(s):
    from multiphysics_fvm_b200.backend import bc_codes
    bcs = [{side: (BC_NAMES[k], v) for side, (k, v) in zip(O.SIDES, row)}
           for row in bc_codes("navier_stokes", s["boundary_conditions"])]
    sch = s["space_schemes"]
    return (s["physical_parameters"], O.Geometry(s["coordinate_system"], s["grid_config"]),
            dict(reconstructor=sch["reconstructor"].__name__, slope_limiter=sch["slope_limiter"].__name__,
                 riemann_solver=sch["riemann_solver"].__name__), bcs, s["time_integrator"].__name__,
            float(s["time_config"]["CFL"]))


def _stack(U):
    from multiphysics_fvm_b200.physics import navier_stokes
    return np.stack([U[k] for k in navier_stokes.VARIABLES])


def _run(s, directory=None, freq=10, restart=None):
    from multiphysics_fvm_b200 import io, solver
    s = dict(s, save_config={"saver": io.save_snapshot if directory else None, "output_frequency": freq,
                             "directory": str(directory)})
    if restart:
        s["restart_from"] = str(restart)
    return solver.run(s, verbose=False)


@pytest.mark.parametrize("kind", ["rt", "kh"])
def test_snapshots_match_the_oracle_loop(kind, tmp_path):
    from multiphysics_fvm_b200 import io
    s = _setup(kind)
    sim = _run(s, tmp_path)
    prm, geo, sch, bcs, integ, cfl = _oracle_args(s)
    Uo = _stack(_initial_state(s))
    t, states = 0.0, {}
    for n in range(25):
        dt = O.run("navier_stokes", Uo, prm, geo, sch, bcs, integ, cfl, 1)[0]
        states[n] = (t, t + dt, Uo.copy())
        t += dt
    assert sorted(p.name for p in tmp_path.iterdir()) == [f"snapshot_{n:06d}.npz" for n in (0, 10, 20)]
    for n in (0, 10, 20):
        path = str(tmp_path / f"snapshot_{n:06d}.npz")
        U, attrs, t_label, it = io.load_snapshot(path)
        t_pre, t_post, Uref = states[n]
        assert it == n
        assert abs(t_label - t_pre) <= 1e-12 * t_pre
        assert abs(io._read(path)[4] - t_post) <= 1e-12 * t_post
        assert rel_l2(_stack(U)[I3], Uref[I3]) <= 1e-10, n
    assert rel_l2(sim.download()[I3], Uo[I3]) <= 1e-10
    t_dev, steps, _ = sim.time()
    assert steps == 25 and abs(t_dev - t) <= 1e-12 * t and sim.status() == 0


def test_t_end_takes_the_reference_loop_step_count():
    s = _setup("kh")
    prm, geo, sch, bcs, integ, cfl = _oracle_args(s)
    Uo = _stack(_initial_state(s))
    ts = np.cumsum([0.0] + O.run("navier_stokes", Uo, prm, geo, sch, bcs, integ, cfl, 9))
    t_end = 0.5 * (ts[6] + ts[7])  # the loop runs while t <= t_end: steps at t_0 .. t_6
    del s["time_config"]["n_steps"]
    s["time_config"]["t_end"] = t_end
    sim = _run(s, freq=0)
    t, steps, _ = sim.time()
    assert steps == 7 and abs(t - ts[7]) <= 1e-12 * ts[7]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["rt", "kh"])
def test_restart_is_bitwise(kind, precision, tmp_path):
    s = _setup(kind, precision)
    a = _run(s, tmp_path / "a")
    b = _run(_setup(kind, precision), tmp_path / "b", restart=tmp_path / "a" / "snapshot_000010.npz")
    assert b.time()[1] == 25 - 11
    assert np.array_equal(a.download(), b.download())
    assert a.time()[0] == b.time()[0]
    assert sorted(p.name for p in (tmp_path / "b").iterdir()) == ["snapshot_000020.npz"]
