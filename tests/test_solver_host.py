"""Host logic of ``solver.run`` and of snapshot restarts, without a GPU.

``solver.run`` is driven with a stand-in simulation object whose clock follows
the reference loop (src/solver.py:137-151: step while t <= t_end, output after
step n when n % output_frequency == 0, labelled with the time before the step),
so the output steps, their labels and the restart numbering can be checked
against a direct restatement of that loop.
"""
import math

import numpy as np
import pytest

from multiphysics_fvm_b200 import backend, io, solver
from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as kh


class FakeSim:
    """Clock and state of a simulation: each step adds 1 to every interior
    density cell and advances t by a step-dependent dt; steps are skipped once
    t > t_end, as the device clock does."""

    def __init__(self):
        self.t, self.n, self.dt, self.t_end, self.U = 0.0, 0, 0.0, math.inf, None

    def upload(self, U):
        self.U = {k: np.array(v) for k, v in U.items()}

    def set_time(self, t0, t_end, cfl):
        self.t, self.n, self.t_end = float(t0), 0, float(t_end)

    @staticmethod
    def dt_at(t):
        return 0.01 + 0.001 * math.sin(7.0 * t)

    def step(self, k):
        for _ in range(k):
            if self.t > self.t_end:
                return
            self.dt = self.dt_at(self.t)
            self.U["mass_density"][1:-1, 1:-1, 1:-1] += 1.0
            self.t += self.dt
            self.n += 1

    def time(self):
        return self.t, self.n, self.dt

    def download_into(self, U):
        for k in U:
            U[k][...] = self.U[k]

    def status(self):
        return 0


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(backend.Simulation, "from_setup", classmethod(lambda cls, s, **kw: FakeSim()))


def reference_loop(t_start, t_end, out_freq, n_max=None):
    """The reference's loop (src/solver.py:137-151) on FakeSim's clock:
    returns the (iteration, label time) of every output and the step count."""
    t, n, outs = t_start, 0, []
    while t <= t_end and (n_max is None or n < n_max):
        dt = FakeSim.dt_at(t)
        if n % out_freq == 0:
            outs.append((n, t))
        t += dt
        n += 1
    return outs, n


def _setup(out_freq, saver, n_steps=None, t_end=5.0):
    s = kh.get_setup(8, 6, 1, n_steps=n_steps)
    s["time_config"]["t_end"] = t_end
    if n_steps is None:
        del s["time_config"]["n_steps"]
    s["save_config"] = {"saver": saver, "output_frequency": out_freq, "directory": "unused"}
    return s


@pytest.mark.parametrize("out_freq,t_end", [(1, 0.05), (7, 0.3), (10, 0.25), (25, 0.1)])
def test_output_steps_and_labels_follow_the_reference_loop(fake, out_freq, t_end):
    seen = []
    sim = solver.run(_setup(out_freq, lambda U, s, t, n, d: seen.append((n, t)), t_end=t_end), verbose=False)
    outs, n_ref = reference_loop(0.0, t_end, out_freq)
    assert sim.n == n_ref
    assert [n for n, _ in seen] == [n for n, _ in outs]
    assert [t for _, t in seen] == [t for _, t in outs]  # exact: read before the output step


def test_step_counted_run_outputs(fake):
    seen = []
    sim = solver.run(_setup(10, lambda U, s, t, n, d: seen.append(n), n_steps=35), verbose=False)
    assert sim.n == 35 and seen == [0, 10, 20, 30]


def test_saved_state_is_the_state_after_the_labelled_step(fake, tmp_path):
    s = _setup(10, io.save_snapshot, n_steps=25)
    s["save_config"]["directory"] = str(tmp_path)
    solver.run(s, verbose=False)
    from multiphysics_fvm_b200.grid.geometry import build_grid
    U0 = s["physics"].allocate_u(s["grid_config"])
    solver.apply_ics(U0, s["physical_parameters"], build_grid("cartesian", s["grid_config"]), s["initial_conditions"])
    I = (slice(1, -1),) * 3
    for it in (0, 10, 20):
        U, attrs, t, n = io.load_snapshot(str(tmp_path / f"snapshot_{it:06d}.npz"))
        assert n == it and np.array_equal(U["mass_density"][I], U0["mass_density"][I] + (it + 1))
        assert attrs["nx1"] == 8 and attrs["coordinate_system"] == "cartesian"


def test_restart_continues_numbering_time_and_state(fake, tmp_path):
    full = tmp_path / "full"
    s = _setup(10, io.save_snapshot, n_steps=35)
    s["save_config"]["directory"] = str(full)
    a = solver.run(s, verbose=False)
    part = tmp_path / "part"
    r = _setup(10, io.save_snapshot, n_steps=35)
    r["save_config"]["directory"] = str(part)
    r["restart_from"] = str(full / "snapshot_000010.npz")
    b = solver.run(r, verbose=False)
    assert b.n == 35 - 11  # steps left after the restart point
    assert sorted(p.name for p in part.iterdir()) == ["snapshot_000020.npz", "snapshot_000030.npz"]
    for it in (20, 30):
        Ua, _, ta, _ = io.load_snapshot(str(full / f"snapshot_{it:06d}.npz"))
        Ub, _, tb, _ = io.load_snapshot(str(part / f"snapshot_{it:06d}.npz"))
        assert ta == tb and all(np.array_equal(Ua[k], Ub[k]) for k in Ua)
    assert a.t == b.t and np.array_equal(a.U["mass_density"], b.U["mass_density"])


def test_restore_snapshot_checks(tmp_path):
    s = kh.get_setup(8, 6, 1)
    from multiphysics_fvm_b200.physics import navier_stokes
    U = navier_stokes.allocate_u(s["grid_config"])
    for k, v in U.items():
        v[...] = np.random.default_rng(len(k)).standard_normal(v.shape)
    with_t = io.save_snapshot(U, s, 0.5, 7, str(tmp_path / "a"), state_time=0.52)
    without_t = io.save_snapshot(U, s, 0.5, 7, str(tmp_path / "b"))
    V = navier_stokes.allocate_u(s["grid_config"])
    assert io.restore_snapshot(with_t, s, V) == (0.52, 8)
    assert all(np.array_equal(U[k], V[k]) for k in U)
    assert len(io.load_snapshot(with_t)) == 4  # the reference's return shape
    with pytest.raises(ValueError, match="state_time"):
        io.restore_snapshot(without_t, s, V)
    other = kh.get_setup(8, 7, 1)
    with pytest.raises(ValueError, match="nx2"):
        io.restore_snapshot(with_t, other, navier_stokes.allocate_u(other["grid_config"]))
    s2 = dict(s, coordinate_system="cylindrical")
    with pytest.raises(ValueError, match="coordinate system"):
        io.restore_snapshot(with_t, s2, V)
    W = {k: v for k, v in V.items() if k != "energy_density"}
    with pytest.raises(ValueError, match="variables"):
        io.restore_snapshot(with_t, s, W)
