"""Snapshot I/O (reference: src/io.py:14-96).

``save_snapshot`` writes ``snapshot_{n:06d}.h5`` with groups ``U`` and
``setup`` and attributes ``time``/``iteration`` when h5py is importable, and
otherwise the same content as ``snapshot_{n:06d}.npz``.  ``load_snapshot``
reads either format and returns ``(U, setup_attrs, time, iteration)``.

As in the reference loop (src/solver.py:140-148), snapshot ``n`` holds the state
after step ``n`` but is labelled with the time before it.  ``solver.run`` also
passes ``state_time``, the time of the stored state, which is written as one
more attribute; ``restore_snapshot`` needs it to restart a run where it stopped
(the reference has no restart).
"""
from __future__ import annotations

import json
import os

import numpy as np

try:  # optional dependency, as in the reference
    import h5py  # type: ignore
except ImportError:  # pragma: no cover - depends on the environment
    h5py = None


def _attrs(setup: dict) -> dict:
    a = {"coordinate_system": setup["coordinate_system"]}
    a.update(setup["grid_config"])
    for k, v in setup["physical_parameters"].items():
        a[k] = v
    return a


def save_snapshot(U: dict, setup: dict, time: float, iteration: int, save_dir: str,
                  state_time: float | None = None) -> str:
    """src/io.py:14-62; ``state_time`` (optional) is stored as a file
    attribute next to ``time``."""
    os.makedirs(save_dir, exist_ok=True)
    attrs = _attrs(setup)
    extra = {} if state_time is None else {"state_time": np.float64(state_time)}
    if h5py is not None:
        path = f"{save_dir}/snapshot_{iteration:06d}.h5"
        with h5py.File(path, "w") as f:
            gu, gs = f.create_group("U"), f.create_group("setup")
            for k, v in attrs.items():
                gs.attrs[k] = v
            f.attrs["time"] = time
            f.attrs["iteration"] = iteration
            for k, v in extra.items():
                f.attrs[k] = v
            for k, v in U.items():
                gu.create_dataset(k, data=v)
        return path
    path = f"{save_dir}/snapshot_{iteration:06d}.npz"
    np.savez(path, time=np.float64(time), iteration=np.int64(iteration), setup=json.dumps(attrs),
             **extra, **{f"U/{k}": v for k, v in U.items()})
    return path


def _read(filepath: str):
    """(U, setup attrs, time, iteration, state_time or None) of either format."""
    if filepath.endswith(".h5"):
        if h5py is None:
            raise ImportError("h5py is required to read .h5 snapshots")
        with h5py.File(filepath, "r") as f:
            setup = dict(f["setup"].attrs.items())
            st = f.attrs["state_time"] if "state_time" in f.attrs else None
            return ({k: f["U"][k][:] for k in f["U"]}, setup, f.attrs["time"], f.attrs["iteration"], st)
    with np.load(filepath) as z:
        U = {k[2:]: z[k] for k in z.files if k.startswith("U/")}
        st = float(z["state_time"]) if "state_time" in z.files else None
        return U, json.loads(str(z["setup"])), float(z["time"]), int(z["iteration"]), st


def load_snapshot(filepath: str):
    """src/io.py:65-96: ``(U, setup_attrs, time, iteration)``."""
    return _read(filepath)[:4]


def restore_snapshot(filepath: str, setup: dict, U: dict):
    """Fill the freshly allocated state ``U`` of ``setup`` from a snapshot and
    return ``(state_time, steps_done)`` for a restart.

    Raises ``ValueError`` when the snapshot has no ``state_time`` (a snapshot
    written without it is labelled with the time before its step, so the time
    of its state is not known), when its coordinate system or grid differs
    from ``setup``'s, or when its variables or array shapes differ from ``U``'s.
    """
    V, attrs, _, iteration, state_time = _read(filepath)
    if state_time is None:
        raise ValueError(f"{filepath}: no state_time attribute; cannot restart from it")
    if attrs.get("coordinate_system") != setup["coordinate_system"]:
        raise ValueError(f"{filepath}: coordinate system {attrs.get('coordinate_system')!r} "
                         f"!= {setup['coordinate_system']!r}")
    for k, v in setup["grid_config"].items():
        if k not in attrs or float(attrs[k]) != float(v):
            raise ValueError(f"{filepath}: grid_config[{k!r}] = {attrs.get(k)!r} != {v!r}")
    if set(V) != set(U):
        raise ValueError(f"{filepath}: variables {sorted(V)} != {sorted(U)}")
    for k in U:
        if V[k].shape != U[k].shape:
            raise ValueError(f"{filepath}: {k} has shape {V[k].shape}, expected {U[k].shape}")
        U[k][...] = V[k]
    return float(state_time), int(iteration) + 1
