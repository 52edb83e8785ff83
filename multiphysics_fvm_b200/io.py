"""Snapshot I/O (reference: src/io.py:14-96).

``save_snapshot`` writes ``snapshot_{n:06d}.h5`` with groups ``U`` and
``setup`` and attributes ``time``/``iteration`` when h5py is importable, and
otherwise the same content as ``snapshot_{n:06d}.npz``.  ``load_snapshot``
reads either format and returns ``(U, setup_attrs, time, iteration)``.
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


def save_snapshot(U: dict, setup: dict, time: float, iteration: int, save_dir: str) -> str:
    os.makedirs(save_dir, exist_ok=True)
    attrs = _attrs(setup)
    if h5py is not None:
        path = f"{save_dir}/snapshot_{iteration:06d}.h5"
        with h5py.File(path, "w") as f:
            gu, gs = f.create_group("U"), f.create_group("setup")
            for k, v in attrs.items():
                gs.attrs[k] = v
            f.attrs["time"] = time
            f.attrs["iteration"] = iteration
            for k, v in U.items():
                gu.create_dataset(k, data=v)
        return path
    path = f"{save_dir}/snapshot_{iteration:06d}.npz"
    np.savez(path, time=np.float64(time), iteration=np.int64(iteration), setup=json.dumps(attrs),
             **{f"U/{k}": v for k, v in U.items()})
    return path


def load_snapshot(filepath: str):
    if filepath.endswith(".h5"):
        if h5py is None:
            raise ImportError("h5py is required to read .h5 snapshots")
        with h5py.File(filepath, "r") as f:
            setup = dict(f["setup"].attrs.items())
            return ({k: f["U"][k][:] for k in f["U"]}, setup, f.attrs["time"], f.attrs["iteration"])
    z = np.load(filepath)
    U = {k[2:]: z[k] for k in z.files if k.startswith("U/")}
    return U, json.loads(str(z["setup"])), float(z["time"]), int(z["iteration"])
