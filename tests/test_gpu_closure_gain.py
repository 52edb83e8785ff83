"""What the trained closure gains over the plain scheme, on a seed it never saw.

The committed network (multiphysics_fvm_b200/data/closure_kh3d_64.npz) was
trained by ``python -m multiphysics_fvm_b200.closure_train`` on 32 seeded 3D
Kelvin-Helmholtz runs at 256^3 filtered to 64^3.  Here a new seed is run at
256^3 on the device, and two things are checked:

* a priori: on windows of that run, the network's predicted defect explains
  most of the plain 64^3 scheme's defect (its loss is well below the loss of no
  correction on the same windows);
* a posteriori: the 64^3 run with the closure attached stays closer to the
  filtered 256^3 run than the plain 64^3 run, at every checkpoint to t = 0.5,
  with no positivity fallback and a clean device status.
"""
import dataclasses
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "multiphysics_fvm_b200", "data", "closure_kh3d_64.npz")
SEED = 4321


def test_trained_closure_beats_the_plain_coarse_run():
    from multiphysics_fvm_b200 import closure as CL
    from multiphysics_fvm_b200 import closure_train as T
    assert os.path.exists(WEIGHTS), WEIGHTS
    meta = json.loads(str(np.load(WEIGHTS)["meta"]))
    net = CL.Closure((64, 64, 64))
    net.load(WEIGHTS)
    net.set_limiter(bool(meta.get("fct", False)))
    beta = float(meta["beta"])
    k = int(meta["config"].get("defect_steps", 1))
    cfg = T.Config(fine=256, factor=4, t_end=0.5, dt_coarse=2e-3, sample_every=10, defect_steps=k, beta=beta)

    U, D = T.generate(dataclasses.replace(cfg, t_end=0.2), [SEED], log=lambda *_: None)
    apri = T.apriori_loss(net, U, D, cfg)
    w = np.asarray(net.norm["loss_weight"])
    zero = float(sum(w[q] * D[:, q].double().pow(2).mean().item() for q in range(5)))
    assert apri < 0.7 * zero, f"a-priori loss {apri:.3f} vs {zero:.3f} without correction"

    row = T.evaluate(cfg, net, [SEED], betas=[beta], checkpoints=2, log=lambda *_: None)[0]
    plain, closed = row["plain"], row[f"closure_b{beta:g}"]
    assert plain["status"] == 0 and closed["status"] == 0
    assert closed["switched"] == 0
    for t, e_c, e_p in zip(row["t"], closed["err"], plain["err"]):
        assert e_c < 0.9 * e_p, f"t={t}: closure {e_c:.4f} vs plain {e_p:.4f}"


def test_setup_closure_key_uses_the_weights_selection():
    """solver.run(setup) with setup["closure"] = {"weights": path} and no beta
    or fct attaches the network with the values stored with the weights: the
    run ends bitwise equal to Simulation + Closure.attach(sim, beta=meta beta)."""
    import math
    from multiphysics_fvm_b200 import closure, solver
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.grid.geometry import build_grid
    from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as kh
    meta = json.loads(str(np.load(WEIGHTS)["meta"]))
    s = kh.get_setup(64, 64, 64, seed=7, n_steps=6, precision="fp32")
    a = solver.run(dict(s, closure={"weights": WEIGHTS}), verbose=False)
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], build_grid("cartesian", s["grid_config"]),
                                           s["initial_conditions"]["parameters"])
    b = Simulation.from_setup(s)
    b.upload(U)
    b.set_time(0.0, math.inf, 0.4)
    net = closure.Closure(b.n)
    net.load(WEIGHTS)
    net.set_limiter(bool(meta.get("fct", False)))
    net.attach(b, beta=float(meta["beta"]))
    b.step(6)
    assert a.status() == 0 and b.status() == 0
    assert np.array_equal(a.download(), b.download())
