"""The long-horizon parity report (oracle/parity.py) on CPU: the f32 oracle
checked against itself and against the f64 oracle over a refined 3D snow
scene, so the report's structure and pass rule are exercised without a GPU."""
import numpy as np

import parity as PY


def test_parity_report_on_oracle_runs():
    from agimp import scenes
    scene = scenes.make_config(3, scale=0.2)
    o32 = PY.make_oracle(scene, False)
    o64 = PY.make_oracle(scene, True)
    steps = 12
    PY.run(o32, scene, 0, steps, 4)
    PY.run(o64, scene, 0, steps, 4)
    p32 = o32.particles()
    boxes = PY.grid_boxes(p32["x"], scene.coarsest, scene.level)
    assert all(n > 0 for _, n in boxes)
    grids = PY.oracle_grids(o32, boxes)
    rep = PY.report({"x": p32["x"], "v": p32["v"], "g": p32["g"]}, grids, o32, o64, scene.x, boxes, steps)
    assert rep["vs_f32_oracle"]["position_rel"] == 0.0
    assert rep["vs_f32_oracle"]["grid_momentum_rel"] == [0.0] * scene.level
    fl = rep["f32_vs_f64_floor"]
    assert 0 < fl["position_rel"] < 1e-3 and fl["velocity_rel"] < 1e-3
    assert all(0 <= e < 1e-3 for e in fl["grid_momentum_rel"])
    assert rep["pass"] and rep["levels_equal_f32"]
    # a planted error in the checked state fails the rule
    bad = {"x": p32["x"] + np.where(np.arange(len(p32["x"]))[:, None] == 0, 0.05, 0.0), "v": p32["v"]}
    assert not PY.report(bad, grids, o32, o64, scene.x, boxes, steps)["pass"]
