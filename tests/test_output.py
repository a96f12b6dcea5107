"""The :saveData output: number formatting and checkpoint ticks (no GPU), and
the files LBMpropagate! writes through the library (GPU)."""
from __future__ import annotations

import csv
import os

import numpy as np
import pytest

from lbmengine import output


@pytest.mark.parametrize("x,text", [(1.0, "1.0"), (1e-5, "1.0e-5"), (123456.0, "123456.0"), (1234567.0, "1.234567e6"),
                                    (0.0001, "0.0001"), (-0.5, "-0.5"), (1e16, "1.0e16"), (2.5e-7, "2.5e-7"),
                                    (1e6, "1.0e6"), (0.00012, "0.00012"), (-64.0, "-64.0"), (0.0, "0.0"),
                                    (float("nan"), "NaN"), (5e-324, "5.0e-324")])
def test_numbers_are_printed_as_julia_prints_them(x, text):
    assert output.julia_float(x) == text
    if text != "NaN":
        assert float(text.replace("e", "e")) == x


def test_checkpoints_follow_julia_range_and_round():
    # round.(range(0, stop = 10, length = 4)) = round.([0, 3.333.., 6.666.., 10]) = [0, 3, 7, 10]
    assert output.checkpoints(0, 1.0, 10, 4) == {0, 3, 7, 10}
    # ties go to even: range(0, stop = 5, length = 3) = [0, 2.5, 5] -> [0, 2, 5]
    assert output.checkpoints(0, 1.0, 5, 3) == {0, 2, 5}
    assert output.checkpoints(7, 1.0, 5, 3) == {7, 10, 12}  # 9.5 -> 10 (even)
    assert len(output.checkpoints(0, 1.0, 100, 100)) == 100


def _read(path):
    with open(path) as f:
        rows = list(csv.reader(f))
    return rows[0], rows[1:]


@pytest.mark.gpu
def test_save_data_writes_the_reference_files(lib, tmp_path, monkeypatch):
    from lbmengine import LBMpropagate, addSquirmer, modelInit
    monkeypatch.chdir(tmp_path)
    kw = dict(dims=2, latticeParameter=1.0, relaxationTimeRatio=0.8, collisionModel="bgk", xlims=(-16.0, 15.0),
              ylims=(-8.0, 7.0), forceDensity=[1e-5, 0.0])
    sq = dict(radius=3.0, position=[0.4, -0.3], swimmingSpeed=2e-3, beta=3.0, coupleForces=True,
              coupleTorques=True, massDensity=2.0)
    m = modelInit(saveData=True, **kw)
    addSquirmer(m, **sq)
    LBMpropagate(m, ticks=30, ticksSaved=4)
    # the same model without output, stepped tick by tick
    ref = modelInit(**kw)
    addSquirmer(ref, **sq)
    names = sorted(os.listdir("output.lbm"))
    assert names == ["fluidTrj_0.csv", "fluidTrj_10.csv", "fluidTrj_20.csv", "fluidTrj_30.csv", "particlesTrj.csv"]
    head, rows = _read("output.lbm/particlesTrj.csv")
    assert head == ["tick", "time", "particleId", "position_x", "position_y", "velocity_x", "velocity_y",
                    "angularVelocity"]
    assert [int(r[0]) for r in rows] == list(range(0, 31))  # at addSquirmer!, then after every tick
    for r in rows[1:]:
        ref.step(1)
        s = ref.particle_states()[0]
        assert [float(v) for v in r[3:8]] == list(s.position[:2]) + list(s.velocity[:2]) + [s.angular_velocity[0]]
        assert r[1] == output.julia_float(ref.time)
    head, rows = _read("output.lbm/fluidTrj_30.csv")
    assert head[:9] == ["tick", "time", "id_x", "id_y", "coordinate_x", "coordinate_y", "massDensity",
                        "fluidVelocity_x", "fluidVelocity_y"] and head[9:] == [f"f{i}" for i in range(1, 10)]
    a = np.array([[float(v) for v in r] for r in rows])
    assert len(rows) == 32 * 16
    np.testing.assert_array_equal(a[:, 6], ref.massDensity.ravel(order="F"))
    np.testing.assert_array_equal(a[:, 7:9], ref.fluidVelocity.reshape(-1, 2, order="F"))
    np.testing.assert_array_equal(a[:, 9:], ref.distributions.reshape(-1, 9, order="F"))
    np.testing.assert_array_equal(a[:, 2], np.tile(np.arange(1, 33), 16))
    assert all(r[6] == output.julia_float(float(r[6])) for r in rows[:50])  # the C++ writer prints as Julia does
