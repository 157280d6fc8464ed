"""Sort cadence by particle speed (host logic of the batch tuner, no GPU)."""
import math
from types import SimpleNamespace

import numpy as np

from particle_transport_b200.batch import cells_per_step, cells_per_step_gamma, sort_cadence, speed_class
from particle_transport_b200.fields import C_LIGHT, M_P
from particle_transport_b200.particles import energy_to_gamma


def test_cells_per_step_of_a_proton():
    # 10 GeV proton: v = c sqrt(1 - 1/gamma^2); dt = 1e-3 s, cells of 1e5 m
    g = energy_to_gamma(10.0)
    p = g * M_P * C_LIGHT * math.sqrt(1 - 1 / g ** 2)
    state = {"p1": np.array([0.6 * p]), "p2": np.array([0.0]), "p3": np.array([0.8 * p])}
    fld = SimpleNamespace(grid=SimpleNamespace(dx=1e5, dy=2e5, dz=3e5))
    v = C_LIGHT * math.sqrt(1 - 1 / g ** 2)
    assert math.isclose(cells_per_step(fld, state, 1e-3), v * 1e-3 / 1e5, rel_tol=1e-12)
    assert math.isclose(cells_per_step_gamma(fld, g, 1e-3), v * 1e-3 / 1e5, rel_tol=1e-12)


def test_speed_classes_and_default_cadence():
    assert speed_class(0.098) == -4 and speed_class(0.98) == -1 and speed_class(9.8) == 3
    assert speed_class(1.0) == speed_class(1.99) != speed_class(2.0)
    assert speed_class(0.0) == speed_class(-1.0)  # clamped, no math domain error
    assert [sort_cadence(c) for c in (0.1, 1.0, 2.0, 3.9, 4.0, 40.0)] == [64, 64, 32, 32, 16, 16]
