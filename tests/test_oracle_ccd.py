"""Known answers of the oracle's line-search step bounds (additive CCD of ACCD.cu:373-535 as
GIPC::self_largestFeasibleStepSize applies it, GIPC.cu:8880; the ground bound of
GIPC::ground_largestFeasibleStepSize, GIPC.cu:8986).

For a head-on approach that closes a unit gap at t = 0.5, with slackness 0.8 (the reference's
slackness_m) the additive CCD takes its first conservative step, 0.8 * d / L = 0.4, where the
remaining gap (0.2) equals the kept fraction eta = 0.2 of the initial one, and stops there:
the step is 0.4.  Tolerance 1e-12.
"""
import numpy as np
import pytest

import oracle

TRI = np.array([[0.2, 0.2, 1.0], [0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
PT = np.array([[-1, 1, 2, 3]], np.int32)  # point 0 against triangle (1, 2, 3)
EDGES = np.array([[-1.0, 0.0, 1.0], [1.0, 0.0, 1.0], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
EE = np.array([[0, 1, 2, 3]], np.int32)


def _dir(n, moving, disp):
    """move_dir: the reference's step direction is -move_dir."""
    d = np.zeros((n, 3))
    d[moving] = -np.asarray(disp)
    return d


def test_point_triangle_head_on():
    a, toi = oracle.self_step(TRI, _dir(4, [0], [0, 0, -2.0]), PT, 0.8)
    assert a == pytest.approx(0.4, rel=1e-12) and toi[0] == pytest.approx(0.4, rel=1e-12)


def test_edge_edge_head_on():
    a, toi = oracle.self_step(EDGES, _dir(4, [0, 1], [0, 0, -2.0]), EE, 0.8)
    assert a == pytest.approx(0.4, rel=1e-12) and toi[0] == pytest.approx(0.4, rel=1e-12)


def test_no_motion_and_separation_allow_the_full_step():
    assert oracle.self_step(TRI, np.zeros((4, 3)), PT, 0.8)[0] == 1.0
    assert oracle.self_step(TRI, _dir(4, [0], [0, 0, 2.0]), PT, 0.8)[0] == 1.0
    assert oracle.self_step(EDGES, _dir(4, [0, 1], [0, 0, 3.0]), EE, 0.8)[0] == 1.0


def test_closest_feature_is_a_vertex_or_edge():
    # the point beyond vertex (1, 0, 0), then beyond the edge t0t1: the approach is
    # measured to that feature, not to the triangle's plane
    x = TRI.copy()
    x[0] = [2.0, -1.0, 0.0]
    a, _ = oracle.self_step(x, _dir(4, [0], [-1.0, 1.0, 0.0]), PT, 0.8)  # closes |(1,-1)| = sqrt 2 at t = 1
    assert 0.35 < a < 0.9
    x[0] = [0.5, -1.0, 0.0]
    a, _ = oracle.self_step(x, _dir(4, [0], [0.0, 2.0, 0.0]), PT, 0.8)  # reaches the edge at t = 0.5
    assert a == pytest.approx(0.4, rel=1e-12)


def test_step_is_the_minimum_over_candidates():
    x = np.vstack([TRI, EDGES + [5.0, 0.0, 0.0]])
    d = np.vstack([_dir(4, [0], [0, 0, -2.0]), _dir(4, [0, 1], [0, 0, -4.0])])
    a, toi = oracle.self_step(x, d, np.vstack([PT, EE + 4]), 0.8)
    assert toi[1] == pytest.approx(0.2, rel=1e-12) and a == pytest.approx(0.2, rel=1e-12)


def test_ground_bound():
    x = np.array([[0.0, 1.0, 0.0], [0.0, 2.0, 0.0]])
    d = np.array([[0.0, 2.0, 0.0], [0.0, -1.0, 0.0]])  # the first falls, the second rises
    assert oracle.ground_step(x, d, [0, 1], 0.0, 0.8) == pytest.approx(0.4, rel=1e-12)
    assert oracle.ground_step(x, d, [1], 0.0, 0.8) == 1.0


def test_cfl_speed():
    d = np.array([[3.0, 4.0, 0.0], [0.0, 0.0, -12.0], [1.0, 0.0, 0.0]])
    assert oracle.cfl_speed(d, [0, 2]) == 5.0
    assert oracle.cfl_speed(d, [0, 1, 2]) == 12.0
    assert oracle.cfl_speed(d, []) == 0.0
