"""The pseudo-trajectory restatement (oracle/post_oracle.py:pivtrajectories)
against hand-computed trajectories of PIVtrajectories(_grid)
(src/postprocessing/postprocessing.jl:988-1120)."""
import numpy as np

import oracle.post_oracle as PO


def test_uniform_field_straight_lines_and_freeze():
    # y moves +1.5 per frame, x -0.5: positions 2, 3.5, 5, 6.5, 8, 9.5, 11 (> 10: frozen at 9.5)
    U = np.full((10, 12, 8, 9), 1.5, np.float32)
    V = np.full_like(U, -0.5)
    W = np.zeros_like(U)
    TY, TX, TZ = PO.pivtrajectories([U, V, W], 1, 9, grid=True, subregion=[(2, 2), (6, 6), (4, 4)])
    assert TY.shape == (8, 1) and TY.dtype == np.float32
    assert TY[:, 0].tolist() == [2, 3.5, 5, 6.5, 8, 9.5, 9.5, 9.5]
    assert TX[:, 0].tolist() == [6, 5.5, 5, 4.5, 4, 3.5, 3.5, 3.5]
    assert TZ[:, 0].tolist() == [4] * 8


def test_sampling_follows_the_rounded_position_ties_to_even():
    # the displacement at y = 3.5 is read at y = 4 (ties to even), at 4.5 from 4, at 5.5 from 6
    U = np.zeros((12, 5, 5, 6), np.float64)
    U[3 - 1, :, :, 0] = 0.5      # frame 1 at y = 3: move to 3.5
    U[4 - 1, :, :, 1] = 1.0      # frame 2 at round(3.5) = 4: move to 4.5
    U[4 - 1, :, :, 2] = 1.0      # frame 3 at round(4.5) = 4: move to 5.5
    U[6 - 1, :, :, 3] = -2.0     # frame 4 at round(5.5) = 6: move to 3.5
    V, W = np.zeros_like(U), np.zeros_like(U)
    TY, _, _ = PO.pivtrajectories([U, V, W], 1, 6, grid=True, subregion=[(3, 3), (2, 2), (2, 2)])
    assert TY[:, 0].tolist() == [3, 3.5, 4.5, 5.5, 3.5]


def test_grid_order_defaults_and_scale():
    U = np.ones((6, 7, 5, 3), np.float32)
    V, W = np.zeros_like(U), np.zeros_like(U)
    TY, TX, TZ = PO.pivtrajectories([U, V, W], 1, 3, grid=True, scale=(2, 1, 1))
    # default region 2:dims-1 per axis, y fastest
    assert TY.shape == (2, 4 * 5 * 3)
    assert TY[0, :4].tolist() == [2, 3, 4, 5] and TX[0, :5].tolist() == [2, 2, 2, 2, 3]
    inside = TY[0] + 2 <= 6  # y = 5 would reach 7 > dims[0] = 6: it stays
    assert (TY[1][inside] == TY[0][inside] + 2).all() and (TY[1][~inside] == TY[0][~inside]).all()


def test_random_starts_are_seeded_and_inside_the_region():
    g = np.random.default_rng(3)
    U = g.normal(0, 1, (9, 8, 7, 4)).astype(np.float32)
    V, W = g.normal(0, 1, U.shape).astype(np.float32), g.normal(0, 1, U.shape).astype(np.float32)
    a = PO.pivtrajectories([U, V, W], 1, 4, numpoints=50, seed=11, subregion=[(3, 6), (1, 0), (2, 2)])
    b = PO.pivtrajectories([U, V, W], 1, 4, numpoints=50, seed=11, subregion=[(3, 6), (1, 0), (2, 2)])
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert ((a[0][0] >= 3) & (a[0][0] <= 6)).all() and ((a[1][0] >= 2) & (a[1][0] <= 7)).all()
    assert (a[2][0] == 2).all()
