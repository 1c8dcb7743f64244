"""bench.solve_bytes: the whole-solve algorithmic HBM bytes from per-k counters, on a
hand-computed case (N = 10, so M = 20; 2 bands; restart dimension 4)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_solve_bytes_hand_computed():
    c = dict(ls_iter=5, refine=2, es_iter=6, restarts=1)
    # CG 5 x (920 + 1120), refinement 2 x (1840 + 960), Lanczos j+1 = 1,2,3,4,3,4:
    # 6 x 1280 + 2 x 17 x 320, restart 8 x 320, restoration 2 x 80 x 16
    assert bench.solve_bytes([c], 10, 2, 4, True) == 39480
    # FP64: the CG iterations move (100 x 16 + 30 x 8) + 7 x 20 x 16 each, no refinement
    c64 = dict(ls_iter=5, refine=0, es_iter=6, restarts=1)
    assert bench.solve_bytes([c64], 10, 2, 4, False) == 5 * (1840 + 2240) + 7680 + 10880 + 2560 + 2560
    assert bench.solve_bytes([c, c], 10, 2, 4, True) == 2 * 39480
