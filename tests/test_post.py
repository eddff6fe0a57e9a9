"""CPU restatement of the reference's post-processing tools, pinned to hand-made
fields with known answers (Extract_Tip.cpp:68-87, coarsening_analysis.cpp:46-165)."""
import numpy as np

import oracle_lib as ol


def test_size_distribution_known_answer_2d():
    f = np.zeros((1, 8, 10))
    f[0, 1:3, 1:3] = 1.0                     # 4 cells, first seed at index 11
    f[0, 5, 0] = f[0, 5, 9] = 1.0            # joined across the x wrap, first seed at index 50
    f[0, 7, 4] = f[0, 0, 4] = 0.9            # joined across the y wrap, first seed at index 4
    avg, vol, sizes = ol.size_distribution(f)
    assert avg == 0.5 and vol == 8            # (max(0.5, 1) + min(0.5, 0)) / 2
    assert sizes.tolist() == [2, 4, 2]        # scan order of first seeds: 4, 11, 50


def test_size_distribution_threshold_and_ge_growth_3d():
    f = np.full((4, 4, 4), 0.1)
    f[0, 0, 0] = 0.9                          # avg = (0.9 + 0.1) / 2 = 0.5
    f[3, 0, 0] = 0.5                          # == avg: grows the island (z wrap) but seeds nothing
    f[2, 2, 2] = 0.5                          # == avg, isolated: no island
    f[1, 3, 3] = 0.7
    avg, vol, sizes = ol.size_distribution(f)
    assert avg == 0.5 and vol == 2
    assert sizes.tolist() == [2, 1]


def test_tip_profile_known_answer():
    g = np.zeros((6, 4, 12))
    g[3, 1, :7] = 0.8
    g[4, 2, :3] = 0.7
    g[5, 0, :11] = 0.6
    g[2, 0, :] = 1.0                          # below the window (z < Nz/2): ignored
    tip, m = ol.tip_profile(g, dz=4)
    assert tip.tolist() == [6, 2, 10, 0, 0] and m == 10
