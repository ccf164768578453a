"""The rasterizer restatement in the oracle (lima_oracle.c part C) on known
answers from the reference's formulas (Rasterizer.cu:150-251,
DisplayV2.cpp:13-51): colour and radius tables, the normalisation, the
depth sort and the shaded discs."""
import numpy as np

from oracle import pyoracle as po

F = np.float32


def _one(x, y, z, kind, box):
    return po.render_balls(np.array([[x, y, z]], np.float32), np.array([kind], np.uint8), box)


def test_ball_of_a_solvent_at_the_centre():
    b = _one(2.0, 2.0, 2.0, 6, 4.0)[0]
    assert tuple(b["pos"]) == (0.0, 0.0, 0.0)
    assert b["radius"] == F(0.25) * (F(0.08) / (F(1) + F(2.0) * F(0.001)))
    assert tuple(b["color"]) == (0x03, 0xA9, 0xF4) and b["disable"] == 0


def test_types_colours_and_radii():
    table = {1: ((0xE0, 0x20, 0x20), 0.12), 2: ((0x30, 0x10, 0x90), 0.1), 3: ((0xFC, 0xF7, 0x5E), 0.15),
             4: ((0x2E, 0x8B, 0x57), 0.1), 5: ((0xF1, 0xF1, 0xF1), 0.04), 6: ((0x03, 0xA9, 0xF4), 0.08)}
    for k, (color, r) in table.items():
        b = _one(1.0, 0.0, 1.0, k, 2.0)[0]
        assert tuple(b["color"]) == color and b["radius"] == F(0.25) * F(r) and b["disable"] == 0
        assert tuple(b["pos"]) == (F(0.0), F(-0.9), F(0.0))


def test_empty_slot_is_disabled_at_the_origin():
    b = _one(1.5, 1.5, 1.5, 0, 3.0)[0]                    # NONE: the position is not used
    assert b["disable"] == 1 and tuple(b["pos"]) == (F(-0.9),) * 3
    assert tuple(b["color"]) == (0xF2, 0xE5, 0xD9) and b["radius"] == F(0.25)


def test_depth_sort_is_ascending_with_ties_in_descending_slot_order():
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 5, (500, 3)).astype(np.float32)
    pos[100:110, 1] = pos[50, 1]                           # 11 balls at one depth
    pos[100:110, 0] = np.arange(10, dtype=np.float32) * 0.1 + 0.05
    kind = np.full(500, 6, np.uint8)
    b = po.render_balls(pos, kind, 5.0)
    assert (np.diff(b["pos"][:, 1]) >= 0).all()
    y50 = F((np.float64(pos[50, 1]) / 5.0 - 0.5) * 1.8)
    tied = b[b["pos"][:, 1] == y50]
    assert len(tied) == 11
    # equal depths in descending slot order (the reference's merge takes the right
    # half's ball on a tie): slots 109..100, then slot 50
    expect_x = [F((np.float64(pos[i, 0]) / 5.0 - 0.5) * 1.8) for i in list(range(109, 99, -1)) + [50]]
    assert tied["pos"][:, 0].tolist() == expect_x


def test_image_of_one_ball():
    b = _one(2.0, 2.0, 2.0, 6, 4.0)
    n = 1001
    img = po.render_image(b, n, n)
    c = n // 2
    # centre pixel: light 0.5 -> floor(colour * 0.5)
    assert tuple(img[c, c]) == (0x03 // 2, 0xA9 // 2, 0xF4 // 2)
    assert not img[0, 0].any() and not img[-1, -1].any()
    R = float(b[0]["radius"]) * n / 2                      # pixels
    lit = img.any(2)
    assert abs(lit.sum() - np.pi * R * R) < 2 * np.pi * R + 4
    # brighter towards the top of the disc (light 0.5 + 0.5 dy / R)
    col = img[:, c, 1].astype(int)
    assert col[c - 5] > col[c] > col[c + 5]
    assert col[c - 9] > 0.9 * 0xA9 and col[c + 9] < 0.1 * 0xA9


def test_front_ball_covers_the_back_one():
    pos = np.array([[2.0, 3.0, 2.0], [2.0, 1.0, 2.0]], np.float32)   # the second is in front (smaller y)
    b = po.render_balls(pos, np.array([1, 2], np.uint8), 4.0)          # O (larger) behind, C in front
    assert tuple(b[0]["color"]) == (0x30, 0x10, 0x90)
    img = po.render_image(b, 640, 640)
    assert img[319, 320, 2] > 2 * img[319, 320, 0]                    # blue C over red O
    # in the ring only the larger back ball reaches, the back ball's colour shows
    r_front, r_back = float(b[0]["radius"]) * 320, float(b[1]["radius"]) * 320
    x = 320 + int(round((r_front + r_back) / 2))
    assert r_front < r_back and img[319, x, 0] > 2 * img[319, x, 2]
