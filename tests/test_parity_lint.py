"""Race freedom of the red/black half-steps, checked on the CPU.

A half-step updates the pixels of one colour ((x + y) even: black) while
reading pixels of the other colour; the update is race-free only if every
offset a pixel reads its neighbours at has an odd x + y.  The offsets are the
reference's (HPM.cu):
  NESP strips      first site +-5, then 4 more 2 apart (HPM.cu:1252-1345)
  strip extension  shifted 10 per round, 3 rounds (HPM.cu:560-1034)
  NESP polylines   (-5,-6), (6,-5), (5,6), (-6,5), then 7 zig-zag steps of 2
                   along x and y in turn (HPM.cu:1346-1471)
  polyline ext.    shifted (8, 8) per round, outward (HPM.cu:560-1034)
  view priors      the 4 strip neighbours at +-5 (HPM.cu:1553)
  filter           +-1, +-3, +-5 along each axis, (+-2, +-1), (+-1, +-2)
                   (HPM.cu:1782-1870)
and the tiling that maps threads to pixels (hpm_pm.cu half_step_pixel_at) must
reach every pixel of the colour exactly once, for every tile width the
batched form may pick.
"""
import itertools

import pytest


def nesp_offsets():
    out = set()
    strips = [(0, -1), (0, 1), (-1, 0), (1, 0)]
    for (dx, dy), r, i in itertools.product(strips, range(3), range(5)):
        d = 5 + 10 * r + 2 * i
        out.add((dx * d, dy * d))
    # polylines: start, even step, odd step per direction (outward shift 8r)
    polys = [((-5, -6), (-2, 0), (0, -2), (-1, -1)), ((6, -5), (0, -2), (2, 0), (1, -1)),
             ((5, 6), (2, 0), (0, 2), (1, 1)), ((-6, 5), (0, 2), (-2, 0), (-1, 1))]
    for (start, even, odd, out_dir), r in itertools.product(polys, range(3)):
        x, y = start[0] + 8 * r * out_dir[0], start[1] + 8 * r * out_dir[1]
        out.add((x, y))
        for k in range(7):
            step = even if k % 2 == 0 else odd
            x, y = x + step[0], y + step[1]
            out.add((x, y))
    return out


def view_prior_offsets():
    return {(0, -5), (0, 5), (-5, 0), (5, 0)}


def filter_offsets():
    out = set()
    for d in (1, 3, 5):
        out |= {(0, d), (0, -d), (d, 0), (-d, 0)}
    out |= {(sx * 2, sy * 1) for sx in (-1, 1) for sy in (-1, 1)}
    out |= {(sx * 1, sy * 2) for sx in (-1, 1) for sy in (-1, 1)}
    return out


@pytest.mark.parametrize("name,offsets", [("NESP sites and extensions", nesp_offsets()),
                                          ("view priors", view_prior_offsets()),
                                          ("filter", filter_offsets())])
def test_every_neighbour_read_is_the_other_colour(name, offsets):
    bad = [(dx, dy) for dx, dy in offsets if (dx + dy) % 2 == 0]
    assert not bad, f"{name}: offsets of the same colour {bad}"
    assert (0, 0) not in offsets


def _covered(W, rows_cov, ww, color):
    wh = 32 // ww
    gx = (W + 2 * ww - 1) // (2 * ww)
    gy = (rows_cov + 2 * wh - 1) // (2 * wh)
    seen = {}
    for by, bx, wv, lane in itertools.product(range(gy), range(gx), range(2), range(32)):
        py = by * (2 * wh) + wv * wh + lane // ww
        px = bx * (2 * ww) + 2 * (lane % ww) + ((py + color) & 1)
        if px < W and py < rows_cov:
            seen[(px, py)] = seen.get((px, py), 0) + 1
    return seen


@pytest.mark.parametrize("ww", [4, 8, 16])
@pytest.mark.parametrize("W,H", [(40, 30), (37, 65), (64, 64)])
def test_half_step_tiles_reach_every_pixel_of_the_colour_once(ww, W, H):
    rows_cov = min(H, 2 * (((H // 2) + 15) // 16) * 16)  # the reference's grid (HPM.cu:1926)
    for color in (0, 1):
        seen = _covered(W, rows_cov, ww, color)
        want = {(x, y) for x in range(W) for y in range(rows_cov) if (x + y) % 2 == color}
        assert set(seen) == want
        assert max(seen.values()) == 1
