"""A CPU model of the resident kernel's 2D protocol
(begputhinning_b200/csrc/resident.cu: res_run2d, res_pass2d): an image cut
into bands of rows that each keep `halo` extra rows on both sides; a pass is
one iteration (N, S, E, W) computed per unit of 24 rows x 8 words on a
register tile with 4 halo rows and one halo word on either side (56 rows in
the two-rows-per-lane build); a unit is
processed in the next pass when it changed or a neighbour changed within 4
pixels of their common border (border bands); the bands run passes in
lockstep with a halo exchange after every fourth pass (16 halo rows: four
passes move wrong values in from a band's edge by at most 16 rows), and stop
after an exchange pass without a core deletion in any band.
Deletions use the oracle's rule table, so the model checks the protocol and
its exactness argument, not the device's arithmetic: it must reproduce the
oracle's thinning on every image, and it must fail when the halo is too
thin for an iteration."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, random2d



def _tables():
    # deletable[dir][n] for the 8-neighbourhood number n (bit i = neighbour i: N, NE, E, SE, S, SW, W, NW)
    out = []
    for d in range(4):
        words = po.rule_table(2, d)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").astype(bool)
        out.append(bits[:256])
    return out


TABLES = _tables()
OFFS = [(-1, 0), (-1, 1), (0, 1), (1, 1), (1, 0), (1, -1), (0, -1), (-1, -1)]


def subit(rows, d, active_rows):
    """One synchronous subiteration on the band's rows (zero outside); only
    rows flagged active may change.  Returns the new rows."""
    h, w = rows.shape
    p = np.pad(rows, 1)
    idx = np.zeros((h, w), np.int64)
    for i, (dy, dx) in enumerate(OFFS):
        idx |= p[1 + dy:1 + dy + h, 1 + dx:1 + dx + w].astype(np.int64) << i
    dele = TABLES[d][idx] & (rows != 0) & active_rows[:, None]
    return np.where(dele, 0, rows).astype(np.uint8)


def run_tile(rows, r0, r1, c0, c1):
    """The kernel's register tile: rows r0-4 .. r1+4 (zero outside the band)
    by pixels c0-32 .. c1+32 (zero outside), four subiterations N, S, E, W,
    only rows r0..r1 and pixels c0..c1 kept."""
    H, W = rows.shape
    t = np.zeros((r1 - r0 + 8, c1 - c0 + 64), np.uint8)
    ya, yb, xa, xb = max(0, r0 - 4), min(H, r1 + 4), max(0, c0 - 32), min(W, c1 + 32)
    t[ya - (r0 - 4):yb - (r0 - 4), xa - (c0 - 32):xb - (c0 - 32)] = rows[ya:yb, xa:xb]
    full = np.ones(t.shape[0], bool)
    for d in range(4):
        t = subit(t, d, full)
    return t[4:4 + (r1 - r0), 32:32 + (c1 - c0)]


def run_band_model(img, bands, halo=16, unit_rows=24, unit_px=8 * 32, every=4):
    H, W = img.shape
    state = img.copy()  # global buffer (the bands' boundary rows are traded through it)
    cuts = [k * H // bands for k in range(bands + 1)]
    B = []
    nch = (W + unit_px - 1) // unit_px
    for k in range(bands):
        r0, r1 = cuts[k], cuts[k + 1]
        h = halo if bands > 1 else 0
        a, b = max(0, r0 - h), min(H, r1 + h)
        rows = img[a:b].copy()
        ns = (b - a + unit_rows - 1) // unit_rows
        until = np.full((ns, nch), -1)
        for s in range(ns):
            for c in range(nch):
                if rows[unit_rows * s:unit_rows * (s + 1), unit_px * c:unit_px * (c + 1)].any():
                    until[s, c] = 0
        B.append(dict(r0=r0, r1=r1, a=a, b=b, rows=rows, until=until))
    for q in range(4000):
        any_core = False
        for bd in B:
            rows, until = bd["rows"], bd["until"]
            ns = until.shape[0]
            new = rows.copy()
            for s in range(ns):
                for c in range(nch):
                    if until[s, c] < q:
                        continue
                    y0, y1 = unit_rows * s, min(unit_rows * (s + 1), rows.shape[0])
                    x0, x1 = unit_px * c, min(unit_px * (c + 1), W)
                    out = run_tile(rows, y0, y1, x0, x1)
                    d = out != rows[y0:y1, x0:x1]
                    if d.any():
                        # border bands: a neighbour is activated only when a
                        # change lies within 4 pixels of its side
                        band_r = {-1: d[:4].any(axis=0), 0: d.any(axis=0), 1: d[unit_rows - 4:].any(axis=0)}
                        for dy in (-1, 0, 1):
                            if dy == 1 and y1 - y0 < unit_rows:
                                continue  # last unit of the band: no unit below
                            rr = band_r[dy]
                            for dx in (-1, 0, 1):
                                hit = rr[:4].any() if dx < 0 else rr[-4:].any() if dx > 0 else rr.any()
                                ns, nc = s + dy, c + dx
                                if hit and 0 <= ns < until.shape[0] and 0 <= nc < nch:
                                    until[ns, nc] = q + 1
                        ga, gb = bd["a"] + y0, bd["a"] + y1
                        ch = d.any(axis=1)
                        ys = np.arange(ga, gb)[ch]
                        any_core |= bool(((ys >= bd["r0"]) & (ys < bd["r1"])).any())
                    new[y0:y1, x0:x1] = out
            bd["rows"] = new
        if bands == 1:
            if not any_core:
                return B[0]["rows"], q + 1
            continue
        if q % every != every - 1:
            continue  # the bands meet after every `every` passes
        for bd in B:  # core rows -> global
            state[bd["r0"]:bd["r1"]] = bd["rows"][bd["r0"] - bd["a"]:bd["r1"] - bd["a"]]
        if not any_core:
            return state, q + 1
        for bd in B:  # halo rows <- neighbours
            old = bd["rows"].copy()
            bd["rows"][:bd["r0"] - bd["a"]] = state[bd["a"]:bd["r0"]]
            bd["rows"][bd["r1"] - bd["a"]:] = state[bd["r1"]:bd["b"]]
            if (old != bd["rows"]).any():
                for st in range(bd["until"].shape[0]):
                    ga, gb = bd["a"] + unit_rows * (st - 1), bd["a"] + unit_rows * (st + 2)
                    if ga < bd["r0"] or gb > bd["r1"]:
                        bd["until"][st, :] = q + 1
    raise AssertionError("no fixed point")


def _images():
    rng = np.random.default_rng(4)
    return [blobs2d(rng, 230, 90, 40, rmax=12), random2d(rng, 150, 70, 0.6), blobs2d(rng, 97, 64, 12),
            random2d(rng, 64, 40, 0.9), blobs2d(rng, 70, 900, 60, rmax=12)]


@pytest.mark.parametrize("unit_rows", [24, 56])
@pytest.mark.parametrize("halo,every", [(16, 4), (8, 2)])
@pytest.mark.parametrize("bands", [1, 2, 3, 5])
def test_band_model_matches_oracle(bands, halo, every, unit_rows):
    for img in _images():
        got, _ = run_band_model(img, bands, halo=halo, every=every, unit_rows=unit_rows)
        assert np.array_equal(got, po.thin2d(img)[0]), (img.shape, bands)


def test_band_model_exchange_every_pass():
    """The earlier protocol: 4 halo rows, an exchange after every pass."""
    for img in _images():
        got, _ = run_band_model(img, 3, halo=4, every=1)
        assert np.array_equal(got, po.thin2d(img)[0]), img.shape


@pytest.mark.parametrize("halo,every", [(1, 1), (3, 2)])
def test_band_model_needs_its_halo(halo, every):
    """With halo rows thinner than the reach of the passes between two
    exchanges (4 rows per pass) some image comes out wrong: the model can
    tell a broken protocol."""
    wrong = 0
    rng = np.random.default_rng(11)
    for img in _images() + [random2d(rng, 160, 90, 0.8), blobs2d(rng, 240, 100, 30, rmax=20)]:
        for bands in (2, 3):
            got, _ = run_band_model(img, bands, halo=halo, every=every)
            wrong += not np.array_equal(got, po.thin2d(img)[0])
    assert wrong > 0
