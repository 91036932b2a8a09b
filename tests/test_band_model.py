"""A CPU model of the resident kernel's 2D protocol
(begputhinning_b200/csrc/resident.cu: res_run2d, res_subit2d): an image cut
into bands of rows that each keep `halo` extra rows on both sides, strips of
32 rows skipped while their neighbourhood has been constant for four
subiterations, the bands' iterations in lockstep with a halo exchange after
each, and the two stopping rules (one band: four subiterations without a
deletion; several bands: an iteration without a core deletion in any band).
Deletions use the oracle's rule table, so the model checks the protocol and
its exactness argument, not the device's arithmetic: it must reproduce the
oracle's thinning on every image, and it must fail when the halo is too
thin for an iteration."""
import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, random2d

LONG_AGO = -(1 << 29)


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


def run_band_model(img, bands, halo=4):
    H, W = img.shape
    state = img.copy()  # global buffer (the bands' boundary rows are traded through it)
    cuts = [k * H // bands for k in range(bands + 1)]
    B = []
    for k in range(bands):
        r0, r1 = cuts[k], cuts[k + 1]
        h = halo if bands > 1 else 0
        a, b = max(0, r0 - h), min(H, r1 + h)
        rows = img[a:b].copy()
        ns = (b - a + 31) // 32
        last = np.full(ns, LONG_AGO)
        for s in range(ns):
            if rows[32 * s:32 * s + 32].any():
                last[s] = -1
        B.append(dict(r0=r0, r1=r1, a=a, b=b, rows=rows, last=last, last_any=-1))
    t = 0
    while True:
        for bd in B:
            ns = len(bd["last"])
            act = np.zeros(bd["b"] - bd["a"], bool)
            lc = bd["last"]
            for s in range(ns):
                m = max(lc[s], lc[s - 1] if s > 0 else LONG_AGO, lc[s + 1] if s + 1 < ns else LONG_AGO)
                if m >= t - 4:
                    act[32 * s:32 * s + 32] = True
            new = subit(bd["rows"], t % 4, act)
            ch = new != bd["rows"]
            for s in range(ns):
                if ch[32 * s:32 * s + 32].any():
                    lc[s] = t
            core = ch[bd["r0"] - bd["a"]:bd["r1"] - bd["a"]].any()
            if core:
                bd["last_any"] = t
            bd["rows"] = new
        if bands == 1:
            bd = B[0]
            if t - bd["last_any"] >= 4:
                return bd["rows"], t
        elif t % 4 == 3:
            p = t // 4
            for bd in B:  # boundary core rows -> global
                state[bd["r0"]:bd["r1"]] = bd["rows"][bd["r0"] - bd["a"]:bd["r1"] - bd["a"]]
            if all(bd["last_any"] < 4 * p for bd in B):
                return state, t
            for bd in B:  # halo rows <- neighbours
                old = bd["rows"].copy()
                bd["rows"][:bd["r0"] - bd["a"]] = state[bd["a"]:bd["r0"]]
                bd["rows"][bd["r1"] - bd["a"]:] = state[bd["r1"]:bd["b"]]
                if (old != bd["rows"]).any():
                    for s in range(len(bd["last"])):
                        ga, gb = bd["a"] + 32 * s, bd["a"] + min(32 * s + 32, bd["b"] - bd["a"])
                        if not (ga >= bd["r0"] and gb <= bd["r1"]):
                            bd["last"][s] = t
        t += 1
        assert t < 4000


def _images():
    rng = np.random.default_rng(4)
    return [blobs2d(rng, 230, 90, 40, rmax=12), random2d(rng, 150, 70, 0.6), blobs2d(rng, 97, 64, 12),
            random2d(rng, 64, 40, 0.9)]


@pytest.mark.parametrize("bands", [1, 2, 3, 5])
def test_band_model_matches_oracle(bands):
    for img in _images():
        got, _ = run_band_model(img, bands)
        assert np.array_equal(got, po.thin2d(img)[0]), (img.shape, bands)


def test_band_model_needs_its_halo():
    """With halo rows thinner than one iteration's reach (4 subiterations)
    some image comes out wrong: the model can tell a broken protocol."""
    wrong = 0
    for img in _images():
        got, _ = run_band_model(img, 3, halo=1)
        wrong += not np.array_equal(got, po.thin2d(img)[0])
    assert wrong > 0
