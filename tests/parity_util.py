"""Comparison helpers of the parity tests (CPU side, numpy only).

Neighbor structures are compared bit for bit. Floating-point fields are compared element by
element: |gpu - ref| <= rtol * |ref| + atol, with rtol and the absolute floor atol stated per
field by each test (the floor covers values near zero, where a relative bound says nothing).
"""
import numpy as np

EMPTY_64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def written_slot_mask(meta, n_f, fmt, batch_chunks=4096):
    """Boolean mask over the packed words of one SELL32 format: True where a lane wrote a slot
    (slot k of a chunk's lane with k < that lane's count). Chunks of one format occupy
    consecutive [pitch][32] blocks in offset order, so the mask is built block-batch by
    block-batch without per-chunk Python loops."""
    key = "w16" if fmt == 0 else "w32"
    size = meta[key].size
    mask = np.zeros(size, bool)
    chunks = np.nonzero((meta["format"] == fmt) & (meta["pitch"] > 0))[0]
    if chunks.size == 0:
        return mask
    cnt = np.zeros(max(int(chunks.max()) * 32 + 32, n_f), np.int64)
    cnt[:n_f] = meta["counts"][:n_f]
    off = meta["offset"].astype(np.int64)
    pitch = meta["pitch"].astype(np.int64)
    for b0 in range(0, chunks.size, batch_chunks):
        cs = chunks[b0:b0 + batch_chunks]
        lens = pitch[cs] * 32
        start = off[cs]
        # entry -> its chunk; position inside the chunk block -> (slot k, lane)
        which = np.repeat(np.arange(cs.size), lens)
        first = np.repeat(start, lens)
        pos = first + (np.arange(lens.sum()) - np.repeat(np.cumsum(lens) - lens, lens))
        rel = pos - first
        k = rel >> 5
        lane = rel & 31
        mask[pos] = k < cnt[cs[which] * 32 + lane]
    return mask


def assert_neighbor_structures_equal(g, o, n_f, n_b, n_r, what=""):
    """Morton cell IDs, sort permutations, cell tables, all six neighbor row sets and the
    SELL32 encoding (counts, pitch, format, bases, offsets and every written packed word)."""
    for sp, n in ((0, n_f), (1, n_b), (2, n_r)):
        if n == 0:
            continue
        assert np.array_equal(g.cell_ids(sp), o.cell_ids(sp)), f"{what} cell ids {sp}"
        assert np.array_equal(g.permutation(sp), o.permutation(sp)), f"{what} permutation {sp}"
        gu, gs = g.cell_table(sp)
        ou, os_ = o.cell_table(sp)
        assert np.array_equal(gu, ou) and np.array_equal(gs, os_), f"{what} cell table {sp}"
    for lst in range(6):
        go, gi = g.rows(lst)
        oo, oi = o.rows(lst)
        assert np.array_equal(go, oo), f"{what} row offsets {lst}"
        assert np.array_equal(gi, oi), f"{what} rows {lst}: {int((gi != oi).sum()) if gi.size == oi.size else -1} entries differ"
        del gi, oi
    if n_f == 0:
        return
    for lst in range(3):
        gm, om = g.sell32(lst), o.sell32(lst)
        for k in ("counts", "pitch", "format", "base", "offset"):
            assert np.array_equal(gm[k], om[k]), f"{what} sell32 {lst} {k}"
        # second base: only meaningful for Delta16x2 chunks
        d = om["format"] == 0
        assert np.array_equal(gm["base2"][d], om["base2"][d]), f"{what} sell32 {lst} base2"
        assert gm["w16"].size == om["w16"].size and gm["w32"].size == om["w32"].size
        for key, fmt in (("w16", 0), ("w32", 1)):
            mask = written_slot_mask(om, n_f, fmt)
            assert np.array_equal(gm[key][mask], om[key][mask]), f"{what} sell32 {lst} {key}"


def elementwise_errors(a, b, rtol, atol):
    """Per-element error of `a` against the reference `b` and the bound rtol*|b| + atol;
    returns (bad mask, summary dict)."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    err = np.abs(a - b)
    lim = rtol * np.abs(b) + atol
    bad = ~(err <= lim)
    big = np.abs(b) > atol / max(rtol, 1e-30)  # where the relative part dominates the bound
    rel = err[big] / np.abs(b[big]) if big.any() else np.zeros(1)
    summary = dict(n=int(a.size), max_abs=float(err.max()) if a.size else 0.0,
                   max_rel_above_floor=float(rel.max()), p99_rel_above_floor=float(np.quantile(rel, 0.99)),
                   scale=float(np.abs(b).max()) if b.size else 0.0, bad=int(bad.sum()), rtol=rtol, atol=atol)
    return bad, summary


def assert_elementwise(a, b, rtol, atol, what=""):
    bad, s = elementwise_errors(a, b, rtol, atol)
    assert not bad.any(), f"{what}: {s['bad']} of {s['n']} beyond rtol {rtol} + atol {atol:.3e}: {s}"
    return s


def report(name, data):
    """Writes a test's measured errors as JSON into $TSP_TEST_REPORT_DIR when that is set (the
    numbers the stated bounds were set from); does nothing otherwise."""
    import json
    import os
    d = os.environ.get("TSP_TEST_REPORT_DIR")
    if not d:
        return
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, f"{name}.json"), "w") as f:
        json.dump(data, f, indent=1, default=float)
