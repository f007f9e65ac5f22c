"""CPU emulation of the column-panel product (panel.cu / panel.cuh), no GPU.

Restates, in numpy, the builder of the panel split (long rows by length,
segments (panel, long row), the greedy chunking of every panel's segments
into records of at most 256 entries and 128 segments with no segment split,
the record's slot layouts and start bits) and the kernels' arithmetic (each
lane's segmented prefix over its 8 entries, a segment as the sum of one
piece per lane it touches, the finish as the sum over panels in order).
On random structures — empty rows, rows crossing every panel, rows shorter
than the threshold, narrow panels, chunks closed by the segment cap — every
long row must receive exactly the sum of its entries and every short row
must be left to the tiled product.  The same records and arithmetic, laid out
for the hot part of Aᵀy (the longest rows of A, one segment per column of a
panel), plus the tiled rest must give every column of Aᵀy exactly.  Products are small integers, so the sums
are exact whatever the order.
"""
import numpy as np
import pytest

IPT = 8                 # entries per lane
ENT = 32 * IPT          # entries per record
SEG_CAP = 128           # segments per record


def val_slot(q):
    return (((q % IPT) // 4) * 32 + q // IPT) * 4 + (q % 4)


def test_val_slot_layout():
    slots = [val_slot(q) for q in range(ENT)]
    assert sorted(slots) == list(range(ENT))          # a permutation of the record's value slots
    # lane l's chunk k (entries 8l + 4k .. 8l + 4k + 3) is the 16-byte unit k * 32 + l
    for lane in range(32):
        for k in range(IPT // 4):
            unit = {val_slot(lane * IPT + 4 * k + t) // 4 for t in range(4)}
            assert unit == {k * 32 + lane}


def build(rp, ci, n, panels_max, thr):
    """The split's host-visible structure: widths, long rows, records."""
    m = len(rp) - 1
    width = -(-n // panels_max)
    width = (width + 3) // 4 * 4
    panels = -(-n // width)
    lens = np.diff(rp)
    long_rows = np.nonzero(lens >= thr)[0]
    L = len(long_rows)
    # segments: entries of long row r with a column in panel p, CSR order
    seg = [[[] for _ in range(L)] for _ in range(panels)]
    for r_idx, i in enumerate(long_rows):
        for k in range(rp[i], rp[i + 1]):
            p = ci[k] // width
            seg[p][r_idx].append(k)
    assert max((len(s) for ps in seg for s in ps), default=0) <= ENT
    records = []   # (panel, first segment, [segment entry lists])
    for p in range(panels):
        r = 0
        while r < L:
            first, ent = r, 0
            while r < L and r - first < SEG_CAP and ent + len(seg[p][r]) <= ENT:
                ent += len(seg[p][r])
                r += 1
            records.append((p, first, [seg[p][q] for q in range(first, r)]))
    return width, panels, long_rows, records


def emulate(rp, ci, val, x, n, panels_max, thr):
    width, panels, long_rows, records = build(rp, ci, n, panels_max, thr)
    L = len(long_rows)
    part = np.full((panels, L), np.nan)
    for p, first, segs in records:
        entries = [k for s in segs for k in s]
        nent = len(entries)
        assert nent <= ENT and len(segs) <= SEG_CAP
        off = np.zeros(len(segs) + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in segs])
        starts = np.zeros(ENT + 1, bool)
        for a, b in zip(off[:-1], off[1:]):
            if a < b:
                starts[a] = True
        if nent < ENT:
            starts[nent] = True                      # padding starts a run no segment reads
        cols = np.zeros(ENT, np.int64)
        vals = np.zeros(ENT)
        cols[:nent] = ci[entries] - p * width
        assert (cols < min(width, n - p * width)).all()
        vals[:nent] = val[entries]
        xs = x[p * width: p * width + width]
        prod = vals * xs[cols]
        # every lane's segmented prefix, stored at the value slots
        pre = np.zeros(ENT)
        for lane in range(32):
            acc = 0.0
            for j in range(IPT):
                q = lane * IPT + j
                acc = prod[q] + (0.0 if starts[q] else acc)
                pre[val_slot(q)] = acc
        for s, (a, b) in enumerate(zip(off[:-1], off[1:])):
            total = 0.0
            if a < b:
                e = min((a | (IPT - 1)) + 1, b)
                total = pre[val_slot(e - 1)]
                while e < b:
                    total += pre[val_slot(min(e + IPT, b) - 1)]
                    e += IPT
            part[p, first + s] = total
    assert not np.isnan(part).any()                  # every (panel, long row) written once
    y = np.full(len(rp) - 1, np.nan)
    y[long_rows] = part.sum(axis=0)
    return y, long_rows


def _csr(m, n, rng, lengths):
    cols = [np.sort(rng.choice(n, size=int(k), replace=False)) for k in lengths]
    rp = np.zeros(m + 1, np.int64)
    rp[1:] = np.cumsum(lengths)
    ci = np.concatenate(cols).astype(np.int64) if m else np.zeros(0, np.int64)
    val = rng.integers(-3, 4, size=ci.size).astype(np.float64)
    return rp, ci, val


@pytest.mark.parametrize("seed,m,n,panels,thr", [
    (0, 400, 3000, 16, 8),       # mixed rows, many crossing lanes
    (1, 300, 100, 148, 2),       # fewer columns than SMs: 25 narrow panels, nearly every row long
    (2, 200, 5000, 16, 40),      # wide panels, long segments spanning lanes
    (3, 600, 800, 32, 1),        # every non-empty row long: empty segments close chunks at the cap
])
def test_panel_split_sums(seed, m, n, panels, thr):
    rng = np.random.default_rng(seed)
    lengths = np.minimum(rng.zipf(1.5, size=m), n // 2)
    lengths[rng.random(m) < 0.1] = 0                  # empty rows
    rp, ci, val = _csr(m, n, rng, lengths)
    x = rng.integers(-4, 5, size=n).astype(np.float64)
    y, long_rows = emulate(rp, ci, val, x, n, panels, thr)
    ref = np.array([val[rp[i]:rp[i + 1]] @ x[ci[rp[i]:rp[i + 1]]] for i in range(m)])
    assert np.array_equal(y[long_rows], ref[long_rows])
    short = np.setdiff1d(np.arange(m), long_rows)
    assert np.isnan(y[short]).all()                   # left to the tiled product
    assert set(long_rows) == set(np.nonzero(lengths >= thr)[0])


def test_segment_cap_closes_chunks():
    # 1,000 long rows with one entry each in panel 0 and none elsewhere:
    # the records of panel 0 hold 128 segments each, the other panels' records
    # hold 128 empty segments each.
    m, n = 1000, 64
    rp = np.arange(m + 1, dtype=np.int64)
    ci = np.zeros(m, np.int64)
    _, panels, long_rows, records = build(rp, ci, n, 16, 1)
    assert len(long_rows) == m
    for p in range(panels):
        mine = [r for r in records if r[0] == p]
        assert len(mine) == -(-m // SEG_CAP)
        assert all(len(r[2]) == SEG_CAP for r in mine[:-1])


# ---------------------------------------------------------------------------
# The hot part of Aᵀy (build_panel_hot): the longest rows of A, their y held by
# every block, one segment per column of the block's panel in column order.
# ---------------------------------------------------------------------------

HOT_MIN_LEN = 32


def chunk_segments(segs):
    """Greedy chunking of one panel's segments (lists of entries)."""
    out, r = [], 0
    while r < len(segs):
        first, ent = r, 0
        while r < len(segs) and r - first < SEG_CAP and ent + len(segs[r]) <= ENT:
            ent += len(segs[r])
            r += 1
        out.append((first, segs[first:r]))
    return out


def run_records(records, vec, nseg):
    """The kernel's arithmetic over (first, [[(gather index, value), ...], ...])
    records: in-lane segmented prefixes, pieces per lane, segment sums."""
    out = np.full(nseg, np.nan)
    for first, segs in records:
        entries = [e for s in segs for e in s]
        nent = len(entries)
        off = np.zeros(len(segs) + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in segs])
        starts = np.zeros(ENT + 1, bool)
        for a, b in zip(off[:-1], off[1:]):
            if a < b:
                starts[a] = True
        if nent < ENT:
            starts[nent] = True
        prod = np.zeros(ENT)
        for q, (g, v) in enumerate(entries):
            prod[q] = v * vec[g]
        pre = np.zeros(ENT)
        for lane in range(32):
            acc = 0.0
            for j in range(IPT):
                q = lane * IPT + j
                acc = prod[q] + (0.0 if starts[q] else acc)
                pre[val_slot(q)] = acc
        for s, (a, b) in enumerate(zip(off[:-1], off[1:])):
            total = 0.0
            if a < b:
                e = min((a | (IPT - 1)) + 1, b)
                total = pre[val_slot(e - 1)]
                while e < b:
                    total += pre[val_slot(min(e + IPT, b) - 1)]
                    e += IPT
            out[first + s] = total
    return out


def emulate_hot(rp, ci, val, y, n, panels_max, vmax):
    m = len(rp) - 1
    lens = np.diff(rp)
    thr = HOT_MIN_LEN
    if m > vmax:
        thr = max(thr, int(np.sort(lens)[::-1][vmax]) + 1)
    hot = lens >= thr
    hidx = np.cumsum(hot) - 1
    hot_rows = np.nonzero(hot)[0]
    assert len(hot_rows) <= vmax
    width = (-(-n // panels_max) + 3) // 4 * 4
    panels = -(-n // width)
    # Aᵀ in column order, rows increasing within a column (the stored transpose)
    cols = [[] for _ in range(panels * width)]
    rest = np.zeros(n)
    for i in range(m):
        for k in range(rp[i], rp[i + 1]):
            if hot[i]:
                cols[ci[k]].append((int(hidx[i]), val[k]))
            else:
                rest[ci[k]] += val[k] * y[i]
    assert max(len(c) for c in cols) <= ENT
    vec = y[hot_rows]
    part = np.full(panels * width, np.nan)
    for p in range(panels):
        segs = cols[p * width:(p + 1) * width]
        recs = chunk_segments(segs)
        assert sum(len(s) for _, s in recs) == width
        part[p * width:(p + 1) * width] = run_records(recs, vec, width)
    assert not np.isnan(part).any()
    return part[:n] + rest, len(hot_rows)


@pytest.mark.parametrize("seed,m,n,panels,vmax,a", [
    (0, 500, 2000, 16, 40, 1.4),     # more long rows than the shared memory holds: the longest 40 or fewer
    (1, 300, 700, 148, 1000, 1.4),   # narrow panels, every row of >= 32 entries hot
    (2, 400, 5000, 8, 7, 1.8),       # few hot rows, wide panels, many empty column segments
])
def test_hot_part_of_transpose_product(seed, m, n, panels, vmax, a):
    rng = np.random.default_rng(seed)
    lengths = np.minimum(rng.zipf(a, size=m), n // 4)
    rp, ci, val = _csr(m, n, rng, lengths)
    y = rng.integers(-4, 5, size=m).astype(np.float64)
    aty, nhot = emulate_hot(rp, ci, val, y, n, panels, vmax)
    ref = np.zeros(n)
    for i in range(m):
        ref[ci[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]] * y[i]
    assert np.array_equal(aty, ref)
    assert 0 < nhot <= vmax
