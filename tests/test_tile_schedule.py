"""CPU emulation of the SpMV schedule (spmv_warp_kernel + spmv_fixup_kernel),
no GPU needed.

Restates, in numpy, the tiled-format builder of csr_device.cu (row
compaction, row-start bitmap, per-tile {first_row, tail_continues}, the
crossing-row list) and the kernels' per-lane logic (row ids from popcounts,
row-end bits, segmented warp scan, per-tile carries, fixup in tile order).
It checks on many random structures — empty rows, rows spanning many tiles,
rows starting exactly on tile boundaries, padding — that every row receives
exactly the sum of its entries, exactly once.  Products are small integers so
sums are exact.
"""
import numpy as np
import pytest

TILE = 512   # 32 lanes x 16 entries, the format unit of the library


def build_format(rp, T):
    m = len(rp) - 1
    nnz = int(rp[-1])
    nt = (nnz + T - 1) // T if nnz else 0
    pad = nt * T
    ne = np.diff(rp) > 0
    rows_c = int(ne.sum())
    row_map = np.nonzero(ne)[0]
    rp_c = np.concatenate([rp[:-1][ne], [nnz, pad]]).astype(np.int64)
    flags = np.zeros(max(pad, 1), np.int64)
    flags[rp_c[:rows_c]] = 1
    if nnz < pad:
        flags[nnz] = 1

    def row_of(q):
        return int(np.searchsorted(rp_c[:rows_c + 1], q, side="right") - 1)

    meta, cross = [], []
    for t in range(nt):
        base, last = t * T, t * T + T - 1
        fr = row_of(base)
        tr = row_of(last)
        tend = int(rp_c[tr + 1])
        cont = int(tr < rows_c and tend > last + 1)
        meta.append((fr, cont))
        if cont and rp_c[tr] >= base:
            cross.append((int(row_map[tr]), t, (tend - 1) // T - t + 1))
    return dict(nt=nt, rows_c=rows_c, row_map=row_map, flags=flags, meta=meta, cross=cross)


def emulate(rp, prod, T=TILE, IPT=8):
    F = build_format(rp, T)
    m = len(rp) - 1
    nt, rows_c, flags, meta = F["nt"], F["rows_c"], F["flags"], F["meta"]
    lanes = T // IPT
    out = {}
    carry = {}

    def emit(row_c, v):
        if row_c >= rows_c:
            return
        r = int(F["row_map"][row_c])
        assert r not in out, f"row {r} emitted twice"
        out[r] = v

    padded = np.zeros(nt * T, np.int64)
    padded[:len(prod)] = prod
    for t in range(nt):
        fr, cont = meta[t]
        fl = flags[t * T:(t + 1) * T]
        pr = padded[t * T:(t + 1) * T]
        s0 = int(fl[0])
        # staged finished rows: meta.x + skip .. , n_fin of them (kernel: base / n_fin)
        ends_total = int(fl.sum()) - s0 + (0 if cont else 1)
        skip = 1 if (s0 == 0 and ends_total > 0) else 0
        base = fr + skip
        n_fin = min(ends_total - skip, rows_c - base)
        fin = [None] * T

        def stage(row_c, v):
            k = row_c - base
            assert 0 <= k < T, (k, T)
            assert fin[k] is None, "staged twice"
            fin[k] = v

        st = []
        for lane in range(lanes):
            q0 = lane * IPT
            bits = fl[q0:q0 + IPT]
            nxt = (0 if cont else 1) if lane == lanes - 1 else fl[q0 + IPT]
            ends = list(bits[1:]) + [nxt]
            row0 = fr + int(fl[:q0].sum()) + int(bits[0]) - s0
            head_before = bits[0] == 0
            acc, cur, nemit, head_pending, head_acc = 0, row0, 0, False, 0
            for j in range(IPT):
                acc += int(pr[q0 + j])
                if ends[j]:
                    if nemit == 0 and head_before:
                        head_acc, head_pending = acc, True
                    else:
                        stage(cur, acc)
                    nemit += 1
                    cur += 1
                    acc = 0
            st.append(dict(f=int(nemit > 0), acc=acc, row0=row0, cur=cur, nemit=nemit,
                           head_pending=head_pending, head_acc=head_acc))
        # inclusive segmented scan of (f, v); carry_in = inclusive value of the previous lane
        incl, v = [], 0
        for s in st:
            v = s["acc"] if s["f"] else v + s["acc"]
            incl.append(v)
        for lane, s in enumerate(st):
            carry_in = incl[lane - 1] if lane > 0 else 0
            if s["head_pending"]:
                tot = s["head_acc"] + carry_in
                if s["row0"] == fr and s0 == 0:
                    carry[(t, 0)] = tot
                else:
                    stage(s["row0"], tot)
            if lane == lanes - 1 and cont:
                tot = s["acc"] if s["nemit"] > 0 else carry_in + s["acc"]
                if s["cur"] == fr and s0 == 0:
                    carry[(t, 0)] = tot
                else:
                    carry[(t, 1)] = tot
        # converged epilogue over the staged rows
        for k in range(max(n_fin, 0)):
            assert fin[k] is not None, (t, k, n_fin)
            emit(base + k, fin[k])
        # only the virtual padding row may be staged beyond n_fin
        for k in range(max(n_fin, 0), T):
            assert fin[k] is None or base + k >= rows_c
    # fixup: crossing rows in tile order, then empty rows
    for row, t0, cnt in F["cross"]:
        s = carry[(t0, 1)]
        for tt in range(t0 + 1, t0 + cnt):
            s += carry[(tt, 0)]
        assert row not in out
        out[row] = s
    for r in range(m):
        if rp[r + 1] == rp[r]:
            assert r not in out
            out[r] = 0
    return out


def check(rp, rng, T=TILE, IPT=8):
    nnz = int(rp[-1])
    prod = rng.integers(-3, 4, size=nnz)
    out = emulate(np.asarray(rp, np.int64), prod, T=T, IPT=IPT)
    m = len(rp) - 1
    assert sorted(out) == list(range(m))
    for r in range(m):
        assert out[r] == int(prod[rp[r]:rp[r + 1]].sum()), r


@pytest.mark.parametrize("mode", range(6))
def test_schedule_random_structures(mode):
    rng = np.random.default_rng(100 + mode)
    T = 64   # small tiles exercise many boundaries per case
    for trial in range(250):
        m = int(rng.integers(1, 50))
        if mode == 0:
            L = rng.integers(0, 5, m)
        elif mode == 1:
            L = rng.integers(0, 200, m)
        elif mode == 2:
            L = rng.choice([0, 1, 63, 64, 65, 128, 8, 7], m)
        elif mode == 3:
            L = (rng.random(m) < 0.5) * rng.integers(0, 300, m)
        elif mode == 4:
            L = rng.choice([64, 128, 192], m)           # rows aligned to tiles
        else:
            L = np.where(rng.random(m) < 0.1, rng.integers(300, 700, m), rng.integers(0, 3, m))
        rp = np.zeros(m + 1, np.int64)
        rp[1:] = np.cumsum(L)
        if rp[-1] == 0:
            continue   # nnz == 0: every row goes through the empty-row pass
        check(rp, rng, T=T)


def test_schedule_library_tile_size():
    rng = np.random.default_rng(7)
    L = np.concatenate([rng.integers(0, 60, 300), [TILE * 3 + 5, TILE, 0, 0, 2 * TILE - 1],
                        rng.integers(0, 9, 200)])
    rp = np.zeros(len(L) + 1, np.int64)
    rp[1:] = np.cumsum(L)
    check(rp, rng, T=TILE, IPT=16)


# ---------------------------------------------------------------------------
# The allocation-free product (noalloc.cu): block merge-path over a plain CSR,
# rows found by binary search, crossing rows finished by a fixup pass.
# ---------------------------------------------------------------------------
def emulate_noalloc(rp, prod, T=64, IPT=8):
    m = len(rp) - 1
    nnz = int(rp[-1])
    nt = (nnz + T - 1) // T
    pad = nt * T

    def rp_at(r):
        return int(rp[r]) if r <= m else pad

    def row_holding(q):
        lo, hi = 0, m
        while lo < hi:
            mid = (lo + hi + 1) >> 1
            if rp[mid] <= q:
                lo = mid
            else:
                hi = mid - 1
        return lo

    y = {}
    carry = {}
    B = T // IPT
    padded = np.zeros(pad, np.int64)
    padded[:nnz] = prod

    def put(r, v):
        assert 0 <= r < m and r not in y, r
        y[r] = v

    for t in range(nt):
        tile_base, tile_end = t * T, t * T + T
        r_lo = 0 if t == 0 else row_holding(tile_base)
        r_hi = m if t == nt - 1 else row_holding(tile_end)
        lanes = []
        for tid in range(B):
            k0, k1 = tile_base + tid * IPT, tile_base + tid * IPT + IPT
            lo, hi = r_lo, r_hi
            while lo < hi:
                mid = (lo + hi) >> 1
                if rp_at(mid + 1) > k0:
                    hi = mid
                else:
                    lo = mid + 1
            r = 0 if (t == 0 and tid == 0) else lo
            st = dict(acc=0, nemit=0, head_row=-1, head_acc=0)

            def finish(row):
                if st["nemit"] == 0 and rp_at(row) < k0:
                    st["head_row"], st["head_acc"] = row, st["acc"]
                else:
                    put(row, st["acc"])
                st["nemit"] += 1
                st["acc"] = 0

            for j in range(IPT):
                while r < m and r <= r_hi and rp_at(r + 1) <= k0 + j:
                    finish(r)
                    r += 1
                st["acc"] += int(padded[k0 + j])
            while r < m and r <= r_hi and rp_at(r + 1) <= k1:
                finish(r)
                r += 1
            lanes.append((r, st["acc"], st))
        # segmented scan by tail row; exclusive value per lane
        incl = []
        for i, (krow, kval, _) in enumerate(lanes):
            if i > 0 and incl[-1][0] == krow:
                incl.append((krow, incl[-1][1] + kval))
            else:
                incl.append((krow, kval))
        for i, (krow, kval, st) in enumerate(lanes):
            erow, ev = incl[i - 1] if i > 0 else (-1, 0)
            if st["head_row"] >= 0:
                tot = st["head_acc"] + (ev if erow == st["head_row"] else 0)
                if rp_at(st["head_row"]) >= tile_base:
                    put(st["head_row"], tot)
                else:
                    carry[2 * t] = tot
            if i == B - 1 and krow < m and rp_at(krow) < tile_end and rp_at(krow + 1) > tile_end:
                carry[2 * t + (1 if rp_at(krow) >= tile_base else 0)] = incl[i][1]
    for t in range(nt - 1):
        R = row_holding(t * T + T - 1)
        if R >= m:
            continue
        start, end = rp_at(R), rp_at(R + 1)
        if start < t * T or end <= t * T + T:
            continue
        s = carry[2 * t + 1]
        for tt in range(t + 1, (end - 1) // T + 1):
            s += carry[2 * tt]
        put(R, s)
    return y


@pytest.mark.parametrize("mode", range(4))
def test_noalloc_schedule_random_structures(mode):
    rng = np.random.default_rng(500 + mode)
    for trial in range(200):
        m = int(rng.integers(1, 50))
        if mode == 0:
            L = rng.integers(0, 5, m)
        elif mode == 1:
            L = rng.integers(0, 200, m)
        elif mode == 2:
            L = rng.choice([0, 1, 63, 64, 65, 128, 8, 7], m)
        else:
            L = np.where(rng.random(m) < 0.1, rng.integers(300, 700, m), rng.integers(0, 3, m))
        rp = np.zeros(m + 1, np.int64)
        rp[1:] = np.cumsum(L)
        if rp[-1] == 0:
            continue
        prod = rng.integers(-3, 4, size=int(rp[-1]))
        y = emulate_noalloc(rp, prod)
        for r in range(m):
            expect = int(prod[rp[r]:rp[r + 1]].sum())
            assert r in y, (trial, r)          # every row is written, empty rows with 0
            assert y[r] == expect, (trial, r)


# ---- integer transformations inside the tile loop ---------------------------
# The kernel computes two warp-level integer results with ballots instead of
# shuffles, and reads its entries through a lane-interleaved record layout.
# These restate both forms and check that they agree exactly.

IPT = 16


def tile_slot(q):
    """Slot of tile-local entry q in a record (spmv.cuh tile_slot): chunk k of
    lane l (entries 16l + 4k .. 16l + 4k + 3) at chunk index k*32 + l."""
    return (((q % IPT) // 4) * 32 + q // IPT) * 4 + (q % 4)


def test_tile_slot_is_a_permutation_with_contiguous_warp_chunks():
    slots = [tile_slot(q) for q in range(TILE)]
    assert sorted(slots) == list(range(TILE))
    for k in range(IPT // 4):                      # chunk read k of the warp
        starts = [tile_slot(16 * lane + 4 * k) for lane in range(32)]
        assert starts == list(range(k * 128, k * 128 + 128, 4))   # 512 contiguous bytes
        for lane in range(32):                     # each chunk holds 4 consecutive entries
            assert [tile_slot(16 * lane + 4 * k + e) for e in range(4)] == list(range(starts[lane], starts[lane] + 4))


def test_ballot_prefix_equals_shuffle_scan():
    """Exclusive prefix and total of per-lane row-start counts (0..16): five
    bit-plane ballots against the inclusive shuffle scan it replaced."""
    rng = np.random.default_rng(5)
    for _ in range(2000):
        cnt = rng.integers(0, IPT + 1, 32)
        incl = np.cumsum(cnt)                                  # shuffle scan
        planes = [sum(1 << l for l in range(32) if (cnt[l] >> b) & 1) for b in range(5)]
        for lane in range(32):
            below = (1 << lane) - 1
            excl = sum(bin(p & below).count("1") << b for b, p in enumerate(planes))
            assert excl == incl[lane] - cnt[lane]
        assert sum(bin(p).count("1") << b for b, p in enumerate(planes)) == incl[-1]


def test_ballot_row_end_windows_equal_flag_shuffles():
    """Segmented scan: at distance d, lane i adds lane i-d's partial only when
    no lane in (i-d, i] ended a row.  The window test on one ballot of the row
    ends must equal the OR-propagated flags of the shuffle form it replaced,
    step for step, and so produce the same sums."""
    rng = np.random.default_rng(6)
    for _ in range(2000):
        ended = rng.random(32) < rng.random()
        acc = rng.integers(-8, 9, 32).astype(np.int64)
        mask = sum(1 << l for l in range(32) if ended[l])
        f = ended.astype(np.int64).copy()
        v_old, v_new = acc.copy(), acc.copy()
        d = 1
        while d < 32:
            fo = np.array([f[i - d] if i >= d else 0 for i in range(32)])
            vo_old = np.array([v_old[i - d] if i >= d else 0 for i in range(32)])
            vo_new = np.array([v_new[i - d] if i >= d else 0 for i in range(32)])
            for i in range(32):
                if i >= d and not f[i]:
                    v_old[i] += vo_old[i]
                lo = max(0, i - d + 1)
                ble = mask & ((2 << i) - 1 if i < 31 else 0xFFFFFFFF)
                if i >= d and (ble >> lo) == 0:
                    v_new[i] += vo_new[i]
            f = np.array([(f[i] | fo[i]) if i >= d else f[i] for i in range(32)])
            d <<= 1
        assert np.array_equal(v_old, v_new)


def _stage_branchy(ends, head_before, row0, base, p):
    """The per-entry row-end loop as first written: a branch per row end."""
    fin, acc, cur, nemit, head_acc, head_pending = {}, 0, row0, 0, 0, False
    for j in range(16):
        acc += p[j]
        if (ends >> j) & 1:
            if nemit == 0 and head_before:
                head_acc, head_pending = acc, True
            else:
                fin[cur - base] = acc
            nemit += 1
            cur += 1
            acc = 0
    return fin, acc, cur, nemit, head_acc, head_pending


def _stage_branch_free(ends, head_before, row0, base, p):
    """spmv_tiles' branch-free form: the first end closes the head row when
    it began earlier; every other end stores at row0 - base + (ends before it)."""
    head_bit = (ends & (-ends & 0xffffffff)) if head_before else 0
    fin, acc, head_acc, k = {}, 0, 0, 0
    for j in range(16):
        acc += p[j]
        e, h = (ends >> j) & 1, (head_bit >> j) & 1
        if e and not h:
            fin[row0 - base + k] = acc
        head_acc = acc if h else head_acc
        k += e
        acc = 0 if e else acc
    return fin, acc, row0 + k, k, head_acc, head_bit != 0


def test_branch_free_row_end_staging_equals_the_branchy_loop():
    rng = np.random.default_rng(11)
    for _ in range(4000):
        ends = int(rng.integers(0, 1 << 16))
        if rng.random() < 0.2:
            ends = 0
        head_before = bool(rng.integers(0, 2))
        row0 = int(rng.integers(0, 1000))
        base = row0 - int(rng.integers(0, 3))
        p = rng.integers(-9, 10, size=16)
        assert _stage_branchy(ends, head_before, row0, base, p) == _stage_branch_free(ends, head_before, row0, base, p)
