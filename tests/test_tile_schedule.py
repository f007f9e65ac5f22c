"""CPU emulation of spmv_tile_kernel's schedule (no GPU needed).

Restates, in numpy, the tiled-format builder of csr_device.cu (row
compaction, row-start bitmap, per-tile {first_row, head_t0, tail_span,
tail_continues}) and the kernel's per-thread logic (row ids from popcounts,
row-end bits, segmented block scan, cross-tile last-arriver rule), then checks
on many random structures — empty rows, rows spanning many tiles, rows
starting exactly on tile boundaries, padding — that every row receives
exactly the sum of its entries, exactly once, and that every arrival counter
returns to zero.  Products are small integers so sums are exact.
"""
import numpy as np
import pytest


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

    meta = []
    for t in range(nt):
        base, last = t * T, t * T + T - 1
        fr = row_of(base)
        head_t0 = int(rp_c[fr] // T) if rp_c[fr] < base else -1
        tr = row_of(last)
        tend = int(rp_c[tr + 1])
        cont = int(tr < rows_c and tend > last + 1)
        span = int((tend - 1) // T - t + 1) if cont and rp_c[tr] >= base else 0
        meta.append((fr, head_t0, span, cont))
    return dict(nt=nt, rows_c=rows_c, row_map=row_map, flags=flags, meta=meta, nnz=nnz)


def emulate(rp, prod, T=64, IPT=8):
    F = build_format(rp, T)
    m = len(rp) - 1
    nt, rows_c, flags, meta = F["nt"], F["rows_c"], F["flags"], F["meta"]
    B = T // IPT
    out = {}
    counter = {}
    carry = {}

    def emit(row_c, v):
        if row_c >= rows_c:
            return
        r = int(F["row_map"][row_c])
        assert r not in out, f"row {r} emitted twice"
        out[r] = v

    def arrive(t, row_c, v, is_tail, slot, count):
        carry[(t, is_tail)] = v
        old = counter.get(slot, 0)
        counter[slot] = old + 1
        if old == count - 1:
            s = carry[(slot, 1)]
            for tt in range(slot + 1, slot + count):
                s += carry[(tt, 0)]
            counter[slot] = 0
            emit(row_c, s)

    padded = np.zeros(nt * T, np.int64)
    padded[:len(prod)] = prod
    for t in range(nt):
        fr, head_t0, span, cont = meta[t]
        fl = flags[t * T:(t + 1) * T]
        pr = padded[t * T:(t + 1) * T]
        st = []
        for tid in range(B):
            q0 = tid * IPT
            bits = fl[q0:q0 + IPT]
            nxt = (0 if cont else 1) if tid == B - 1 else fl[q0 + IPT]
            ends = list(bits[1:]) + [nxt]
            row0 = fr + int(fl[1:q0 + 1].sum())
            head_before = bits[0] == 0
            acc, cur, nemit, head_pending, head_acc = 0, row0, 0, False, 0
            for j in range(IPT):
                acc += int(pr[q0 + j])
                if ends[j]:
                    if nemit == 0 and head_before:
                        head_acc, head_pending = acc, True
                    else:
                        emit(cur, acc)
                    nemit += 1
                    cur += 1
                    acc = 0
            st.append(dict(f=int(nemit > 0), v=acc, row0=row0, cur=cur, nemit=nemit,
                           head_pending=head_pending, head_acc=head_acc))
        # exclusive segmented scan of (f, v)
        pf, pv = 0, 0
        for tid in range(B):
            s = st[tid]
            carry_in = pv
            if s["head_pending"]:
                tot = s["head_acc"] + carry_in
                if s["row0"] == fr and head_t0 >= 0:
                    arrive(t, s["row0"], tot, 0, head_t0, meta[head_t0][2])
                else:
                    emit(s["row0"], tot)
            if tid == B - 1 and cont:
                tot = s["v"] if s["nemit"] > 0 else carry_in + s["v"]
                if s["cur"] == fr and head_t0 >= 0:
                    arrive(t, s["cur"], tot, 0, head_t0, meta[head_t0][2])
                else:
                    arrive(t, s["cur"], tot, 1, t, span)
            if s["f"]:
                pf, pv = 1, s["v"]
            else:
                pv += s["v"]
    # rows without entries come from the empty-row pass (value 0)
    for r in range(m):
        if rp[r + 1] == rp[r]:
            assert r not in out
            out[r] = 0
    assert all(v == 0 for v in counter.values()), counter
    return out


def check(rp, rng, T=64):
    nnz = int(rp[-1])
    prod = rng.integers(-3, 4, size=nnz)
    out = emulate(np.asarray(rp, np.int64), prod, T=T)
    m = len(rp) - 1
    assert sorted(out) == list(range(m))
    for r in range(m):
        assert out[r] == int(prod[rp[r]:rp[r + 1]].sum()), r


@pytest.mark.parametrize("mode", range(6))
def test_schedule_random_structures(mode):
    rng = np.random.default_rng(100 + mode)
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
        check(rp, rng)


def test_schedule_production_tile_size():
    rng = np.random.default_rng(7)
    L = np.concatenate([rng.integers(0, 60, 300), [2048 * 3 + 5, 2048, 0, 0, 4095], rng.integers(0, 9, 200)])
    rp = np.zeros(len(L) + 1, np.int64)
    rp[1:] = np.cumsum(L)
    check(rp, rng, T=2048)
