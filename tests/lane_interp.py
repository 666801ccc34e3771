"""A host interpreter of the lane solve's records (the semantics of lane_solve.cuh), for checking
layouts on the CPU: every right-hand side is one lane, each warp's live slots and prefetch ring
(slots, lanes) arrays, the warps run between block barriers one after another. It also checks that
every row is read from its ring slot after its prefetch and before the slot is refilled."""
import numpy as np

FWD_ROW0, FWD_PRE1, BWD_ROW0, BWD_PRE1 = 0, 5, 9, 14
FWD_ROWN, FWD_MORE, BWD_ROWN, BWD_BEGIN, BWD_MORE, BWD_END = range(18, 24)
PREFETCH, PHASE, TOP_SUM, FLUSH, IMPORT, BARRIER, END, PAGE_END = range(24, 32)
RING, BATCH = 8, 4
PAGE_RING, BARRIERS = 2, 4
TOP_SUMS, TOP_LOAD, TOP_ROW, TOP_ROW_MORE = range(4)  # the modes of a TOP_SUM record


def warp_bytes(lay):
    """A warp's shared bytes (lane_warp_bytes_of): slots, the prefetch ring, the page ring and its
    barriers, rounded to 128; the dense top's block-wide offsets count in them."""
    row = 32 * lay["value_bytes"] * lay.get("rpl", 1)
    b = lay["slots"] * row + RING * row + PAGE_RING * lay["page_bytes"] + PAGE_RING * 8
    return (b + 127) // 128 * 128


def records(lay, warp):
    """Yields (kind, ring, self, count, word, tail, vals, words, offsets, body) for each record of a warp."""
    pb, vb = lay["page_bytes"], lay["value_bytes"]
    ftype = np.float64 if vb == 8 else np.float32
    entry = 16 if vb == 8 else 8
    blob = lay["blob"]
    for k in range(lay["warp_page"][warp], lay["warp_page"][warp + 1]):
        page = blob[k * pb:(k + 1) * pb]
        pos = 0
        while True:
            assert pos + 16 <= pb, "a page without its end record"
            head, word = (int(v) for v in page[pos:pos + 8].view(np.uint32))
            self_, kb, count = head & 0xFFFF, (head >> 16) & 0xFF, head >> 24
            kind, ring = kb & 31, kb >> 5
            if kind == PAGE_END:
                break
            tail = page[pos + 8:pos + 16]
            body = page[pos + 16:pos + 16 + ((count * entry + 15) & ~15)]
            assert pos + 16 + count * entry <= pb, "a record past its page"
            vals = np.array([body[e * entry:e * entry + vb].view(ftype)[0] for e in range(count)], np.float64)
            words = np.array([body[e * entry:e * entry + 4].view(np.uint32)[0] for e in range(count)], np.int64)
            offs = np.array([body[e * entry + vb:e * entry + vb + 4].view(np.uint32)[0] for e in range(count)], np.int64)
            yield kind, ring, self_, count, word, tail, vals, words, offs, body
            if kind == END:
                return
            pos += 16 + ((count * entry + 15) & ~15)


def warp_steps(lay, warp, work, partial, lanes, lives):
    """Runs one warp's records, yielding at each block barrier; lives[w] is warp w's slots."""
    vb = lay["value_bytes"]
    ftype = np.float64 if vb == 8 else np.float32
    row = 32 * vb * lay.get("rpl", 1)  # a slot or row: 32 lanes of rpl values
    live = lives[warp]
    wb = warp_bytes(lay)
    ring = np.full((RING, lanes), np.nan)
    pending = np.zeros(RING, bool)  # a prefetched row not read yet
    z = None

    def prefetch(block):
        assert len(block) == 16
        words = block.view(np.uint32).copy()
        nrows, base = int(words[0] & 7), BATCH if words[0] & 8 else 0
        words[0] &= ~np.uint32(15)
        assert nrows <= BATCH
        for q in range(nrows):
            assert words[q] % row == 0
            assert not pending[base + q], "a prefetch over a row not read yet"
            assert 0 <= words[q] // row < work.shape[0], "a prefetch outside the work array"
            ring[base + q] = work[words[q] // row]
            pending[base + q] = True

    for kind, rs, self_, count, word, tail, vals, words, offs, body in records(lay, warp):
        s, w = self_ * 16 // row, word // row
        fwd = kind < BWD_ROW0 or kind in (FWD_ROWN, FWD_MORE)
        bwd = BWD_ROW0 <= kind < FWD_ROWN or BWD_ROWN <= kind <= BWD_END
        if fwd or bwd:
            dinv = float(tail[:vb].view(ftype)[0])
            assert 0 <= w < work.shape[0], "a row outside the work array"
        if kind in range(FWD_ROW0, FWD_PRE1) or kind in range(BWD_ROW0, BWD_PRE1):
            assert count == kind - (FWD_ROW0 if fwd else BWD_ROW0)
        if kind in range(FWD_PRE1, BWD_ROW0) or kind in range(BWD_PRE1, FWD_ROWN):
            c = kind - (FWD_PRE1 if fwd else BWD_PRE1) + 1
            pad = (c * (16 if vb == 8 else 8) + 15) // 16 * 16
            assert len(body) == pad + 16, "a row's prefetch block after its entries"
            prefetch(body[pad:pad + 16])
            vals, offs = vals[:c], offs[:c]
        if fwd and kind != FWD_MORE:
            assert pending[rs], "a row read before its prefetch"
            pending[rs] = False
            z = (ring[rs] + live[s]) * dinv
            live[s] = 0.0
            work[w] = z
        if fwd:
            for v, o in zip(vals, offs):
                live[o // row] -= v * z
        elif bwd:
            if kind not in (BWD_MORE, BWD_END):
                assert pending[rs], "a row read before its prefetch"
                pending[rs] = False
                z = ring[rs].copy()
            for v, o in zip(vals, offs):
                z = z - v * live[o // row]
            if kind not in (BWD_BEGIN, BWD_MORE):
                x = z * dinv
                live[s] = x
                work[w] = x
        elif kind == PREFETCH:
            prefetch(body)
        elif kind == PHASE:
            assert not pending.any(), "a phase that leaves prefetched rows unread"
            ring[:] = np.nan
        elif kind == TOP_SUM:
            mode = int(tail[:4].view(np.uint32)[0])
            if mode == TOP_SUMS:
                assert 0 <= w < work.shape[0], "a row outside the work array"
                for k in words:
                    work[w] = work[w] + partial[k // row]
            elif mode == TOP_LOAD:
                for p, o in zip(words, offs):
                    assert 2 <= o // row < lay["slots"], "a top value loaded into the zero or the sink slot"
                    live[o // row] = work[p // row]
            else:
                assert mode in (TOP_ROW, TOP_ROW_MORE), f"unknown top mode {mode}"
                assert 0 <= w < work.shape[0], "a row outside the work array"
                acc = np.zeros(lanes) if mode == TOP_ROW else work[w].copy()
                for v, a in zip(vals, offs):
                    owner, rest = divmod(int(a), wb)
                    assert 0 <= owner < lay["warps"] and rest % row == 0 and 2 <= rest // row < lay["slots"], \
                        "a dense top offset outside every warp's slots"
                    acc = acc + v * lives[owner][rest // row]
                work[w] = acc
        elif kind == FLUSH:
            for k, o in zip(words, offs):
                partial[k // row] = live[o // row]
                live[o // row] = 0.0
        elif kind == IMPORT:
            for p, o in zip(words, offs):
                live[o // row] = work[p // row]
        elif kind == BARRIER:
            yield
        elif kind == END:
            assert not live[0].any(), "the zero slot was written"
            return
        else:
            raise AssertionError(f"unknown record kind {kind}")


def run(lay, n, rhs):
    """Solves the rows of `rhs` (count x n, natural order) through the records."""
    rhs = np.atleast_2d(np.asarray(rhs, np.float64))
    lanes = rhs.shape[0]
    work = np.zeros((n, lanes))
    work[lay["in_pos"]] = rhs.T
    partial = np.zeros((max(lay["partials"], 1), lanes))
    lives = [np.zeros((lay["slots"], lanes)) for _ in range(lay["warps"])]
    warps = [warp_steps(lay, w, work, partial, lanes, lives) for w in range(lay["warps"])]
    for _ in range(BARRIERS + 1):  # the epochs around the barriers
        for g in warps:
            next(g, None)
    return work[lay["out_pos"]].T.copy()
