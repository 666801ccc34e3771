"""A host interpreter of the lane solve's records (the semantics of lane_solve.cuh), for checking
layouts on the CPU: every right-hand side is one lane, each warp's live slots a (slots, lanes)
array, the warps run between block barriers one after another."""
import numpy as np

ROW, ROW_BEGIN, ROW_MORE, ROW_END, PHASE, PARTIALS, FLUSH, IMPORT, BARRIER, END, PAGE_END = range(11)
BACKWARD = 0x100


def records(lay, warp):
    """Yields (kind, self, count, head_word, dinv, vals, words, offsets) for each record of a warp."""
    pb, vb = lay["page_bytes"], lay["value_bytes"]
    ftype = np.float64 if vb == 8 else np.float32
    entry = 16 if vb == 8 else 8
    blob = lay["blob"]
    for k in range(lay["warp_page"][warp], lay["warp_page"][warp + 1]):
        page = blob[k * pb:(k + 1) * pb]
        pos = 0
        while pos + 16 <= pb:
            self_, word = (int(v) for v in page[pos:pos + 8].view(np.uint32))
            kind, count = word >> 16, word & 0xFFFF
            if kind == PAGE_END:
                break
            head_word = int(page[pos + 8:pos + 12].view(np.uint32)[0])
            dinv = float(page[pos + 8:pos + 8 + vb].view(ftype)[0])
            body = page[pos + 16:pos + 16 + count * entry]
            vals = np.array([body[e * entry:e * entry + vb].view(ftype)[0] for e in range(count)], np.float64)
            words = np.array([body[e * entry:e * entry + 4].view(np.uint32)[0] for e in range(count)], np.int64)
            offs = np.array([body[e * entry + vb:e * entry + vb + 4].view(np.uint32)[0] for e in range(count)], np.int64)
            yield kind, self_, count, head_word, dinv, vals, words, offs
            if kind == END:
                return
            pos += 16 + ((count * entry + 15) & ~15)


def warp_steps(lay, warp, work, partial, lanes):
    """Runs one warp's records, yielding at each block barrier."""
    slot_bytes = 32 * lay["value_bytes"]
    live = np.zeros((lay["slots"], lanes))
    start = i = 0
    backward = False
    z = None
    cur = 0

    def next_row():
        nonlocal i, cur
        cur = start - i if backward else start + i
        i += 1
        return work[cur].copy()

    for kind, self_, count, head_word, dinv, vals, words, offs in records(lay, warp):
        s = self_ // slot_bytes
        if kind <= ROW_END:
            if not backward:
                if kind <= ROW_BEGIN:
                    z = (next_row() + live[s]) * dinv
                    live[s] = 0.0
                    work[cur] = z
                for v, o in zip(vals, offs):
                    live[o // slot_bytes] -= v * z
            else:
                if kind <= ROW_BEGIN:
                    z = next_row()
                for v, o in zip(vals, offs):
                    z = z - v * live[o // slot_bytes]
                if kind in (ROW, ROW_END):
                    x = z * dinv
                    live[s] = x
                    work[cur] = x
        elif kind & 0xFF == PHASE:
            start, i, backward = self_, 0, bool(kind & BACKWARD)
        elif kind == PARTIALS:
            for k in words:
                live[s] = live[s] + partial[k]
        elif kind == FLUSH:
            for k, o in zip(words, offs):
                partial[k] = live[o // slot_bytes]
                live[o // slot_bytes] = 0.0
        elif kind == IMPORT:
            for p, o in zip(words, offs):
                live[o // slot_bytes] = work[p]
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
    warps = [warp_steps(lay, w, work, partial, lanes) for w in range(lay["warps"])]
    for _ in range(3):  # the epochs between the two barriers
        for g in warps:
            next(g, None)
    return work[lay["out_pos"]].T.copy()
