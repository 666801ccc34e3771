"""A host interpreter of the domain solve's record streams (test infrastructure).

It executes, in numpy, what the domain solve kernel does with the pages of a
`host.domain_layout`: stage by stage, each warp's records in order. Tests run it against the
oracle's solves, so the layout builder is checked on the CPU before any kernel runs.
"""
from __future__ import annotations

import numpy as np

ROWS, SPLIT, DENSE, COPY, END = 4, 1, 2, 3, -1
FIRST, LAST, TO_TAIL = 1, 2, 4


def _a16(v: int) -> int:
    return (v + 15) & ~15


def parse(layout: dict) -> list:
    """Each warp's records as (stage, kind, fields)."""
    vt = np.float64 if layout["value_bytes"] == 8 else np.float32
    s = layout["value_bytes"]
    blob, pb, wp = layout["blob"], layout["page_bytes"], layout["warp_page"]
    streams = []
    for w in range(layout["warps"]):
        recs = []
        for page in range(wp[w], wp[w + 1]):
            base = page * pb
            pos = 0
            while pos + 16 <= pb:
                kind, stage, z, flags = (int(x) for x in blob[base + pos: base + pos + 16].view(np.int32))
                if kind < 0:
                    break
                if kind == ROWS:
                    kl, nent, size, _ = (int(x) for x in blob[base + pos + 16: base + pos + 32].view(np.int32))
                    oi, od, oc, ov = (int(x) for x in blob[base + pos + 32: base + pos + 48].view(np.int32))
                    rb = base + pos
                    info = blob[rb + oi: rb + oi + 8 * z].view(np.int32).reshape(z, 2)
                    dv = blob[rb + od: rb + od + s * z].view(vt)
                    cols = blob[rb + oc: rb + oc + 2 * nent].view(np.uint16).astype(np.int64)
                    vals = blob[rb + ov: rb + ov + s * nent].view(vt)
                    assert z << kl <= 32 and pos + size <= pb
                    recs.append((stage, kind, (info.copy(), dv.copy(), cols, vals.copy(), flags, kl)))
                    pos += size
                elif kind == DENSE:
                    t, j0 = (int(x) for x in blob[base + pos + 16: base + pos + 24].view(np.int32))
                    vals = blob[base + pos + 32: base + pos + 32 + s * z].view(vt)
                    recs.append((stage, kind, (t, j0, vals.copy(), flags)))
                    pos += 32 + _a16(s * z)
                elif kind == COPY:
                    recs.append((stage, kind, None))
                    pos += 16
                elif kind == SPLIT:
                    row, dest = (int(x) for x in blob[base + pos + 16: base + pos + 24].view(np.int32))
                    dinv = blob[base + pos + 32: base + pos + 32 + s].view(vt)[0]
                    col = blob[base + pos + 48: base + pos + 48 + 4 * z].view(np.int32).astype(np.int64)
                    q = base + pos + 48 + _a16(4 * z)
                    vals = blob[q: q + s * z].view(vt)
                    recs.append((stage, kind, (row, dest, dinv, col, vals.copy(), flags)))
                    pos += 48 + _a16(4 * z) + _a16(s * z)
                else:
                    raise AssertionError(f"unknown record kind {kind}")
        streams.append(recs)
    return streams


def run(layout: dict, n: int, in_slot: np.ndarray, out_slot: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Solves the columns of b ((count, n), natural order) as the kernel does, all columns as one
    tile. Values are float64 or float32 as the layout's value bytes say."""
    vt = np.float64 if layout["value_bytes"] == 8 else np.float32
    W = b.shape[0]
    m = layout["top"]
    Y = np.zeros((n + 2, W), vt)
    Tb = np.zeros((m + 1, W), vt)
    tslot = np.concatenate([layout["top_slot"], [n]]).astype(np.int64)
    Y[in_slot] = b.T.astype(vt)
    streams = parse(layout)
    for stage in range(layout["stages"]):
        for recs in streams:
            acc = np.zeros(W, vt)
            for st, kind, rec in recs:
                if min(st, layout["stages"]) != stage:
                    continue
                if kind == ROWS:
                    info, dv, cols, vals, flags, _ = rec
                    out = []
                    for r in range(info.shape[0]):
                        x0, x1 = int(info[r, 0]), int(info[r, 1])
                        slot, length = x0 & 0xFFFF, (x0 >> 16) & 0xFFFF
                        start, dest = x1 & 0xFFFF, (x1 >> 16) & 0xFFFF
                        p = np.arange(start, start + length)
                        total = (vals[p, None] * Y[cols[p]]).sum(axis=0) if length else np.zeros(W, vt)
                        v = Y[slot] - total
                        out.append((dest, v if flags & TO_TAIL else v * dv[r]))
                    for dest, v in out:
                        if flags & TO_TAIL:
                            Tb[dest] = v
                        else:
                            Y[dest] = v
                elif kind == DENSE:
                    t, j0, vals, flags = rec
                    if flags & FIRST:
                        acc = np.zeros(W, vt)
                    acc = acc + (vals[:, None] * Tb[j0: j0 + vals.size]).sum(axis=0)
                    if flags & LAST:
                        Y[tslot[t]] = acc
                elif kind == COPY:
                    Tb[:m] = Y[tslot[:m]]
                elif kind == SPLIT:
                    row, dest, dinv, col, vals, flags = rec
                    if flags & FIRST:
                        acc = np.zeros(W, vt)
                    acc = acc + (vals[:, None] * Y[col]).sum(axis=0)
                    if flags & LAST:
                        if flags & TO_TAIL:
                            Tb[dest] = Y[row] - acc
                        else:
                            Y[row] = (Y[row] - acc) * dinv
    return Y[out_slot].T.astype(np.float64)
