"""The worker-task queue of the fused search launch (riv_test_worker_queue enumerates it with
the same functions the kernel uses), on CPU.  The launch's groups take tasks strictly in
queue order and a task waits only for tasks earlier in the queue, which is what makes every
wait end: checked here for every frame shape and mode, with each task present exactly once.
Waits: deblock band b on the residual of MB rows b-1 .. b+1; the SAD-table MBs of row r (and
the row loader of row r) on deblocked bands r-1 .. r+1 (on residual rows r-1 .. r+1 when the
deblock level is 0); the scan on every residual row; the pack rows on the scan."""
import numpy as np
import pytest


def _tiles(w):
    return (w + 127) // 128 + 2 * ((w // 2 + 63) // 64)


@pytest.mark.parametrize("bw,bh", [(1, 1), (7, 5), (22, 18), (120, 68), (240, 135)])
@pytest.mark.parametrize("defer,deblock,compact", [(False, False, False), (True, True, True), (True, False, True),
                                                   (True, True, False)])
def test_queue_order_and_completeness(bw, bh, defer, deblock, compact):
    from riv2_b200.encoder import worker_queue
    w = bw * 16
    q = worker_queue(bw, bh, w, defer, deblock, True, compact)
    kinds, rows, idxs = q[:, 0], q[:, 1], q[:, 2]
    nr = (bw + 1) // 2 if defer else 0
    nd = _tiles(w) if defer and deblock else 0
    ncomp = 1 + bh if defer and compact else 0
    assert len(q) == bh * (nr + nd + bw) + ncomp
    # each task exactly once
    for kind, per_row in ((0, nr), (1, nd), (2, bw)):
        sel = q[kinds == kind]
        assert len(sel) == bh * per_row
        assert len({(r, i) for _, r, i in sel}) == len(sel)
        if per_row:
            assert sel[:, 1].min() == 0 and sel[:, 1].max() == bh - 1 and sel[:, 2].max() == per_row - 1
    assert (kinds == 3).sum() == (1 if ncomp else 0) and (kinds == 4).sum() == (bh if ncomp else 0)
    # position of the last task of each residual row / deblock band
    pos = np.arange(len(q))
    last_res = {r: pos[(kinds == 0) & (rows == r)].max() for r in range(bh)} if nr else {}
    last_db = {b: pos[(kinds == 1) & (rows == b)].max() for b in range(bh)} if nd else {}
    near = lambda r: range(max(r - 1, 0), min(r + 1, bh - 1) + 1)
    for i, (kind, row, _) in enumerate(q):
        if kind == 1:
            assert all(last_res[r] < i for r in near(row))
        elif kind == 2 and defer:
            before = last_db if nd else last_res
            assert all(before[r] < i for r in near(row))
        elif kind == 3:
            assert all(v < i for v in last_res.values())
        elif kind == 4:
            assert pos[kinds == 3][0] < i
