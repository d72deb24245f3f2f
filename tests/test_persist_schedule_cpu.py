"""Model of the persistent batch kernel's work queue (fortress_b200/csrc/
fgpe_persist.cuh), run on the CPU.

The kernel's blocks take tickets from one counter: per step, the column tiles
of every instance, then the row chunks of every instance.  A column tile of
step s waits until the instance's step s-1 is published (fin >= s); a row
chunk of step s waits until all of the instance's column tiles of step s are
done; the block that finishes an instance's last row chunk of a step
publishes it (fin = s + 1).  A block waits only while it holds no other
unfinished item.

The model runs that protocol with fewer blocks than items and a random
interleaving of their actions, and checks that every launch finishes (no
deadlock, for any number of resident blocks and any order), that every item
starts only after the items it reads, and that the step publication of an
instance happens exactly once per step, after all its row chunks."""
import numpy as np
import pytest


def _items(cols, rows, nsteps):
    per = []
    for i, c in enumerate(cols):
        per += [("col", i, t) for t in range(c)]
    for i, r in enumerate(rows):
        per += [("row", i, t) for t in range(r)]
    return [(s,) + it for s in range(nsteps) for it in per]


def _run(cols, rows, nsteps, nblocks, seed):
    rng = np.random.default_rng(seed)
    items = _items(cols, rows, nsteps)
    n = len(cols)
    col_done = [0] * n
    row_done = [0] * n
    fin = [0] * n
    published = []
    ticket = 0
    # block state: None (idle), ("wait", item), ("work", item, remaining actions)
    blocks = [None] * nblocks
    done_items = set()
    idle_rounds = 0
    while True:
        live = [b for b in range(nblocks) if blocks[b] is not None or ticket < len(items)]
        if not live:
            break
        b = int(rng.choice(live))
        st = blocks[b]
        progressed = False
        if st is None:
            blocks[b] = ("wait", ticket)
            ticket += 1
            progressed = True
        elif st[0] == "wait":
            s, kind, i, t = items[st[1]]
            ok = fin[i] >= s if kind == "col" else col_done[i] >= (s + 1) * cols[i]
            if ok:
                # everything this item reads is done
                if kind == "col":
                    assert all(((s - 1, "row", i, u) in done_items) for u in range(rows[i])) or s == 0
                else:
                    assert all(((s, "col", i, u) in done_items) for u in range(cols[i]))
                blocks[b] = ("work", st[1], int(rng.integers(1, 4)))
                progressed = True
        else:
            k = st[1]
            if st[2] > 1:
                blocks[b] = ("work", k, st[2] - 1)
            else:
                s, kind, i, t = items[k]
                done_items.add(items[k])
                if kind == "col":
                    col_done[i] += 1
                else:
                    row_done[i] += 1
                    if row_done[i] == (s + 1) * rows[i]:
                        assert fin[i] == s
                        fin[i] = s + 1
                        published.append((i, s))
                blocks[b] = None
            progressed = True
        idle_rounds = 0 if progressed else idle_rounds + 1
        assert idle_rounds < 100000, "no block can make progress (deadlock)"
    assert len(done_items) == len(items)
    assert fin == [nsteps] * n
    assert sorted(published) == sorted((i, s) for i in range(n) for s in range(nsteps))


@pytest.mark.parametrize("nblocks", [1, 2, 3, 7, 64])
def test_queue_always_finishes(nblocks):
    cols = [4, 2, 8, 1]
    rows = [2, 4, 1, 3]
    for seed in range(20):
        _run(cols, rows, nsteps=3, nblocks=nblocks, seed=seed)


def test_single_instance_single_block():
    # one block, one instance: each row chunk right after the last column tile
    _run([3], [2], nsteps=4, nblocks=1, seed=0)
