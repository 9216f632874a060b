"""The map invariant checker (fusion_b200/invariants.py) on tables built on
the host by a restatement of the reference's sequential insertion
(DeviceMap::CreateBlock / CreateEntry, DeviceMap.cu:12-62, no contention):
a sound table passes, and each planted defect is reported.  CPU only."""
import numpy as np

from fusion_b200 import invariants as I

NB, NE, NS = 128, 64, 200


def build(blocks):
    e = np.zeros((NB + NE, 5), np.int64)
    e[:, 3] = -1
    heap = NS - 1 - np.arange(NS)
    counter, entry_ptr = NS - 1, 1
    for x, y, z in blocks:
        b = int(I.bucket_of(x, y, z, NB))
        slot, last, found, empty = b, b, False, None
        while True:
            if tuple(e[slot, :3]) == (x, y, z) and e[slot, 3] >= 0:
                found = True
                break
            if e[slot, 3] < 0 and empty is None:
                empty = slot
            last = slot
            if e[slot, 4] <= 0:
                break
            slot = NB + e[slot, 4] - 1
        if found:
            continue
        old = counter
        counter -= 1
        ptr = int(heap[old]) * 512
        if empty is not None:
            e[empty] = (x, y, z, ptr, e[last, 4])
        else:
            off = entry_ptr
            entry_ptr += 1
            e[NB + off - 1] = (x, y, z, ptr, 0)
            e[last, 4] = off
    return e, counter, entry_ptr


def sound():
    rng = np.random.default_rng(3)
    blocks = [tuple(int(v) for v in rng.integers(-6, 7, 3)) for _ in range(120)]
    e, hc, ep = build(blocks)
    assert (e[NB:, 3] >= 0).sum() > 5          # chains exist
    return e, hc, ep


def test_sound_table_passes():
    e, hc, ep = sound()
    assert I.check_map(e, NB, NE, NS, heap_counter=hc, entry_ptr=ep) == []


def test_hash_is_the_unsigned_modulo_of_the_wrapped_products():
    # int res = (...) % NumBuckets with NumBuckets unsigned: the 32-bit pattern
    # of the xor of the wrapped products, modulo NumBuckets as unsigned
    def ref(x, y, z, n):
        h = (((x * 73856093) % 2 ** 32) ^ ((y * 19349669) % 2 ** 32) ^ ((z * 83492791) % 2 ** 32))
        return h % n
    for x, y, z in [(0, 0, 0), (1, 2, 3), (-1, -2, -3), (4000, -5000, 60), (-32767, 32767, -1)]:
        for n in (64, 1000000, 1 << 20):
            assert int(I.bucket_of(x, y, z, n)) == ref(x, y, z, n)


def _kinds(msgs):
    return " | ".join(msgs)


def test_planted_defects_are_reported():
    e, hc, ep = sound()
    occ_b = [i for i in range(NB) if e[i, 3] >= 0]
    occ_x = [NB + j for j in range(NE) if e[NB + j, 3] >= 0]
    # a block moved to a foreign bucket slot
    t = e.copy()
    free = next(i for i in range(NB) if t[i, 3] < 0)
    t[free, :4] = t[occ_b[0], :4]
    t[occ_b[0], 3] = -1
    assert "foreign bucket" in _kinds(I.check_map(t, NB, NE, NS))
    # two entries on one pool block
    t = e.copy()
    t[occ_b[1], 3] = t[occ_b[2], 3]
    assert "pool block shared" in _kinds(I.check_map(t, NB, NE, NS))
    # a pool index that is not a block boundary, and one past the pool
    t = e.copy()
    t[occ_b[0], 3] += 1
    t[occ_b[1], 3] = NS * 512
    assert _kinds(I.check_map(t, NB, NE, NS)).count("bad pool index") == 2
    # a cut chain
    t = e.copy()
    head = next(i for i in range(NB) if t[i, 4] > 0)
    t[head, 4] = 0
    assert "unreachable excess entry" in _kinds(I.check_map(t, NB, NE, NS))
    # ... which is expected once the pool has run out
    assert "unreachable" not in _kinds(I.check_map(t, NB, NE, NS, exhausted=True))
    # a cycle
    t = e.copy()
    x = occ_x[0]
    t[x, 4] = x - NB + 1
    assert "chain cycle" in _kinds(I.check_map(t, NB, NE, NS))
    # a link out of range
    t = e.copy()
    t[occ_b[0], 4] = NE + 5
    assert "link out of range" in _kinds(I.check_map(t, NB, NE, NS))
    # a block entered twice
    t = e.copy()
    free = next(i for i in range(NB) if t[i, 3] < 0)
    b0 = occ_b[0]
    t[free] = (t[b0, 0], t[b0, 1], t[b0, 2], (NS - 1) * 512 if (NS - 1) * 512 not in t[:, 3] else 0, 0)
    msgs = _kinds(I.check_map(t, NB, NE, NS))
    assert "entries" in msgs and "foreign bucket" in msgs
    # counters that disagree with the table
    msgs = _kinds(I.check_map(e, NB, NE, NS, heap_counter=hc + 1, entry_ptr=1))
    assert "heap_counter" in msgs and "entry_ptr" in msgs


def test_reference_tables_show_its_allocator_races():
    """The reference's own tables after one 128x96 frame (golden fixture from
    its CUDA kernels, frames A and B): every head entry lies in the bucket
    the checker's hash gives (the restatement of DeviceMap::Hash agrees with
    the reference on every slot), and the reference's racy CreateBlock
    (DeviceMap.cu:23-62: the bucket lock is released without a fence, the
    entry written as a plain 32-byte store) shows as excess entries whose
    chain link was overwritten, blocks entered more than once, and pool
    blocks handed out by the heap that no entry holds."""
    from tests import golden_util as G
    fz = G.load("fuse_128x96.npz")
    c = G.meta()["constants"]
    NBr, NEr, NSr = int(c["num_buckets"]), int(c["num_excess"]), int(c["num_blocks"])
    for p in "ab":
        t = np.zeros((NBr + NEr, 5), np.int64)
        t[:, 3] = -1
        t[fz[p + "_slots"]] = fz[p + "_entries"]
        hc, ep = (int(v) for v in fz[p + "_counters"])
        msgs = I.check_map(t, NBr, NEr, NSr, heap_counter=hc, entry_ptr=ep, limit=10 ** 6)
        unreached = [m for m in msgs if m.startswith("unreachable excess entry")]
        repeated = [m for m in msgs if m.startswith("block ") and " entries" in m]
        leaked = [m for m in msgs if m.startswith("allocated entries")]
        print(p, len(unreached), "unreachable,", len(repeated), "repeated blocks,", leaked)
        assert len(unreached) + len(repeated) + len(leaked) == len(msgs)   # nothing else, no foreign bucket
        assert len(unreached) >= 20 and len(repeated) >= 40 and len(leaked) == 1
        n_entries = len(fz[p + "_slots"])
        assert NSr - 1 - hc > 1.5 * n_entries                              # most of the leak: lost entries
