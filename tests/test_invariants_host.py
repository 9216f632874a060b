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


def test_hash_matches_signed_wrapping_modulo():
    # ((x*73856093) ^ (y*19349669) ^ (z*83492791)) % n in int32, + n if negative
    def ref(x, y, z, n):
        def w(v):
            return ((v + 2 ** 31) % 2 ** 32) - 2 ** 31
        h = w(w(x * 73856093) ^ w(y * 19349669) ^ w(z * 83492791))
        r = abs(h) % n * (1 if h >= 0 else -1)
        return r + n if r < 0 else r
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
