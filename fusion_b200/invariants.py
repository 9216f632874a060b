"""Structural invariants of a session's voxel-block hash map, checked on the
host from a download of the table (fb_map_download_entries,
fb_map_get_stats).

The layout is the reference's (Mapping/DeviceMap.h:110-161,
Mapping/DeviceMap.cu:3-62): num_buckets bucket slots followed by num_excess
excess slots, each {x, y, z, ptr, offset}; ptr is a voxel index (pool block
* 512) or -1; a chain continues at slot num_buckets + offset - 1 while
offset > 0.  A map built by this library satisfies:

- every occupied bucket slot holds a block that hashes to that slot
  (DeviceMap::Hash, DeviceMap.cu:3-10);
- every occupied excess slot is reached from its block's bucket by the
  chain links, and every chain ends within num_excess links (no cycle);
- no block appears twice among the reachable entries, and no pool block is
  used by two entries; pool indices are multiples of 512 below
  num_blocks * 512;
- the counters agree with the table: allocated entries = num_blocks - 1 -
  heap_counter (the heap hands out blocks from the top,
  DeviceMap.cu:14-20), and excess slots in use < entry_ptr (the excess
  allocator's next slot, DeviceMap.cu:44-58).

Once the block pool has run out (FB_ERR_HEAP_EXHAUSTED), the reference's
allocator writes entries without a block (ptr -1), and a later insertion
that reuses such a slot in the middle of a chain gives it the offset of the
chain's last entry (DeviceMap.cu:44-48), which cuts the chain; its heap
counter also keeps counting failed requests.  This library reproduces that,
so after exhaustion the reachability and counter checks are skipped
(check_map(..., exhausted=True)).

check_map returns the violations found (an empty list for a sound map);
check_session downloads a session's table and checks it.
"""
import numpy as np


def bucket_of(x, y, z, num_buckets):
    """DeviceMap::Hash: ((x * 73856093) ^ (y * 19349669) ^ (z * 83492791))
    % NumBuckets, the products wrapping at 32 bits; NumBuckets is an unsigned
    constant, so the remainder is taken of the 32-bit pattern as unsigned
    (the reference's `res < 0` correction never applies)."""
    x, y, z = (np.asarray(v, np.int64) for v in (x, y, z))
    m = 0xFFFFFFFF
    h = ((x * 73856093) & m) ^ ((y * 19349669) & m) ^ ((z * 83492791) & m)
    return (h % int(num_buckets)).astype(np.int64)


def check_map(entries, num_buckets, num_excess, num_blocks, heap_counter=None, entry_ptr=None, exhausted=False,
              limit=20):
    """Violations of the invariants above in a table `entries` of shape
    (num_buckets + num_excess, 5); at most `limit` messages per kind."""
    e = np.asarray(entries, np.int64)
    NB, NE, NS = int(num_buckets), int(num_excess), int(num_blocks)
    out = []
    if e.shape != (NB + NE, 5):
        return [f"table shape {e.shape}, expected {(NB + NE, 5)}"]

    def report(kind, idx, what):
        idx = np.asarray(idx)
        for i in idx[:limit]:
            out.append(f"{kind}: slot {int(i)} {what(int(i))}")
        if len(idx) > limit:
            out.append(f"{kind}: ... {len(idx) - limit} more")

    occ = e[:, 3] >= 0
    # pool indices
    bad_ptr = np.nonzero(occ & ((e[:, 3] % 512 != 0) | (e[:, 3] >= NS * 512)))[0]
    report("bad pool index", bad_ptr, lambda i: f"ptr {e[i, 3]}")
    ptrs = e[occ, 3]
    u, cnt = np.unique(ptrs, return_counts=True)
    for p in u[cnt > 1][:limit]:
        out.append(f"pool block shared: ptr {int(p)} in slots {np.nonzero(e[:, 3] == p)[0].tolist()}")
    # bucket slots hold blocks of their own bucket
    b_occ = np.nonzero(occ[:NB])[0]
    if len(b_occ):
        h = bucket_of(e[b_occ, 0], e[b_occ, 1], e[b_occ, 2], NB)
        wrong = b_occ[h != b_occ]
        report("block in a foreign bucket", wrong, lambda i: f"block {tuple(e[i, :3])}")
    # chains: links in range, no cycle; collect the excess slots reached
    off = e[:, 4]
    bad_link = np.nonzero((off < 0) | (off > NE))[0]
    report("link out of range", bad_link, lambda i: f"offset {off[i]}")
    reached = np.zeros(NE, bool)
    reach_bucket = np.full(NE, -1, np.int64)
    cyc = []
    for b in np.nonzero((off[:NB] > 0) & (off[:NB] <= NE))[0]:
        j, steps = int(off[b]), 0
        while 0 < j <= NE:
            s = NB + j - 1
            if reached[j - 1] and reach_bucket[j - 1] == b:
                cyc.append(b)
                break
            if reached[j - 1] and reach_bucket[j - 1] != b:
                out.append(f"excess slot {s} linked from buckets {int(reach_bucket[j - 1])} and {int(b)}")
                break
            reached[j - 1] = True
            reach_bucket[j - 1] = b
            steps += 1
            if steps > NE:
                cyc.append(b)
                break
            j = int(off[s])
    report("chain cycle", np.array(cyc, np.int64), lambda i: "")
    x_occ = np.nonzero(occ[NB:])[0]
    if not exhausted:
        unreached = x_occ[~reached[x_occ]]
        report("unreachable excess entry", NB + unreached, lambda i: f"block {tuple(e[i, :3])}")
    rx = x_occ[reached[x_occ]]
    if len(rx):
        h = bucket_of(e[NB + rx, 0], e[NB + rx, 1], e[NB + rx, 2], NB)
        wrong = NB + rx[h != reach_bucket[rx]]
        report("excess entry in a foreign chain", wrong, lambda i: f"block {tuple(e[i, :3])}")
    # one entry per block
    keys = e[occ][:, :3]
    if len(keys):
        uk, kc = np.unique(keys, axis=0, return_counts=True)
        for k in uk[kc > 1][:limit]:
            out.append(f"block {tuple(int(v) for v in k)} has {int(kc[(uk == k).all(1)][0])} entries")
    # counters
    n_alloc = int(occ.sum())
    if heap_counter is not None and not exhausted and n_alloc != NS - 1 - int(heap_counter):
        out.append(f"allocated entries {n_alloc} != num_blocks - 1 - heap_counter = {NS - 1 - int(heap_counter)}")
    if entry_ptr is not None and len(x_occ) and int(x_occ.max()) + 1 >= int(entry_ptr):
        out.append(f"excess slot {int(x_occ.max())} in use at or past entry_ptr {int(entry_ptr)}")
    return out


FB_ERR_HEAP_EXHAUSTED = 0x1


def check_session(session):
    """check_map on a session's downloaded table and counters."""
    st = session.stats()
    c = session.cfg
    return check_map(session.entries(), c.num_buckets, c.num_excess, c.num_blocks,
                     heap_counter=st["heap_counter"], entry_ptr=st["entry_ptr"],
                     exhausted=bool(st["error_flags"] & FB_ERR_HEAP_EXHAUSTED))
