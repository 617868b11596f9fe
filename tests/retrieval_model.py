"""Python restatement of the device retrieval structure's format and construction (test
infrastructure): levels of buckets, h = remix(key + 0x9E3779B97F4A7C15 * (level + 1)),
bucket = fastrange64(h, B), priority p = (h >> 8) & 127, a bucket keeps the keys with p < t for the
largest t with at most 248 such keys, rows = four remix words of h, forward elimination in column
order with the free columns at zero; an inconsistent kept set drops its highest priority value.
Pure Python integers: for a few thousand keys."""
M64 = (1 << 64) - 1
LOAD, CAP, PRIO, WORDS = 240, 248, 128, 4


def remix(z):
    # Stafford Mix13, the reference's remix
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def level_hash(key, level):
    return remix(key + 0x9E3779B97F4A7C15 * (level + 1))


def prio(h):
    return (h >> 8) & (PRIO - 1)


def row(h):
    """256-bit row as a Python int, word i in bits [64 i, 64 i + 64)."""
    r = 0
    for i in range(WORDS):
        r |= remix(h + 0xD6E8FEB86659FD93 * (i + 1)) << (64 * i)
    return r


def fastrange64(h, n):
    return (h * n) >> 64


def solve(rows, rhs):
    """Forward elimination in column order (lowest non-pivot row as pivot), back substitution with
    free columns at zero. Returns the 256-bit solution or None when inconsistent."""
    rows, rhs = list(rows), list(rhs)
    done = [False] * len(rows)
    pivot = [None] * (64 * WORDS)
    for c in range(64 * WORDS):
        p = next((i for i in range(len(rows)) if not done[i] and (rows[i] >> c) & 1), None)
        if p is None:
            continue
        pivot[c] = p
        done[p] = True
        for i in range(len(rows)):
            if not done[i] and (rows[i] >> c) & 1:
                rows[i] ^= rows[p]
                rhs[i] ^= rhs[p]
    if any(not done[i] and rhs[i] for i in range(len(rows))):
        return None
    x = 0
    for c in reversed(range(64 * WORDS)):
        p = pivot[c]
        if p is None:
            continue
        if (rhs[p] + bin(rows[p] & x).count("1")) & 1:
            x |= 1 << c
    return x


def build(keys, bits):
    """-> (level_buckets, solutions [4 words per bucket], thresholds)."""
    level_buckets, sols, thrs = [], [], []
    cur = list(zip(keys, bits))
    level = 0
    while cur:
        assert level < 40, "duplicate keys with different bits"
        nb = max(1, (len(cur) + LOAD - 1) // LOAD)
        buckets = [[] for _ in range(nb)]
        for k, b in cur:
            h = level_hash(k, level)
            buckets[fastrange64(h, nb)].append((h, k, b))
        nxt = []
        for bk in buckets:
            hist = [0] * PRIO
            for h, _, _ in bk:
                hist[prio(h)] += 1
            t, run = 0, 0
            for p in range(PRIO):
                run += hist[p]
                if run <= CAP:
                    t = p + 1
            while True:
                kept = [(h, b) for h, _, b in bk if prio(h) < t]
                x = solve([row(h) for h, _ in kept], [b for _, b in kept])
                if x is not None:
                    break
                t = max(prio(h) for h, _ in kept)
            sols.extend((x >> (64 * i)) & M64 for i in range(WORDS))
            thrs.append(t)
            nxt.extend((k, b) for h, k, b in bk if prio(h) >= t)
        level_buckets.append(nb)
        cur = nxt
        level += 1
    return level_buckets, sols, thrs


def query(level_buckets, sols, thrs, key):
    first = 0
    for level, nb in enumerate(level_buckets):
        h = level_hash(key, level)
        b = first + fastrange64(h, nb)
        if prio(h) < thrs[b]:
            r = row(h)
            x = sum(sols[b * WORDS + i] << (64 * i) for i in range(WORDS))
            return bin(r & x).count("1") & 1
        first += nb
    return 0
