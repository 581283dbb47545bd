"""CPU checks of two warp algorithms of the BF16 scan (harmony_b200/csrc/k_tc.cu),
restated step for step in Python with a lane per list element:

- fetch_item's 32-way search of the per-list item offsets (a warp probes 32
  positions per round; the lanes at or under the item form a prefix), which
  must find the list l with item_off[l] <= item < item_off[l + 1], empty lists
  included;
- the split of coarse_tc's (centroid tile, query tile) pairs over CTAs
  (k_coarse_tc.cu coarse_range): contiguous ranges covering every pair once;
- the chunk-minimum row selection (k_select.cu select_rows_chunk_kernel):
  the k-th smallest chunk minimum T bounds the row's k-th smallest value, so
  the values <= T of the chunks with minimum <= T hold the k smallest keys;
- warp_kth_small8, the k-th smallest of up to 256 keys held eight per lane
  for small k (a sorting network per lane, then k rounds of a warp minimum);
- warp_kth_smallest, the radix selection over four 8-bit digits with a
  256-bin histogram (lane L owns bins 8L .. 8L+7), digits shared by the
  smallest and largest key skipped; used by the seed bound, the re-rank and
  the two-stage bound of k > 16.

Both are compared with the obvious answer (bisect, sorted) on random inputs,
ties and degenerate sizes included."""
import bisect
import random


def search_32way(item_off, nlist, item):
    lo, hi = 0, nlist
    while hi - lo > 1:
        step = max(1, (hi - lo) // 32)
        le = [lo + (j + 1) * step < hi and item_off[lo + (j + 1) * step] <= item for j in range(32)]
        n = sum(le)
        assert le == [True] * n + [False] * (32 - n)  # a prefix: the ballot's popcount is its length
        if n < 32:
            hi = min(hi, lo + (n + 1) * step)
        lo += n * step
    return lo


def warp_kth_smallest(vals, k):
    lo, hi = min(vals), max(vals)
    prefix, pmask, need = 0, 0, k
    for shift in (24, 16, 8, 0):
        if (lo >> shift) == (hi >> shift):
            # every key has this digit: no count
            prefix |= lo & (255 << shift)
            pmask |= 255 << shift
            continue
        h = [0] * 256
        for v in vals:
            if (v & pmask) == prefix:
                h[(v >> shift) & 255] += 1
        sums = [sum(h[8 * lane:8 * lane + 8]) for lane in range(32)]
        incl, acc = [], 0
        for s in sums:
            acc += s
            incl.append(acc)
        excl = [incl[lane] - sums[lane] for lane in range(32)]
        src = next(lane for lane in range(32) if excl[lane] < need <= incl[lane])
        before, b = excl[src], None
        for j in range(8):
            if before + h[8 * src + j] >= need:
                b = 8 * src + j
                break
            before += h[8 * src + j]
        need -= before
        prefix |= b << shift
        pmask |= 255 << shift
    return prefix


NET8 = [(0, 1), (2, 3), (4, 5), (6, 7), (0, 2), (1, 3), (4, 6), (5, 7), (1, 2), (5, 6),
        (0, 4), (1, 5), (2, 6), (3, 7), (2, 4), (3, 5), (1, 2), (3, 4), (5, 6)]


def warp_kth_small8(lanes, k):
    """lanes: 32 lists of 8 keys (0xFFFFFFFF pads)."""
    lanes = [list(v) for v in lanes]
    for v in lanes:
        for a, b in NET8:
            v[a], v[b] = min(v[a], v[b]), max(v[a], v[b])
    m = 0
    for _ in range(k):
        m = min(v[0] for v in lanes)
        who = next(i for i, v in enumerate(lanes) if v[0] == m)  # lowest lane pops
        lanes[who] = lanes[who][1:] + [0xFFFFFFFF]
    return m


def test_sorting_network_of_eight():
    # 0-1 principle: a comparator network sorts every input iff it sorts every 0/1 input
    for bits in range(256):
        v = [(bits >> i) & 1 for i in range(8)]
        for a, b in NET8:
            v[a], v[b] = min(v[a], v[b]), max(v[a], v[b])
        assert v == sorted(v)


def test_small_kth_matches_sort():
    rng = random.Random(4)
    for _ in range(400):
        n = rng.randint(1, 256)
        vals = [rng.choice([rng.getrandbits(32), rng.getrandbits(6)]) for _ in range(n)]
        k = rng.randint(1, min(n, 32))
        lanes = [[vals[32 * i + lane] if 32 * i + lane < n else 0xFFFFFFFF for i in range(8)] for lane in range(32)]
        assert warp_kth_small8(lanes, k) == sorted(vals)[k - 1]


def test_32way_search_finds_the_list():
    rng = random.Random(1)
    for _ in range(600):
        nlist = rng.choice([1, 2, 31, 32, 33, 63, 64, 65, 100, 1229, 4096, rng.randint(1, 9000)])
        cnt = [rng.choice([0, 0, 1, 2, 5]) for _ in range(nlist)]
        if sum(cnt) == 0:
            cnt[rng.randrange(nlist)] = 1
        off = [0]
        for c in cnt:
            off.append(off[-1] + c)
        for _ in range(10):
            item = rng.randrange(off[-1])
            assert search_32way(off, nlist, item) == bisect.bisect_right(off, item) - 1


def test_radix_kth_matches_sort():
    rng = random.Random(2)
    for _ in range(400):
        n = rng.randint(1, 300)
        if rng.random() < 0.3:
            pool = [rng.getrandbits(32) for _ in range(rng.randint(1, 4))]
            vals = [rng.choice(pool) for _ in range(n)]
        else:
            bits = rng.choice([32, 12, 4])
            vals = [rng.getrandbits(bits) for _ in range(n)]
        k = rng.randint(1, n)
        assert warp_kth_smallest(vals, k) == sorted(vals)[k - 1]


def test_radix_kth_clustered_keys():
    # keys of one query share their top bits (one exponent): skipped digits
    rng = random.Random(3)
    for _ in range(300):
        base = rng.getrandbits(32) & 0xFFF00000
        n = rng.randint(1, 300)
        vals = [base | rng.getrandbits(rng.choice([4, 12, 20])) for _ in range(n)]
        k = rng.randint(1, n)
        assert warp_kth_smallest(vals, k) == sorted(vals)[k - 1]


def select_by_chunk_minima(row, k, w=16):
    nch = (len(row) + w - 1) // w
    cm = [min(row[w * c:w * c + w]) for c in range(nch)]
    T = sorted(cm)[k - 1]
    keys = [(row[j], j) for c in range(nch) if cm[c] <= T for j in range(w * c, min(w * c + w, len(row))) if row[j] <= T]
    return sorted(keys)[:k]


def test_chunk_minimum_selection_matches_sort():
    rng = random.Random(5)
    for _ in range(300):
        n = rng.choice([37, 130, 300, 1000, 4096, rng.randint(1, 5000)])
        pool = rng.choice([None, [rng.random() for _ in range(5)]])
        row = [rng.choice(pool) if pool else rng.random() for _ in range(n)]
        nch = (n + 15) // 16
        k = rng.randint(1, nch)
        assert select_by_chunk_minima(row, k) == sorted((v, j) for j, v in enumerate(row))[:k]


def coarse_range(b, G, pairs):
    return b * pairs // G, (b + 1) * pairs // G


def test_coarse_pair_ranges_cover_every_pair_once():
    rng = random.Random(6)
    for _ in range(300):
        qt, ct = rng.randint(1, 120), rng.randint(1, 64)
        pairs = qt * ct
        G = max(1, min(pairs, rng.choice([148, 132, 7, 1])))
        seen, prev_end = [], 0
        for b in range(G):
            p0, p1 = coarse_range(b, G, pairs)
            assert p0 == prev_end and p1 > p0  # contiguous, never empty (pairs >= G)
            prev_end = p1
            seen.extend(range(p0, p1))
            # pairs are centroid-tile major: a CTA loads ceil-ish (range / qt) + 1 tiles at most
            tiles = {p // qt for p in range(p0, p1)}
            assert len(tiles) <= (p1 - p0 + qt - 1) // qt + 1
        assert seen == list(range(pairs))
