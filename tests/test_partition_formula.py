"""The many-thread restatement of the introselect partition step that the device photon-tree build uses
(ray-tracing_b200/csrc/lrt_photon_tree.cu), checked on the CPU against the sequential Hoare loop it
replaces: for random ranges with many equal keys, swapping the k-th left stop with the k-th right stop
for k <= K = max_x min(#left stops before x, #right stops at or after x), and cutting at
min(L_{K+1}, R_K), leaves the same arrangement and the same cut as the sequential scans."""
import numpy as np


def sequential(keys, first, last):
    """median-of-three pivot to `first`, then the unguarded Hoare partition of [first + 1, last)"""
    a = list(keys)
    mid = first + (last - first) // 2
    x, y, z = first + 1, mid, last - 1
    if a[x] < a[y]:
        m = y if a[y] < a[z] else (z if a[x] < a[z] else x)
    else:
        m = x if a[x] < a[z] else (z if a[y] < a[z] else y)
    a[first], a[m] = a[m], a[first]
    pivot = a[first]
    i, j = first + 1, last
    while True:
        while a[i] < pivot:
            i += 1
        j -= 1
        while pivot < a[j]:
            j -= 1
        if not i < j:
            return a, i
        a[i], a[j] = a[j], a[i]
        i += 1


def restated(keys, first, last):
    a = np.array(keys, dtype=np.float64)
    mid = first + (last - first) // 2
    x, y, z = first + 1, mid, last - 1
    if a[x] < a[y]:
        m = y if a[y] < a[z] else (z if a[x] < a[z] else x)
    else:
        m = x if a[x] < a[z] else (z if a[y] < a[z] else y)
    a[[first, m]] = a[[m, first]]
    pivot = a[first]
    seg = a[first + 1:last]
    is_l = ~(seg < pivot)
    is_r = ~(pivot < seg)
    cl = np.concatenate([[0], np.cumsum(is_l)])[:-1]      # left stops before x
    cr = np.concatenate([[0], np.cumsum(is_r)])[:-1]      # right stops before x
    total_r = int(is_r.sum())
    k = int(np.max(np.minimum(cl, total_r - cr))) if len(seg) else 0
    lpos = np.flatnonzero(is_l) + first + 1
    rpos = (np.flatnonzero(is_r) + first + 1)[::-1]
    for q in range(k):
        a[[lpos[q], rpos[q]]] = a[[rpos[q], lpos[q]]]
    nxt = lpos[k] if k < len(lpos) else np.iinfo(np.int64).max
    cut = min(nxt, rpos[k - 1] if k > 0 else last)
    return list(a), int(cut)


def test_partition_restatement_matches_sequential_hoare():
    rng = np.random.default_rng(5)
    for trial in range(3000):
        n = int(rng.integers(4, 60))
        levels = int(rng.integers(1, 8)) if trial % 3 else 1000
        keys = list(rng.integers(0, levels, n).astype(np.float64))
        first = int(rng.integers(0, 3))
        keys = [float(v) for v in rng.integers(0, levels, first)] + keys
        last = len(keys)
        if last - first <= 3:
            continue
        a_seq, cut_seq = sequential(keys, first, last)
        a_par, cut_par = restated(keys, first, last)
        assert cut_seq == cut_par, (keys, first, last)
        assert a_seq == a_par, (keys, first, last)
