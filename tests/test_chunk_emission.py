"""The instance pass's chunk records (k_instances in csrc/vgcut_kernels.cu): a warp lays its 32 items (one per lane,
lengths n, some empty) end to end, cuts them into windows of 2^shift meshlets and writes, for chunk t, the index of its
first span record and its span count. The kernel finds them lane-parallel, with three searches over the lanes' sorted
item starts and ends; restated here, they must equal the serial definition (the last item starting at or before the
window, the windows that item crossed before it, the non-empty items meeting the window) on random warps."""
import numpy as np
import pytest


def layout(ns, shift):
    st = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    spans = np.array([((s + n - 1) >> shift) - (s >> shift) + 1 if n else 0 for s, n in zip(st, ns)])
    q = np.concatenate([[0], np.cumsum(spans)[:-1]])
    total = int(np.sum(ns))
    return st, q, (total + (1 << shift) - 1) >> shift


def serial(ns, shift):
    st, q, N = layout(ns, shift)
    chunk = 1 << shift
    out = []
    for t in range(N):
        X = t << shift
        owner = max(j for j in range(32) if st[j] <= X)
        spans = sum(1 for j in range(32) if ns[j] > 0 and st[j] < X + chunk and st[j] + ns[j] > X)
        out.append((int(q[owner] + t - (st[owner] >> shift)), spans))
    return out


def lane_parallel(ns, shift):
    st, q, N = layout(ns, shift)
    chunk = 1 << shift
    e = st + np.asarray(ns)
    nonempty = sum(1 << j for j in range(32) if ns[j] > 0)
    out = []
    for t in range(N):
        X = t << shift
        owner = a = b = 0
        for step in (16, 8, 4, 2, 1):  # last lane with st <= X; with st < X + chunk; with st + n <= X
            if st[owner + step] <= X:
                owner += step
            if st[a + step] < X + chunk:
                a += step
            if e[b + step] <= X:
                b += step
        below = lambda j: bin(nonempty & ((2 << j) - 1)).count("1")
        before = below(b) if e[0] <= X else 0
        out.append((int(q[owner] + t - (st[owner] >> shift)), below(a) - before))
    return out


@pytest.mark.parametrize("shift", [6, 8, 9, 10])
def test_lane_parallel_chunk_records_equal_the_serial_ones(shift):
    rng = np.random.default_rng(shift)
    choices = [0, 0, 1, 3, 17, 64, 200, 511, 512, 513, 1500]
    for trial in range(600):
        ns = [int(rng.choice(choices)) if rng.random() < 0.8 else int(rng.integers(0, 5000)) for _ in range(32)]
        if trial % 5 == 0:  # one long item among empty ones
            ns = [0] * 32
            ns[int(rng.integers(32))] = int(rng.integers(1, 9000))
        if sum(ns) == 0:
            continue
        assert lane_parallel(ns, shift) == serial(ns, shift), (ns, shift)
