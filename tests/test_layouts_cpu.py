"""Shared-memory layouts of the in-place correlation windows (xch_in_column /
xch_in_row in packed_b200/csrc/pcx_ragged.cu, restated here): the slot map is a
permutation inside the window's column (row), and the 8-byte accesses of a
half-warp -- 16 lanes, one 128-byte wavefront -- fall on 32 distinct banks for
the writes (slot 16t + j) and reads (slot t + TT*i) of the exchange, for the
8192-point window (128 rows x 64 columns, row stride 66 complex)."""

RS, N1, N2, TT1, TT2 = 66, 128, 64, 8, 4


def col_slot(m, l, sw=TT1 - 1):
    return (l ^ ((l >> 4) & sw)) * RS + m


def row_slot(m, l, sw=TT2 - 1):
    return m * RS + (l ^ ((l >> 4) & sw))


def banks(addrs):
    out = []
    for a in addrs:    # complex64: two 4-byte banks per element
        out += [(2 * a) % 32, (2 * a + 1) % 32]
    return out


def conflict_free(addrs):
    b = banks(addrs)
    return len(b) == len(set(b))


def test_slot_maps_are_permutations():
    assert sorted(l ^ ((l >> 4) & (TT1 - 1)) for l in range(N1)) == list(range(N1))
    assert sorted(l ^ ((l >> 4) & (TT2 - 1)) for l in range(N2)) == list(range(N2))


def test_column_exchange_banks():
    # a half-warp holds two column groups (columns n2, n2 + 1) of 8 threads
    for n2 in range(0, N2, 2):
        for j in range(16):
            assert conflict_free([col_slot(g, 16 * t + j) for g in (n2, n2 + 1) for t in range(TT1)])
        for i in range(16):
            assert conflict_free([col_slot(g, t + TT1 * i) for g in (n2, n2 + 1) for t in range(TT1)])


def test_row_exchange_banks_and_cover():
    # row groups of 4 threads; a half-warp's four groups take rows 2 apart
    def rows_of(half):
        out = []
        for lane in range(16):
            tid = 16 * half + lane
            g, t = tid // TT2, tid % TT2
            bb, u = g // 4, g % 4
            out.append(((bb // 2) * 8 + (bb % 2) + 2 * u, t))
        return out
    covered = set()
    for half in range(512 // 16):
        rt = rows_of(half)
        covered |= {r for r, _ in rt}
        for j in range(16):
            assert conflict_free([row_slot(r, 16 * t + j) for r, t in rt])
        for i in range(16):
            assert conflict_free([row_slot(r, t + TT2 * i) for r, t in rt])
    assert covered == set(range(N1))
