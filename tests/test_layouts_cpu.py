"""Shared-memory layouts of the in-place correlation windows (xrw_cfg,
xch_in_column / xch_in_row and xrw_window's row map in
packed_b200/csrc/pcx_ragged.cu, restated here): the slot map is a permutation
inside the window's column (row), and the 8-byte accesses of a half-warp --
16 lanes, one 128-byte wavefront -- fall on 32 distinct banks for the writes
(slot 16t + j) and reads (slot t + TT*i) of the exchange.  Two window shapes:
8192 points (one window of 128 rows x 64 columns, row stride 66 complex) and
4096 points (two windows of 64 x 64, row stride 68)."""
import pytest

NT = 512    # compute threads of the ragged kernel


def cfg(logn):
    n1, n2 = 1 << ((logn + 1) // 2), 1 << (logn // 2)
    tt1, tt2 = n1 // 16, n2 // 16
    w = 8192 // (n1 * n2)
    rs = n2 + (2 if tt1 == 8 else 4)
    return dict(N1=n1, N2=n2, TT1=tt1, TT2=tt2, W=w, RS=rs)


CFGS = [cfg(13), cfg(12)]


def col_slot(c, m, l):
    sw = c["TT1"] - 1
    return (l ^ ((l >> 4) & sw)) * c["RS"] + m


def row_slot(c, m, l):
    sw = c["TT2"] - 1
    return m * c["RS"] + (l ^ ((l >> 4) & sw))


def row_of_group(c, g):
    """The stacked row (window * N1 + k1) that row group g transforms."""
    if c["RS"] % 16 == 2:
        s, u_n = c["TT2"] // 2, 16 // c["TT2"]
        bb, u = g // u_n, g % u_n
        return (bb // s) * 8 + (bb % s) + u * s
    return g


def banks(addrs):
    out = []
    for a in addrs:    # complex64: two 4-byte banks per element
        out += [(2 * a) % 32, (2 * a + 1) % 32]
    return out


def conflict_free(addrs):
    b = banks(addrs)
    return len(b) == len(set(b))


@pytest.mark.parametrize("c", CFGS, ids=["8192", "4096"])
def test_shapes_fill_the_threads(c):
    assert c["W"] * c["N2"] * c["TT1"] == NT
    assert c["W"] * c["N1"] * c["TT2"] == NT
    assert c["W"] * c["N1"] * c["RS"] * 8 <= 69632    # one ring stage


@pytest.mark.parametrize("c", CFGS, ids=["8192", "4096"])
def test_slot_maps_are_permutations(c):
    assert sorted(l ^ ((l >> 4) & (c["TT1"] - 1)) for l in range(c["N1"])) == list(range(c["N1"]))
    assert sorted(l ^ ((l >> 4) & (c["TT2"] - 1)) for l in range(c["N2"])) == list(range(c["N2"]))


@pytest.mark.parametrize("c", CFGS, ids=["8192", "4096"])
def test_column_exchange_banks(c):
    tt1 = c["TT1"]
    per_half = 16 // tt1    # column groups in a half-warp: consecutive columns
    for half in range(NT // 16):
        groups = [(16 * half) // tt1 + k for k in range(per_half)]
        cols = [(g // c["N2"], g % c["N2"]) for g in groups]
        base = lambda w: w * c["N1"] * c["RS"]
        for j in range(16):
            assert conflict_free([base(w) + col_slot(c, n2, 16 * t + j) for w, n2 in cols for t in range(tt1)])
        for i in range(16):
            assert conflict_free([base(w) + col_slot(c, n2, t + tt1 * i) for w, n2 in cols for t in range(tt1)])


@pytest.mark.parametrize("c", CFGS, ids=["8192", "4096"])
def test_row_exchange_banks_and_cover(c):
    tt2 = c["TT2"]
    covered = set()
    for half in range(NT // 16):
        rt = []
        for lane in range(16):
            tid = 16 * half + lane
            rt.append((row_of_group(c, tid // tt2), tid % tt2))
        covered |= {r for r, _ in rt}
        for j in range(16):
            assert conflict_free([row_slot(c, r, 16 * t + j) for r, t in rt])
        for i in range(16):
            assert conflict_free([row_slot(c, r, t + tt2 * i) for r, t in rt])
    assert covered == set(range(c["W"] * c["N1"]))
