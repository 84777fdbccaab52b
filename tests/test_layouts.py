"""Shared-memory layouts of the 8x8 kernels, restated in Python: the index
maps the kernels use must be bijective and send the 32 lanes of each access
phase to 32 different banks (4-byte words; 64-bit words take bank pairs and
are served per half-warp). These are the layout claims the kernels' comments
make (group8.cu Shape::at, finish.cu vs_col / vs_pitch, match8.cu swz)."""
import pytest


def group_at(G, row, col):
    lp = 32 // G
    rpl = 8 // lp
    return row * 8 + (col ^ (row // rpl))


@pytest.mark.parametrize("G", [4, 8, 16])
def test_group_cube_is_a_permutation_per_patch(G):
    assert sorted(group_at(G, r, c) for r in range(8) for c in range(8)) == list(range(64))


@pytest.mark.parametrize("G", [4, 8, 16])
def test_group_cube_phases_conflict_free(G):
    lp, rpl = 32 // G, 8 // (32 // G)
    S = 64 + lp
    lanes = [(lane // lp, lane % lp) for lane in range(32)]  # (patch g, lane in patch q)
    # row phase: lane (g, q) owns rows q*RPL + r and walks j
    for r in range(rpl):
        for j in range(8):
            banks = {(g * S + group_at(G, q * rpl + r, j)) % 32 for g, q in lanes}
            assert len(banks) == 32, ("row", G, r, j)
    # column phase: lane (g, q) owns columns q + LP*t and walks the rows i
    for t in range(rpl):
        for i in range(8):
            banks = {(g * S + group_at(G, i, q + lp * t)) % 32 for g, q in lanes}
            assert len(banks) == 32, ("column", G, t, i)
    # tube phase: lane l reads coefficient f = l + 32h of every patch gg
    for h in range(2):
        for gg in range(G):
            banks = {(gg * S + group_at(G, (l + 32 * h) >> 3, (l + 32 * h) & 7)) % 32 for l in range(32)}
            assert len(banks) == 32, ("tube", G, h, gg)


def vs_col(cc):
    return cc + (cc >> 3)


def vs_pitch(B, fx=64):
    return (vs_col(fx + B - 2) + 1 + 7) // 16 * 16 + 8


@pytest.mark.parametrize("B", [1, 2, 4, 8, 12, 16, 32])
def test_finish_table_fits_and_is_conflict_free(B):
    pitch = vs_pitch(B)
    assert pitch % 16 == 8 and pitch >= vs_col(64 + B - 2) + 1
    # horizontal phase: thread t -> row t >> 3, segment t & 7; 64-bit words,
    # one half-warp (2 rows x 8 segments) per wavefront: 16 distinct bank pairs
    for half in range(0, 256, 16):
        for k in range(8 + B - 1):
            pairs = set()
            for t in range(half, half + 16):
                r, seg = t >> 3, t & 7
                pairs.add((2 * (r * pitch + vs_col(8 * seg + k))) % 32)
            assert len(pairs) == 16, (B, half, k)


def swz(c):
    return c ^ ((c >> 5) & 3)


def test_matcher_tile_swizzle_conflict_free():
    # 32 lanes read 32 columns 4 apart (two lanes per reference, references 8
    # columns apart) at any starting column of the window walk
    for start in range(0, 288 - 4 * 31):
        banks = {swz(start + 4 * lane) % 32 for lane in range(32)}
        assert len(banks) == 32, start
    # the swizzle stays inside each aligned group of 4 columns
    for c in range(288):
        assert swz(c) >> 2 == c >> 2
