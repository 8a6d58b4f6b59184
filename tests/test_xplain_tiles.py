"""CPU check of the plain X stage's tile plan (difx_tests_b200/csrc/fx_xplain.cu), restated from
the kernel's decode: every signal pair i <= j of a channel is accumulated by exactly one thread,
and with 8 (or 4) blocks of 8 signals the diagonal-pair threads fill whole warps (their branch
is warp-uniform) and the CTA is 8 warps."""


def decode(tile, nb):
    """(kind, I, J) of a thread's tile: 'tile' = the I x J block pair, 'pair' = the upper triangles of
    diagonal blocks I and J."""
    paired = nb in (4, 8)
    noff = nb * (nb - 1) // 2
    if paired and tile >= noff:
        i = tile - noff
        return "pair", i, nb - 1 - i
    lead = 1 if paired else 0
    i, rem = 0, tile
    while rem >= nb - lead - i:
        rem -= nb - lead - i
        i += 1
    return "tile", i, i + lead + rem


def ntile(nb):
    return nb * (nb - 1) // 2 + nb // 2 if nb in (4, 8) else nb * (nb + 1) // 2


def test_every_pair_once():
    for nb in range(1, 9):
        nsig = 8 * nb
        seen = {}
        for t in range(ntile(nb)):
            kind, I, J = decode(t, nb)
            if kind == "pair":
                cells = [(8 * B + ii, 8 * B + jj) for B in (I, J) for jj in range(8) for ii in range(jj + 1)]
            else:
                cells = [(8 * I + ii, 8 * J + jj) for ii in range(8) for jj in range(8) if 8 * I + ii <= 8 * J + jj]
            for c in cells:
                seen[c] = seen.get(c, 0) + 1
        want = {(i, j) for i in range(nsig) for j in range(i, nsig)}
        assert set(seen) == want
        assert all(v == 1 for v in seen.values())


def test_paired_plan_is_eight_whole_warps():
    cg = 8                                   # channels per CTA of the 64-signal plans
    kinds = [decode(tid // cg, 8)[0] for tid in range(ntile(8) * cg)]
    assert len(kinds) == 256
    for w in range(8):
        assert len(set(kinds[32 * w: 32 * w + 32])) == 1


def test_paired_plan_of_four_blocks_is_whole_warps():
    for cg, nthreads in ((32, 256), (16, 128)):       # the two 32-signal plans
        kinds = [decode(tid // cg, 4)[0] for tid in range(ntile(4) * cg)]
        assert len(kinds) == nthreads
        for w in range(nthreads // 32):
            assert len(set(kinds[32 * w: 32 * w + 32])) == 1
