"""CPU check of the plain X stage's tile plan (difx_tests_b200/csrc/fx_xplain.cu), restated from
the kernel's decode: every signal pair i <= j of a channel is accumulated by exactly one thread,
and with 8 (or 4) blocks of 8 signals the diagonal-pair threads fill whole warps (their branch
is warp-uniform) and the CTA is 8 warps.  Also the library's time-segment cut of the stage for jobs
whose channel groups fill the SMs poorly (through its debug entry point, host arithmetic only)."""


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


def lib_segments(ctas, slots, T):
    import ctypes as C
    import difx_tests_b200 as fx
    ts, tl = C.c_int(), C.c_int()
    assert fx.lib().fxc_debug_xplain_segments(ctas, slots, T, C.byref(ts), C.byref(tl)) == 0
    return ts.value, tl.value


def model_cost(ctas, slots, T, tlen):
    nseg = -(-T // tlen)
    return -(-ctas * nseg // slots) * (tlen + 32)


def test_segment_cut_is_the_cheapest_of_the_model():
    """The library's time-segment cut of the plain X stage (fx_xplain.cu xplain_segment_model): the
    segments cover the T slots in lengths that are multiples of 16 and at least 64, at most 32 of
    them, and no cut of the same family costs fewer waves x (length + 32) slots."""
    for ctas in (1, 8, 24, 48, 64, 128, 148, 200, 296, 1024):
        for slots in (148, 296, 888):
            for T in (64, 128, 512, 1024, 3136, 4096):
                tseg, tlen = lib_segments(ctas, slots, T)
                if tseg == 1:
                    assert tlen == T
                else:
                    assert tlen % 16 == 0 and tlen >= 64 and 2 <= tseg <= 32
                    assert (tseg - 1) * tlen < T <= tseg * tlen
                cands = [T] + [-(-(-(-T // s)) // 16) * 16 for s in range(2, 33) if -(-(-(-T // s)) // 16) * 16 >= 64]
                best = min(model_cost(ctas, slots, T, L) for L in cands)
                assert model_cost(ctas, slots, T, tlen) == best


def test_segment_cut_examples():
    assert lib_segments(8, 888, 3136) == (28, 112)       # 4 ant x 256 ch: 224 CTAs, one wave
    assert lib_segments(24, 148, 4096) == (6, 688)       # 24 sig x 128 ch x 6 sb: one full wave
    assert lib_segments(1024, 148, 512) == (1, 512)      # 64 sig x 1024 ch x 8 sb: no cut
    assert lib_segments(10, 148, 64) == (1, 64)          # chunks shorter than 128 slots: no cut
