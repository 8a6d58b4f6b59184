"""CPU checks of the tensor-core F stage's shared-memory and TMEM layout arithmetic
(difx_tests_b200/csrc/fx_ftc.cu), restated here from the kernel's formulas: every role
writes and reads the rows and swizzled 16-byte chunks the other roles expect, the
stores land in distinct shared-memory banks, and the staged-input reads stay inside the
staging buffer for every sample offset.  A change to one role's index mapping that the
others do not follow fails here before any GPU run."""
import itertools

F = 2048          # FFT length
F1, F2 = 32, 64   # n = 64 n1 + n2, k = k1 + 32 k2
TB = 16           # FFTs per work item
INB = 544         # staged bytes per FFT


def a1_row(b, o, i2):
    """A1 row of sample n2 = 4 o + i2 of FFT b of a pair (producer)."""
    return b * 64 + 8 * i2 + (o & 7) + 32 * (o >> 3)


def sw128(r, c):
    """Byte offset of 16-byte chunk c of row r in a K-major SWIZZLE_128B tile."""
    return r * 128 + ((c ^ (r & 7)) << 4)


def twiddle_row_to_n2(r):
    """(b % 2, n2) of D1 row r as the twiddle warps decode it."""
    bl, rr = r >> 6, r & 63
    return bl, 4 * ((rr & 7) + 8 * (rr >> 5)) + ((rr >> 3) & 3)


def test_a1_rows_are_a_bijection_the_twiddle_inverts():
    rows = {a1_row(b, o, i2) for b in range(2) for o in range(16) for i2 in range(4)}
    assert rows == set(range(128))
    for r in range(128):
        bl, n2 = twiddle_row_to_n2(r)
        assert a1_row(bl, n2 // 4, n2 % 4) == r


def test_producer_quarter_warps_store_to_eight_bank_groups():
    # thread tp: FFT tp >> 6, o = tp & 15, h = (tp & 63) >> 4; store (i2, jj) writes row a1_row(.., o, i2),
    # chunk 2 h + jj.  A 16-byte store is served a quarter-warp (8 lanes) at a time.
    for warp, i2, jj in itertools.product(range(4), range(4), range(2)):
        for q in range(4):
            banks = set()
            for lane in range(8 * q, 8 * q + 8):
                tp = 32 * warp + lane
                b, o, h = tp >> 6, tp & 15, (tp & 63) >> 4
                off = sw128(a1_row(b, o, i2), 2 * h + jj)
                banks.add((off % 128) // 16)      # 16-byte bank group within the 128-byte line
            assert len(banks) == 8, (warp, i2, jj, q)


def test_twiddle_stores_fill_a2_without_conflicts_and_cover_every_element():
    seen = set()
    for p, k1 in itertools.product(range(TB // 2), range(F1)):
        for q in range(4):                        # warp q of the twiddle group: D1 lanes 32q..32q+31
            words = set()
            for lane in range(32):
                bl, n2 = twiddle_row_to_n2(32 * q + lane)
                b = 2 * p + bl
                R = ((k1 & 7) << 4) + b
                khalf, cl, wd = n2 >> 5, (n2 & 31) >> 2, n2 & 3
                off = sw128(R, cl) + wd * 4
                words.add(off // 4 % 32)          # 4-byte bank
                seen.add((k1 >> 3, khalf, off))
            assert len(words) == 32               # one store instruction, 32 distinct banks
    # every (tile, K half, row, 4-byte word) of A2 written exactly once per item
    assert len(seen) == 4 * 2 * 128 * 32


def test_output_rows_match_a2_rows():
    # step-2 row R of tile j = (k1 % 8, b); the output thread of TMEM lane r takes k1 % 8 = r >> 4, b = r & 15
    for r in range(128):
        kl, b = r >> 4, r & 15
        assert ((kl & 7) << 4) + b == r


def test_staged_input_reads_stay_inside_the_buffer():
    # window: base = (offset >> 2) & ~15, nvec = (F/4 + 1 + first - base + 15) >> 4 vectors of 16 bytes;
    # bit of sample 0 in the window P = 2 (offset - 4 base); thread (o, h) reads words w0 + 4 n1 and + 1
    for offset in range(0, 256):
        first = offset >> 2
        base = first & ~15
        nvec = (F // 4 + 1 + (first - base) + 15) >> 4
        assert 16 * nvec <= INB - 16
        p_bit = 2 * (offset - 4 * base)
        for o, h in itertools.product(range(16), range(4)):
            w0 = (p_bit + 8 * o) >> 5
            sh = (p_bit + 8 * o) & 31
            for i1 in range(8):
                idx = w0 + 4 * (8 * h + i1)
                assert 4 * (idx + 2) <= INB              # the second word of the funnel shift is in the buffer
                last_bit = 32 * idx + sh + 7             # the 8 bits (4 samples) this read uses
                assert last_bit < 8 * 16 * nvec          # ... lie inside the copied window


# --------------------------------------------------------------------------------------------
# FP32-grade tensor-core F stage (difx_tests_b200/csrc/fx_ftc32.cu): 8-FFT items, A1 in TMEM
# (lane = row (b, n2) of the pair), A2 tiles of rows 8 (k1 % 16) + b, two FP16 limbs.
TB32 = 8


def test_tc32_producer_reads_stay_inside_the_staged_window():
    # sample 64 n1 + n2 at bit wv + 128 n1 + 2 n2; the thread reads word (wv + 2 n2) / 32 + 4 n1
    # and two bits at shift (wv + 2 n2) % 32; wv = 2 (offset - 4 base), offset - 4 base < 64
    for d in range(64):                    # offset - 4 * base: (first - base) * 4 + offset % 4
        wv = 2 * d
        first_minus_base, rem = divmod(d, 4)
        nvec = (F // 4 + 1 + first_minus_base + 15) // 16
        copied = 16 * nvec
        assert copied <= INB
        for n2 in range(64):
            bit = wv + 2 * n2
            sh = bit % 32
            assert sh <= 30                     # the two bits never straddle a word
            for n1 in range(F1):
                w = bit // 32 + 4 * n1
                assert 4 * w + 3 < INB          # the word is inside the staging buffer
                # the sample's own bits are inside the copied bytes
                sbit = bit + 128 * n1
                assert (sbit + 1) // 8 < copied


def tc32_a2_offset(R, n2):
    """Byte of (row R, K element (n2, re|im)) in the 16 KB buffer of K half n2 // 32 (twiddle store)."""
    col = (((n2 & 31) >> 2) << 4) + 4 * (n2 & 3)
    return R * 128 + (col ^ ((R & 7) << 4))


def test_tc32_a2_stores_cover_each_tile_once_and_match_the_mma_layout():
    for khalf in range(2):
        seen = set()
        for R in range(128):
            for n2 in range(32 * khalf, 32 * khalf + 32):
                o = tc32_a2_offset(R, n2)
                assert 0 <= o and o + 4 <= 128 * 128
                # the MMA reads K element 2 (n2 % 32) + c of row R from chunk (n2 % 32) // 4 swizzled
                assert o == sw128(R, (n2 & 31) >> 2) + 4 * (n2 & 3)
                seen.add(o)
        assert len(seen) == 128 * 32             # every 4-byte word of the K half exactly once


def test_tc32_twiddle_warp_stores_hit_distinct_banks():
    # one store instruction of a twiddle warp: 32 lanes = 32 consecutive n2 (same K half), one row R
    for q in range(4):
        for R in range(128):
            banks = {(tc32_a2_offset(R, 32 * (q & 1) + lane) // 4) % 32 for lane in range(32)}
            assert len(banks) == 32


def test_tc32_rows_and_tmem_columns():
    # D1 / A1 rows: lane r = 64 b + n2 of the pair; twiddle warp quarter q covers FFT q // 2,
    # n2 = 32 (q % 2) + lane; A2 / D2 rows 8 kl + b of tile k1 // 16; output lane r -> (r // 8, r % 8)
    a1 = {(r >> 6, r & 63) for r in range(128)}
    assert a1 == {(b, n2) for b in range(2) for n2 in range(64)}
    tw = {(q >> 1, 32 * (q & 1) + lane) for q in range(4) for lane in range(32)}
    assert tw == a1
    rows = {(8 * kl + b) for kl in range(16) for b in range(TB32)}
    assert rows == set(range(128))
    out = {(r >> 3, r & 7) for r in range(128)}
    assert out == {(kl, b) for kl in range(16) for b in range(TB32)}
    # TMEM: A1 2 stages x 64, D1 4 pairs x 64, D2 2 tiles x 64 inside the 512 allocated columns
    a1c = [(64 * s, 64 * s + 64) for s in range(2)]
    d1c = [(128 + 64 * p, 128 + 64 * p + 64) for p in range(TB32 // 2)]
    d2c = [(384 + 64 * j, 384 + 64 * j + 64) for j in range(2)]
    spans = sorted(a1c + d1c + d2c)
    assert spans[0][0] == 0 and spans[-1][1] == 512
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


def test_tc32_output_indices_cover_the_item_once():
    # F16 layout [chan][row][T]: output thread (k1 = 16 j + kl, b) writes channel k1 + 32 k2 of slot tb0 + b
    for j in range(2):
        got = {(16 * j + (r >> 3) + 32 * k2, r & 7) for r in range(128) for k2 in range(32)}
        assert len(got) == 16 * 32 * TB32
    allk = {(16 * j + (r >> 3) + 32 * k2) for j in range(2) for r in range(128) for k2 in range(32)}
    assert allk == set(range(1024))


def test_tc32_output_boxes_cover_the_item_once_and_store_conflict_free():
    # FP16 output: output warp w = 4 g + q (group g, TMEM lane quarter q) takes D2 columns 32 g ..
    # 32 g + 31 (k2 = 16 g + kk) of its 32 rows (kl = 4 q + lane // 8, b = lane % 8) of tile j; it
    # writes half (kk, kl % 4, c, b) at kk * 64 + (lane // 8) * 16 + c * 8 + b of a 1024-half box
    # [k2 % 16][k1 % 4][re|im][b], stored by one tensor store at (T = tb0, row 2 ant, k1 = 16 j + 4 q,
    # 32 sb + 16 g) with box extents (8, 2, 4, 16).
    covered = set()
    for j in range(2):
        for g in range(2):
            for q in range(4):
                box = {}
                for lane in range(32):
                    kl, b = 4 * q + lane // 8, lane % 8
                    for kk in range(16):
                        for c in range(2):
                            idx = kk * 64 + (lane // 8) * 16 + c * 8 + b
                            assert 0 <= idx < 16 * 4 * 2 * TB32
                            # the tensor store's box order (T innermost, then row, k1, k2)
                            t_, r_, z_, w_ = idx % 8, (idx // 8) % 2, (idx // 16) % 4, idx // 64
                            assert (t_, r_, z_, w_) == (b, c, kl % 4, kk)
                            k1 = 16 * j + 4 * q + z_
                            k2 = 16 * g + w_
                            box[idx] = (k1 + 32 * k2, c, b)
                assert len(box) == 1024 and len(set(box.values())) == 1024
                covered |= set(box.values())
                # one store instruction (fixed kk, c): 32 lanes, four 16-byte runs 32 bytes apart,
                # so each 4-byte bank word is shared by one lane pair only and 16 distinct banks
                for kk in range(16):
                    for c in range(2):
                        words = [(kk * 64 + (lane // 8) * 16 + c * 8 + lane % 8) // 2 for lane in range(32)]
                        assert len(set(words)) == 16 and len({w % 32 for w in words}) == 16
    assert covered == {(k, c, b) for k in range(1024) for c in range(2) for b in range(TB32)}
    # box origins: k1 = 16 j + 4 q in [0, 28], k2 = 16 g in {0, 16}: boxes stay inside the 32 x 32 channel grid
    assert max(16 * j + 4 * q + 4 for j in range(2) for q in range(4)) <= 32
