"""CPU check of the index arithmetic of the tensor-core X stage on FP32 spectra
(difx_tests_b200/csrc/fx_xtc32.cu, k_xtc32), restated from the kernel: the FP32 stage ring fits its
shared-memory region, the cast's reads stay inside a stage, its stores fill every 4-byte word of K
half h of rows < 2 nsig of each channel's FP16 tile exactly once, with the FFT pair the K-major
SWIZZLE_128B layout puts there, and take at most two bank passes."""
import pytest

BT, CB, MAXSIG, NCW = 32, 4, 64, 8
RING_BYTES = 2 * MAXSIG * BT * CB * 8
MAXS32 = 8


def stage_bytes(nsig):
    return nsig * BT * CB * 8


def ns32(nsig):
    return min(MAXS32, RING_BYTES // stage_bytes(nsig))


def sw128(row, chunk):
    """Byte offset of 16-byte chunk `chunk` of row `row` in a K-major SWIZZLE_128B tile."""
    return row * 128 + ((chunk ^ (row & 7)) << 4)


def cast_ops(nsig, h):
    """(reads, writes) of one FP32 stage's cast into K half h: reads = [(warp, lane, byte)],
    writes = [(warp, lane, instruction, byte_in_tile, fft_lo, channel_slot)] with fft_lo the first
    of the two FFTs (within the 64-FFT tile row) the written word holds."""
    reads, writes = [], []
    for warp in range(2, 2 + NCW):
        for s0 in range(warp - 2, nsig, 4 * NCW):
            for u in range(4):
                if s0 + NCW * u >= nsig:
                    break
                for lane in range(32):
                    t = lane
                    s = s0 + NCW * u
                    reads.append((warp, lane, s * 1024 + t * 32))
                    reads.append((warp, lane, s * 1024 + t * 32 + 16))
                    w = lane & 3
                    part = (lane >> 2) & 1
                    src_a = (lane & ~7) + 2 * w
                    k = 4 * h + (t >> 3)
                    row = 2 * s + part
                    off = sw128(row, k) + 4 * w
                    for c in range(CB):
                        writes.append((warp, lane, (s0, u, c), off, 32 * h + src_a, c, row))
    return reads, writes


@pytest.mark.parametrize("nsig", [1, 2, 3, 7, 8, 16, 31, 32, 33, 63, 64])
def test_ring_fits(nsig):
    assert 1 <= ns32(nsig) <= MAXS32
    assert ns32(nsig) * stage_bytes(nsig) <= RING_BYTES
    assert stage_bytes(nsig) % 1024 == 0          # every stage starts 128-byte aligned for the copy engine
    assert (nsig <= 32) == (ns32(nsig) >= 4)


@pytest.mark.parametrize("nsig", [1, 5, 16, 32, 33, 64])
@pytest.mark.parametrize("h", [0, 1])
def test_cast_reads_inside_the_stage_and_writes_each_word_once(nsig, h):
    reads, writes = cast_ops(nsig, h)
    assert all(0 <= b and b + 16 <= stage_bytes(nsig) for _, _, b in reads)
    per_tile = {}
    for _, _, _, off, fft_lo, c, row in writes:
        per_tile.setdefault(c, []).append((off, fft_lo, row))
    for c in range(CB):
        offs = [o for o, _, _ in per_tile[c]]
        assert len(offs) == len(set(offs)), "a word written twice"
        want = {sw128(r, k) + 4 * w for r in range(2 * nsig) for k in range(4 * h, 4 * h + 4) for w in range(4)}
        assert set(offs) == want
        for off, fft_lo, row in per_tile[c]:
            # the K-major layout: FFT f of row r is the 2-byte element f of the row's logical chunks
            chunk_phys = (off % 128) >> 4
            chunk = chunk_phys ^ (row & 7)
            assert fft_lo == 8 * chunk + ((off % 16) >> 2) * 2
            assert 0 <= fft_lo < 64 and fft_lo % 2 == 0


@pytest.mark.parametrize("nsig", [8, 32, 64])
def test_cast_store_bank_conflicts_are_at_most_two_way(nsig):
    """A warp's 4-byte store: the 8 lanes of one FFT group hit 8 different banks (Re and Im rows take
    different swizzled chunks); across the warp's 4 groups the chunks of FFT groups g and g ^ 1 meet
    (Re row of one, Im row of the other), so a store takes at most 2 bank passes."""
    _, writes = cast_ops(nsig, 0)
    groups, warps = {}, {}
    for warp, lane, instr, off, _, _, _ in writes:
        groups.setdefault((warp, instr, lane >> 3), []).append(off)
        warps.setdefault((warp, instr), []).append(off)
    for offs in groups.values():
        assert len({(o // 4) % 32 for o in offs}) == len(offs)
    for offs in warps.values():
        banks = {}
        for o in set(offs):
            banks[(o // 4) % 32] = banks.get((o // 4) % 32, 0) + 1
        assert max(banks.values()) <= 2


def test_zeroed_rows_are_the_rest_of_the_tile():
    for nsig in (1, 17, 64):
        written = {sw128(r, k) for r in range(2 * nsig) for k in range(8)}
        zeroed = {(2 * nsig + rem // 8) * 128 + (rem % 8) * 16 for rem in range((128 - 2 * nsig) * 8)}
        assert not written & zeroed
        assert len(written | zeroed) == 128 * 8
