"""The host entropy path: the library's range coder, its frame-initial CDF set
and the tile packer against the oracle's range decoder (OdEcDecoder,
src/odec.rs:615-760) and its own assembly of Cdfs::new.  The round trips
restate the reference's tests (src/odec.rs:763-921: the rav1e boolean case,
signed sub-exponential with reference, literals, fixed and adaptive symbols,
a mixed stream); the packer is checked against live coding of the same
symbols (the reference's tokens == live entropy coding property,
src/coder/aq_tests.rs:330) and by decoding its payload.  No device call."""
import numpy as np
import pytest

from maroontree_b200 import entropy as en


class XorShift:
    def __init__(self, s):
        self.s = s

    def next(self):
        s = self.s
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        self.s = s
        return s


def uniform_icdf(n):
    """src/odec.rs:35-45 uniform_icdf."""
    cdf = np.zeros(n + 1, np.uint16)
    for i in range(n):
        cdf[i] = 32768 - ((i + 1) * 32768) // n
    return cdf


def test_bool_roundtrip_reference_case(mt_lib, oracle_lib):
    cases = [(False, 1), (True, 2), (False, 3), (True, 1), (True, 2), (False, 3)]
    e = en.RangeEncoder()
    for v, f in cases:
        e.bool(v, f)
    d = oracle_lib.RangeDecoder(e.done())
    assert [d.bool(f) for _, f in cases] == [v for v, _ in cases]


def test_subexp_with_ref_roundtrip(mt_lib, oracle_lib):
    ranges = [(-5, 11, 3, 1), (-23, 9, -7, 2), (-17, 47, 15, 3)]
    rng = XorShift(123)
    e = en.RangeEncoder()
    cases = []
    for _ in range(20_000):
        lo, hi, mid, k = ranges[rng.next() % 3]
        v = lo + rng.next() % (hi - lo)
        e.signed_subexp_with_ref(v, lo, hi, k, mid)
        cases.append((v, lo, hi, k, mid))
    d = oracle_lib.RangeDecoder(e.done())
    for v, lo, hi, k, r in cases:
        assert d.signed_subexp_with_ref(lo, hi, k, r) == v


def test_literal_roundtrip(mt_lib, oracle_lib):
    rng = XorShift(7)
    e = en.RangeEncoder()
    vals = []
    for _ in range(20_000):
        bits = 1 + rng.next() % 16
        v = rng.next() & 0xFFFFFFFF & ((1 << bits) - 1)
        vals.append((v, bits))
        e.literal(v, bits)
    d = oracle_lib.RangeDecoder(e.done())
    assert all(d.literal(b) == v for v, b in vals)


def test_fixed_cdf_symbol_roundtrip(mt_lib, oracle_lib):
    cdf = uniform_icdf(5)
    rng = XorShift(99)
    syms = [rng.next() % 5 for _ in range(20_000)]
    e = en.RangeEncoder()
    for s in syms:
        e.symbol(s, cdf, adapt=False)
    d = oracle_lib.RangeDecoder(e.done())
    assert [d.symbol(cdf, adapt=False) for _ in syms] == syms


def test_adaptive_symbol_roundtrip(mt_lib, oracle_lib):
    rng = XorShift(0xBADC0DE)
    n = 8
    syms = []
    for _ in range(60_000):
        r = rng.next() % 100
        syms.append(0 if r < 60 else 1 if r < 80 else 2 + r % (n - 2))
    e = en.RangeEncoder()
    cdf_e = uniform_icdf(n)
    for s in syms:
        e.symbol(s, cdf_e)
    d = oracle_lib.RangeDecoder(e.done())
    cdf_d = uniform_icdf(n)
    assert [d.symbol(cdf_d) for _ in syms] == syms
    assert np.array_equal(cdf_e, cdf_d)


def test_mixed_stream_roundtrip(mt_lib, oracle_lib):
    e = en.RangeEncoder()
    cdf_e = uniform_icdf(4)
    e.symbol(2, cdf_e)
    e.bool(True, 10000)
    e.literal(0b1101, 4)
    e.symbol(0, cdf_e)
    e.literal(0x2A, 6)
    d = oracle_lib.RangeDecoder(e.done())
    cdf_d = uniform_icdf(4)
    assert d.symbol(cdf_d) == 2 and d.bool(10000) and d.literal(4) == 0b1101
    assert d.symbol(cdf_d) == 0 and d.literal(6) == 0x2A


@pytest.mark.parametrize("qctx", range(4))
def test_frame_cdf_set_matches_oracle_assembly(mt_lib, oracle_lib, qctx):
    slots = oracle_lib.cdfs_new_slots(qctx)
    data, off, lens = en.cdfs_default(qctx)
    assert len(slots) == len(off) == mt_lib.load().mt_cdf_slot_count()
    for i, want in enumerate(slots):
        assert lens[i] == len(want) and np.array_equal(data[off[i]:off[i] + lens[i]], want), i


def _random_tokens(oracle_lib, slots, rng, nsb, per_sb):
    """Superblock token streams over the real CDF set: adaptive and
    non-adapting symbols on random slots, bools, and gathered partition bools
    on the 10-symbol partition CDFs; plus each SB's read_cdef() point."""
    part = [i for i, s in enumerate(slots) if len(s) == 10]
    sbs, points = [], []
    for b in range(nsb):
        toks = []
        for _ in range(per_sb):
            kind = rng.next() % 10
            if kind < 6:
                i = rng.next() % len(slots)
                toks.append((i << 8) | (rng.next() % len(slots[i])))
            elif kind < 7:
                i = rng.next() % len(slots)
                toks.append(en.TOKEN_NOUPDATE | (i << 8) | (rng.next() % len(slots[i])))
            elif kind < 9:
                f = 1 + rng.next() % 32767
                toks.append(en.TOKEN_BOOL | (f << 1) | (rng.next() & 1))
            else:
                i = part[rng.next() % len(part)]
                toks.append(en.TOKEN_GATHERED_PARTITION | (i << 2) | (rng.next() & 3))
        sbs.append(np.array(toks, np.uint32))
        points.append(-1 if b % 3 == 2 else int(rng.next() % (per_sb + 1)))
    return sbs, points


def _decode_tokens(oracle_lib, d, slots, toks, point=-1, literal_bits=0, want_literal=None):
    for k, t in enumerate(toks):
        if k == point and literal_bits:
            assert d.literal(literal_bits) == want_literal
        tag = int(t) & (3 << 30)
        if tag in (0, en.TOKEN_NOUPDATE):
            cdf = slots[(int(t) >> 8) & 0xFFFF]
            assert d.symbol(cdf, adapt=tag == 0) == int(t) & 0xFF
        elif tag == en.TOKEN_BOOL:
            assert d.bool((int(t) >> 1) & 0xFFFF) == bool(int(t) & 1)
        else:
            p = oracle_lib.gather_split_prob(slots[(int(t) >> 2) & 0xFFFF], bool(int(t) & 1))
            assert d.bool(p) == bool(int(t) & 2)
    if point == len(toks) and literal_bits:
        assert d.literal(literal_bits) == want_literal


@pytest.mark.parametrize("qidx", [35, 70, 116, 200])
def test_packer_payload_decodes_to_its_tokens(mt_lib, oracle_lib, qidx):
    qctx = oracle_lib.qcat(qidx)
    slots = oracle_lib.cdfs_new_slots(qctx)
    rng = XorShift(qidx + 11)
    sbs, points = _random_tokens(oracle_lib, slots, rng, 12, 300)
    payload = en.pack_tile(qidx, sbs, points)
    d = oracle_lib.RangeDecoder(payload)
    for toks in sbs:
        _decode_tokens(oracle_lib, d, slots, toks)


def test_packer_equals_live_coding(mt_lib, oracle_lib):
    """The same symbols coded directly through the range encoder against a live
    copy of the frame-initial CDF set give the packer's bytes."""
    slots = oracle_lib.cdfs_new_slots(2)
    sbs, points = _random_tokens(oracle_lib, slots, XorShift(5), 6, 400)
    live = [s.copy() for s in slots]
    e = en.RangeEncoder()
    for toks in sbs:
        for t in toks:
            tag = int(t) & (3 << 30)
            if tag in (0, en.TOKEN_NOUPDATE):
                e.symbol(int(t) & 0xFF, live[(int(t) >> 8) & 0xFFFF], adapt=tag == 0)
            elif tag == en.TOKEN_BOOL:
                e.bool(int(t) & 1, (int(t) >> 1) & 0xFFFF)
            else:
                e.bool(int(t) & 2, oracle_lib.gather_split_prob(live[(int(t) >> 2) & 0xFFFF], bool(int(t) & 1)))
    assert e.done() == en.pack_tile(70, sbs, points)


def test_non_updating_cdfs(mt_lib, oracle_lib):
    slots = oracle_lib.cdfs_new_slots(1)
    sbs, points = _random_tokens(oracle_lib, slots, XorShift(9), 4, 200)
    payload = en.pack_tile(50, sbs, points, updating_cdf=False)
    d = oracle_lib.RangeDecoder(payload)
    for toks in sbs:  # every symbol decodes against the frame-initial CDFs
        _decode_tokens(oracle_lib, d, slots, [t if (int(t) >> 30) != 0 else (int(t) | en.TOKEN_NOUPDATE)
                                              for t in toks])


def test_filter_replay_inserts_cdef_literals(mt_lib, oracle_lib):
    """replay_tile_with_filters: without a grid the trace re-emits the packer's
    bytes; with one, each SB with a read_cdef() point carries its unit's
    cdef_idx literal there."""
    slots = oracle_lib.cdfs_new_slots(2)
    w, h = 64 * 4, 64 * 3
    sbs, points = _random_tokens(oracle_lib, slots, XorShift(21), 12, 150)
    payload, trace = en.pack_tile(70, sbs, points, want_trace=True)
    assert en.replay_tile_with_filters(trace, (0, 0, w, h)) == payload
    bits = 3
    grid = np.array([(7 * k + 3) % 8 for k in range(12)], np.uint8)
    out = en.replay_tile_with_filters(trace, (0, 0, w, h), grid, unit_cols=4, cdef_bits=bits)
    d = oracle_lib.RangeDecoder(out)
    for k, toks in enumerate(sbs):
        _decode_tokens(oracle_lib, d, slots, toks, points[k], bits if points[k] >= 0 else 0, int(grid[k]))


@pytest.mark.parametrize("bits,updating", [(0, True), (1, True), (2, False), (3, True)])
def test_single_pass_filtered_pack_equals_pack_then_replay(mt_lib, oracle_lib, bits, updating):
    """mt_pack_tile_filtered gives the bytes of pack_tile followed by
    replay_tile_with_filters on a tile whose units are its superblocks."""
    slots = oracle_lib.cdfs_new_slots(1)
    w, h = 64 * 5, 64 * 3
    sbs, points = _random_tokens(oracle_lib, slots, XorShift(31 + bits), 15, 120)
    grid = np.array([(5 * k + 1) % (1 << max(bits, 1)) for k in range(15)], np.uint8)
    payload, trace = en.pack_tile(60, sbs, points, updating_cdf=updating, want_trace=True)
    want = en.replay_tile_with_filters(trace, (0, 0, w, h), grid if bits else None, unit_cols=5, cdef_bits=bits,
                                       updating_cdf=updating)
    got = en.pack_tile_filtered(60, sbs, points, grid if bits else None, bits, updating_cdf=updating)
    assert got == want
    if bits == 0:
        assert got == payload


def test_packer_rejects_bad_tokens(mt_lib, oracle_lib):
    from maroontree_b200 import MtError

    n = mt_lib.load().mt_cdf_slot_count()
    for bad in ([(n << 8) | 0], [(0 << 8) | 2], [en.TOKEN_GATHERED_PARTITION | (0 << 2)]):
        with pytest.raises(MtError):
            en.pack_tile(70, [np.array(bad, np.uint32)])
