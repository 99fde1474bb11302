"""CPU tests of the C ABI library: it loads without a GPU, exports every
function include/ipuma_b200.h declares, and its host helpers (encoders,
matrices, buffer sizes) match the reference tables in tests/golden/."""
import json
import os
import re

import numpy as np
import pytest

import ipuma_b200 as ib
import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(REPO, "include", "ipuma_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ipuma_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = ib.lib()
    declared = _declared()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(ib.EXPORTS) == declared


def test_version_and_error_strings():
    assert b"sm_100a" in ib.lib().ipuma_version()
    with pytest.raises(ib.IpumaError) as ei:
        ib.select_matrix("simple")
    assert ei.value.code == ib.ERR_INVALID_ARG
    assert "simple" in ib.last_error()


@pytest.mark.parametrize("sim,args", [("na", (1, -1, -1)), ("na", (2, -3, -5)),
                                      ("blosum50", (1, -1, -1)), ("blosum62", (1, -1, -1))])
def test_matrices_match_reference_tables(sim, args):
    np.testing.assert_array_equal(ib.select_matrix(sim, *args), oracle.select_matrix(sim, *args))


def test_encoders_match_reference_tables():
    t = json.load(open(os.path.join(REPO, "tests", "golden", "tables.json")))
    for dt, key in (("na", "NA_CODE"), ("aa", "AA_CODE")):
        for ch, code in t[key].items():
            if ch == "\\0":
                continue
            assert ib.encode(dt, ch)[0] == code
            assert ib.encode(dt, ch.lower())[0] == code
    assert ib.encode("aa", "?")[0] == t["AA_CODE"]["\\0"]
    with pytest.raises(ib.IpumaError) as ei:
        ib.encode("na", "ACGX")
    assert ei.value.code == ib.ERR_BAD_SEQUENCE


def test_input_buffer_words():
    a = ib.algo_config(tiles_used=7, max_batches=9, bufsize=4001)
    assert ib.input_buffer_words(a) == 7 * 1001 + 7 * 9 * 4


def test_create_without_device_fails_cleanly():
    if ib.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(ib.IpumaError) as ei:
        ib.Engine(ib.sw_config())
    assert ei.value.code == ib.ERR_NO_DEVICE


@pytest.mark.parametrize("n", [0, 1, 2, 7, 64, 100_001, (1 << 23) + 5])
def test_pack_codes4_layout(n):
    """Residue 2k in the low nibble of byte k, 2k+1 in the high nibble; an
    odd count leaves the last high nibble 0 (large inputs pack on several
    threads)."""
    codes = np.random.default_rng(n).integers(0, 16, n).astype(np.uint8)
    packed = ib.pack_codes4(codes)
    assert packed.size == (n + 1) // 2
    want = np.zeros((n + 1) // 2 * 2, np.uint8)
    want[:n] = codes
    np.testing.assert_array_equal(packed, want[0::2] | (want[1::2] << 4))


def test_pack_codes4_rejects_codes_above_15():
    codes = np.zeros(5_000_000, np.uint8)
    codes[3_000_001] = 16
    codes[4_000_000] = 200
    with pytest.raises(ib.IpumaError) as ei:
        ib.pack_codes4(codes)
    assert ei.value.code == ib.ERR_BAD_SEQUENCE
    assert "3000001" in str(ei.value)


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 64, 100_003, (1 << 24) + 7])
def test_pack_codes2_layout(n):
    """A, T, C, G (codes 1..4) four per byte as code - 1, residue 4k+q in
    bits 2q..2q+1 of byte k; missing residues of the last byte are 0."""
    codes = np.random.default_rng(n).integers(1, 5, n).astype(np.uint8)
    packed = ib.pack_codes(codes, 2)
    assert packed.size == (n + 3) // 4
    v = np.zeros((n + 3) // 4 * 4, np.uint8)
    v[:n] = codes - 1
    want = v[0::4] | (v[1::4] << 2) | (v[2::4] << 4) | (v[3::4] << 6)
    np.testing.assert_array_equal(packed, want)


@pytest.mark.parametrize("bad", [0, 5, 15, 16])
def test_pack_codes2_takes_only_acgt(bad):
    """N (code 0) and the IUPAC codes 5..15 need the 4-bit path."""
    codes = np.full(1_000, 2, np.uint8)
    codes[777] = bad
    with pytest.raises(ib.IpumaError) as ei:
        ib.pack_codes(codes, 2)
    assert ei.value.code == ib.ERR_BAD_SEQUENCE and "777" in str(ei.value)
    with pytest.raises(ib.IpumaError):
        ib.pack_codes(codes, 3)


def _bitstream(values, bits):
    """Little-endian bit stream of `bits`-bit fields (the restatement the
    packer is checked against): field r in bits [bits*r, bits*r + bits)."""
    n = values.size
    nbytes = (n * bits + 7) // 8
    bitpos = np.arange(n, dtype=np.int64)[:, None] * bits + np.arange(bits)[None, :]
    bitval = (values.astype(np.int64)[:, None] >> np.arange(bits)[None, :]) & 1
    flat = np.zeros(nbytes * 8, np.uint8)
    flat[bitpos.ravel()] = bitval.ravel()
    return np.packbits(flat.reshape(-1, 8)[:, ::-1], axis=1).ravel()


@pytest.mark.parametrize("n", [0, 1, 7, 8, 9, 63, 64, 100_003, (1 << 23) + 5])
def test_pack_codes5_layout(n):
    """Amino-acid codes 0..24 as a little-endian bit stream of 5-bit fields;
    the last byte's missing bits are 0 (large inputs pack on several
    threads)."""
    codes = np.random.default_rng(n).integers(0, 25, n).astype(np.uint8)
    packed = ib.pack_codes(codes, 5)
    assert packed.size == (5 * n + 7) // 8
    np.testing.assert_array_equal(packed, _bitstream(codes, 5))


@pytest.mark.parametrize("bits", [2, 4])
def test_pack_codes_2_and_4_are_the_same_bit_stream(bits):
    codes = np.random.default_rng(bits).integers(1, 5, 1001).astype(np.uint8)
    packed = ib.pack_codes(codes, bits)
    np.testing.assert_array_equal(packed, _bitstream(codes - 1 if bits == 2 else codes, bits))


def test_pack_codes5_rejects_codes_above_31():
    codes = np.full(500, 3, np.uint8)
    codes[321] = 32
    with pytest.raises(ib.IpumaError) as ei:
        ib.pack_codes(codes, 5)
    assert ei.value.code == ib.ERR_BAD_SEQUENCE and "321" in str(ei.value)
