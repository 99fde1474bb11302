"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference benchmarks on downloaded read and protein sets that are not
available offline; these generators stand in for them with the stated
length and mutation distributions.  Everything is vectorised with numpy so
that a million pairs take seconds.

Each generator returns a ``Workload``: one code array holding every A then
every B (swatlib codes of the datatype, src/swatlib/encoding.h:26-72), the
per-pair offsets and lengths, and the scoring.

* ``dna_plain``      10,000 pairs: A = 150 uniform ACGT; B = A with 5 %
                     substitutions and 2 % single-base indels inside uniform
                     flanks, total length U[150, 300]; +1/-1, open/extend 1/1.
* ``dna_batched``    1,000,000 pairs: |A| ~ U[50, 250]; |B| lognormal
                     (median 300, sigma 0.5) clipped to [100, 1000]; B = A
                     with 3-15 % substitutions and 1-5 % indels of length 1-3
                     inside flanks; 10 % unrelated pairs; scoring as above.
* ``protein``        200,000 pairs: residues i.i.d. from the Robinson &
                     Robinson (1991, PNAS 88:5120) background frequencies;
                     |A| ~ Gamma(2, 175) clipped to [30, 2000]; B = A with
                     20-60 % BLOSUM62-weighted substitutions (y drawn with
                     probability ~ p_y 2^(S62(x,y)/2)) and geometric indels of
                     length 1-5; BLOSUM62, gap open 11 / extend 1.
* ``protein_mixed``  500,000 pairs: 90 % |A| ~ U[50, 400], 9 % U[400, 2000],
                     1 % U[2000, 8000]; 0.5 % near-identical long pairs
                     (|A| >= 7000, <= 1 % substitutions) whose scores exceed
                     int16; otherwise as ``protein``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

NA_ACGT = np.array([1, 4, 3, 2], dtype=np.uint8)  # codes of A C G T (A=1 T=2 C=3 G=4)
# Robinson & Robinson (1991) background frequencies, order A R N D C Q E G H I L K M F P S T W Y V
# (= amino-acid codes 0..19).
AA_BACKGROUND = np.array([0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295,
                          0.07377, 0.02199, 0.05142, 0.09019, 0.05744, 0.02243, 0.03856,
                          0.05203, 0.07120, 0.05841, 0.01330, 0.03216, 0.06441])
AA_BACKGROUND = AA_BACKGROUND / AA_BACKGROUND.sum()


@dataclasses.dataclass
class Workload:
    name: str
    datatype: str          # "na" | "aa"
    similarity: str        # "na" | "blosum62" | "blosum50"
    match: int
    mismatch: int
    ambiguity: int
    gap_init: int
    gap_extend: int
    codes: np.ndarray      # uint8
    a_off: np.ndarray      # int64
    a_len: np.ndarray      # int32
    b_off: np.ndarray      # int64
    b_len: np.ndarray      # int32
    seed: int

    @property
    def n(self) -> int:
        return int(self.a_len.size)

    @property
    def cells(self) -> int:
        return int(np.dot(self.a_len.astype(np.int64), self.b_len.astype(np.int64)))

    def subset(self, idx) -> "Workload":
        """Pairs `idx` with their own compact code array."""
        idx = np.asarray(idx)
        al = self.a_len[idx]
        bl = self.b_len[idx]
        parts_a = _gather(self.codes, self.a_off[idx], al)
        parts_b = _gather(self.codes, self.b_off[idx], bl)
        codes = np.concatenate([parts_a, parts_b])
        a_off = np.zeros(idx.size, dtype=np.int64)
        a_off[1:] = np.cumsum(al[:-1].astype(np.int64))
        b_off = parts_a.size + np.zeros(idx.size, dtype=np.int64)
        b_off[1:] += np.cumsum(bl[:-1].astype(np.int64))
        if codes.size == 0:
            codes = np.zeros(1, dtype=np.uint8)
        return dataclasses.replace(self, codes=codes, a_off=a_off, a_len=al.astype(np.int32),
                                   b_off=b_off, b_len=bl.astype(np.int32))

    def seqs(self, p):
        return (self.codes[self.a_off[p]:self.a_off[p] + self.a_len[p]],
                self.codes[self.b_off[p]:self.b_off[p] + self.b_len[p]])


def _gather(codes, off, ln):
    ln = ln.astype(np.int64)
    total = int(ln.sum())
    if total == 0:
        return np.zeros(0, dtype=np.uint8)
    starts = np.repeat(off.astype(np.int64) - np.concatenate([[0], np.cumsum(ln)[:-1]]), ln)
    return codes[starts + np.arange(total)]


def _letters(rng, alphabet_codes, probs, size):
    if probs is None:
        return alphabet_codes[rng.integers(0, alphabet_codes.size, size)]
    return alphabet_codes[rng.choice(alphabet_codes.size, size=size, p=probs)]


def _subst_cdf(sim62):
    """Per source residue x: cumulative distribution over targets y != x with
    weights p_y 2^(S62(x,y)/2)."""
    p = AA_BACKGROUND
    w = p[None, :] * np.power(2.0, sim62[:20, :20] / 2.0)
    np.fill_diagonal(w, 0.0)
    w = w / w.sum(axis=1, keepdims=True)
    return np.cumsum(w, axis=1)


def mutate(rng, src: np.ndarray, pair_of: np.ndarray, npairs: int, sub_rate: np.ndarray,
           indel_rate: np.ndarray, indel_len_max: int, alphabet: np.ndarray, probs,
           subst_cdf=None, geometric_p: float | None = None):
    """Mutates the concatenated sequences `src` (pair id per residue in
    `pair_of`) and returns (out, out_len_per_pair)."""
    n = src.size
    out = src.copy()
    # substitutions
    r = rng.random(n)
    sub = r < sub_rate[pair_of]
    ns = int(sub.sum())
    if ns:
        if subst_cdf is None:
            # uniform over the other letters
            cur = out[sub]
            rep = _letters(rng, alphabet, probs, ns)
            same = rep == cur
            while same.any():
                rep[same] = _letters(rng, alphabet, probs, int(same.sum()))
                same = rep == cur
            out[sub] = rep
        else:
            cur = out[sub].astype(np.int64)
            u = rng.random(ns)
            rep = np.empty(ns, dtype=np.uint8)
            for x in range(20):
                m = cur == x
                if m.any():
                    rep[m] = np.searchsorted(subst_cdf[x], u[m], side="right").clip(0, 19)
            out[sub] = rep
    # indel events: half deletions, half insertions
    r2 = rng.random(n)
    ev = r2 < indel_rate[pair_of]
    evpos = np.nonzero(ev)[0]
    if geometric_p is not None:
        lens = np.minimum(rng.geometric(geometric_p, evpos.size), indel_len_max)
    else:
        lens = rng.integers(1, indel_len_max + 1, evpos.size)
    is_del = rng.random(evpos.size) < 0.5
    keep = np.ones(n, dtype=np.int64)
    # deletions of `len` residues starting at the event, not crossing pairs
    dpos, dlen = evpos[is_del], lens[is_del]
    pair_end = np.cumsum(np.bincount(pair_of, minlength=npairs))
    dend = np.minimum(dpos + dlen, pair_end[pair_of[dpos]])  # deletions stay inside their pair
    diff = np.zeros(n + 1, dtype=np.int64)
    np.add.at(diff, dpos, 1)
    np.add.at(diff, dend, -1)
    deleted = np.cumsum(diff[:-1]) > 0
    keep[deleted] = 0
    ins_cnt = np.zeros(n, dtype=np.int64)
    ins_cnt[evpos[~is_del]] = lens[~is_del]
    counts = keep + ins_cnt
    total = int(counts.sum())
    src_idx = np.repeat(np.arange(n), counts)
    # position within the group: first `keep` copies are the residue itself
    starts = np.cumsum(counts) - counts
    within = np.arange(total) - np.repeat(starts, counts)
    res = out[src_idx].copy()
    inserted = within >= np.repeat(keep, counts)
    k = int(inserted.sum())
    if k:
        res[inserted] = _letters(rng, alphabet, probs, k)
    out_pair = pair_of[src_idx]
    out_len = np.bincount(out_pair, minlength=npairs)
    return res, out_len


def _assemble(rng, a_all, a_len, core, core_len, target_len, unrelated, alphabet, probs):
    """B = [left flank | core | right flank] of total max(target, core) (or
    a fresh random sequence for unrelated pairs); returns codes and offsets."""
    n = a_len.size
    core_len = core_len.astype(np.int64)
    target_len = np.maximum(target_len.astype(np.int64), 1)
    b_len = np.maximum(target_len, core_len)
    b_len = np.where(unrelated, target_len.astype(np.int64), b_len)
    b_total = int(b_len.sum())
    b_all = _letters(rng, alphabet, probs, b_total)
    b_start = np.concatenate([[0], np.cumsum(b_len)[:-1]])
    slack = np.maximum(b_len - core_len, 0)
    left = (rng.random(n) * (slack + 1)).astype(np.int64)
    left = np.minimum(left, slack)
    copy_len = np.where(unrelated, 0, core_len)
    core_start = np.concatenate([[0], np.cumsum(core_len)[:-1]])
    tot = int(copy_len.sum())
    if tot:
        dst = np.repeat(b_start + left, copy_len) + (np.arange(tot) - np.repeat(
            np.concatenate([[0], np.cumsum(copy_len)[:-1]]), copy_len))
        srcp = np.repeat(core_start, copy_len) + (np.arange(tot) - np.repeat(
            np.concatenate([[0], np.cumsum(copy_len)[:-1]]), copy_len))
        b_all[dst] = core[srcp]
    codes = np.concatenate([a_all, b_all])
    a_off = np.concatenate([[0], np.cumsum(a_len.astype(np.int64))[:-1]])
    b_off = a_all.size + b_start
    return codes, a_off.astype(np.int64), b_off.astype(np.int64), b_len.astype(np.int32)


def _related(rng, a_len, alphabet, probs, sub_lo, sub_hi, indel_lo, indel_hi, indel_len_max,
             target_len, unrelated_frac, subst_cdf=None, geometric_p=None):
    n = a_len.size
    a_all = _letters(rng, alphabet, probs, int(a_len.sum()))
    pair_of = np.repeat(np.arange(n), a_len)
    sub_rate = rng.uniform(sub_lo, sub_hi, n)
    indel_rate = rng.uniform(indel_lo, indel_hi, n)
    core, core_len = mutate(rng, a_all, pair_of, n, sub_rate, indel_rate, indel_len_max, alphabet,
                            probs, subst_cdf=subst_cdf, geometric_p=geometric_p)
    unrelated = rng.random(n) < unrelated_frac
    return a_all, _assemble(rng, a_all, a_len, core, core_len, target_len, unrelated, alphabet, probs)


def dna_plain(n=10_000, seed=1000) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    a_len = np.full(n, 150, dtype=np.int32)
    target = rng.integers(150, 301, n)
    _, (codes, a_off, b_off, b_len) = _related(rng, a_len, NA_ACGT, None, 0.05, 0.05, 0.02, 0.02,
                                               1, target, 0.0)
    return Workload("dna_plain_10k", "na", "na", 1, -1, -1, 0, -1, codes, a_off, a_len, b_off,
                    b_len, seed)


def dna_batched(n=1_000_000, seed=1001) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    a_len = rng.integers(50, 251, n).astype(np.int32)
    target = np.clip(np.round(np.exp(rng.normal(np.log(300.0), 0.5, n))), 100, 1000).astype(np.int64)
    _, (codes, a_off, b_off, b_len) = _related(rng, a_len, NA_ACGT, None, 0.03, 0.15, 0.01, 0.05,
                                               3, target, 0.10)
    return Workload("dna_batched_1m", "na", "na", 1, -1, -1, 0, -1, codes, a_off, a_len, b_off,
                    b_len, seed)


def _blosum62():
    from ipuma_b200 import select_matrix  # product tables (checked against the reference)
    return select_matrix("blosum62").astype(np.float64)


def protein(n=200_000, seed=1002, sim62=None) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    sim62 = _blosum62() if sim62 is None else sim62
    a_len = np.clip(np.round(rng.gamma(2.0, 175.0, n)), 30, 2000).astype(np.int32)
    cdf = _subst_cdf(sim62)
    aa = np.arange(20, dtype=np.uint8)
    target = a_len.astype(np.int64)  # B is the mutated query (no flanks)
    _, (codes, a_off, b_off, b_len) = _related(rng, a_len, aa, AA_BACKGROUND, 0.20, 0.60, 0.01,
                                               0.05, 5, target, 0.0, subst_cdf=cdf,
                                               geometric_p=0.5)
    return Workload("protein_200k", "aa", "blosum62", 1, -1, -1, -10, -1, codes, a_off, a_len,
                    b_off, b_len, seed)


def protein_mixed(n=500_000, seed=1003, sim62=None, long_identical_frac=0.005) -> Workload:
    rng = np.random.Generator(np.random.PCG64(seed))
    sim62 = _blosum62() if sim62 is None else sim62
    u = rng.random(n)
    a_len = np.where(u < 0.90, rng.integers(50, 401, n),
                     np.where(u < 0.99, rng.integers(400, 2001, n), rng.integers(2000, 8001, n)))
    n_ident = int(round(n * long_identical_frac))
    ident = np.zeros(n, dtype=bool)
    ident[rng.choice(n, n_ident, replace=False)] = True
    a_len = np.where(ident, rng.integers(7000, 8001, n), a_len).astype(np.int32)
    cdf = _subst_cdf(sim62)
    aa = np.arange(20, dtype=np.uint8)
    a_all = _letters(rng, aa, AA_BACKGROUND, int(a_len.sum()))
    pair_of = np.repeat(np.arange(n), a_len)
    sub_rate = np.where(ident, rng.uniform(0.0, 0.01, n), rng.uniform(0.20, 0.60, n))
    indel_rate = np.where(ident, 0.0, rng.uniform(0.01, 0.05, n))
    core, core_len = mutate(rng, a_all, pair_of, n, sub_rate, indel_rate, 5, aa, AA_BACKGROUND,
                            subst_cdf=cdf, geometric_p=0.5)
    codes, a_off, b_off, b_len = _assemble(rng, a_all, a_len, core, core_len,
                                           core_len.astype(np.int64), np.zeros(n, dtype=bool),
                                           aa, AA_BACKGROUND)
    return Workload("protein_mixed_500k", "aa", "blosum62", 1, -1, -1, -10, -1, codes, a_off,
                    a_len, b_off, b_len, seed)


CONFIGS = {
    "dna_plain": dna_plain,
    "dna_batched": dna_batched,
    "protein": protein,
    "protein_mixed": protein_mixed,
}
