"""Seeded synthetic PairHMM workloads with the shapes of the benchmark configs.

The reference benchmarks this stage on no public dataset, so reads and
haplotypes are simulated (numpy.random.default_rng(seed), seeds 0-4):

* ``single_region``  one region: hap0 300 bp uniform ACGT, hap1 = hap0 with an SNV at
  150 and a 3 bp deletion at 220; 64 reads of 150 bp, start uniform, source
  haplotype 50/50, 1% substitution and 0.1% 1-bp indel error, qualities i.i.d.
  from Q{10,20,30,40} with probabilities {.05,.15,.5,.3}; gap-open Q45,
  gap-continuation Q10.
* ``batched_regions``  10,000 regions; haplotypes per region U{2..16}, first haplotype
  U{100..1000} bp, every other one the first with 1-4 SNVs and one 1-10 bp
  indel; reads per region round(lognormal(ln 60, 1.0)) clipped to 10..500,
  read length U{100..250} (at most the source haplotype's length); errors and
  qualities as single_region.
* ``long_haplotype_stress``  2,000 regions x 4 haplotypes of U{1000..5000} bp; 50 reads of
  U{150..300} bp per region; 20% of the reads carry 5% substitution error with
  qualities U{2..15}.
* ``planted_error_model``  1,000 regions shaped as batched_regions, with reads drawn from the
  PairHMM's own generative model under planted parameters: gap-open Q40,
  gap-continuation Q8, and true base errors 10^(-(q + o_bin)/10) for the
  reported quality q with bin offsets (+2, -1, 0, +3) (bins q<15, q<25,
  q<35, q>=35, i.e. the Q10/20/30/40 levels).  A read starts in M at a
  uniform column of its source haplotype; every M state moves to M, I or D
  with 1-2g, g, g; I and D extend with x; M emits the haplotype base (a
  uniform other base with probability e), I a uniform base, D nothing.
* ``mixed_length_regions``  200,000 regions; haplotype length lognormal (median 400, sigma
  0.6) clipped to 80..8000, U{2..32} haplotypes; reads lognormal (median 40,
  sigma 1.0) clipped to 4..2000 of 150 bp; 2% of regions instead carry
  U{2..8} reads of 1-10 kb at 8% error (6% substitution, 2% 1-bp indel) against
  haplotypes long enough to contain them.

Every workload is a region batch in the packed layout of vd_batch.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

ALPHABET = np.frombuffer(b"ACGT", np.uint8)
Q_LEVELS = np.array([10, 20, 30, 40], np.uint8)
Q_PROBS = np.array([0.05, 0.15, 0.5, 0.3])
GAP_Q45 = 10.0 ** -4.5
EXT_Q10 = 0.1


@dataclass
class Workload:
    name: str
    read_bases: np.ndarray
    read_quals: np.ndarray
    read_off: np.ndarray
    hap_bases: np.ndarray
    hap_off: np.ndarray
    region_read_off: np.ndarray
    region_hap_off: np.ndarray
    gap: float = GAP_Q45
    ext: float = EXT_Q10
    anchored: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def n_regions(self) -> int:
        return len(self.region_read_off) - 1

    def read_lengths(self) -> np.ndarray:
        return np.diff(self.read_off)

    def hap_lengths(self) -> np.ndarray:
        return np.diff(self.hap_off)

    def pairs(self) -> int:
        return int(np.sum(np.diff(self.region_read_off) * np.diff(self.region_hap_off)))

    def cells(self) -> int:
        rl = self.read_lengths()
        hl = self.hap_lengths()
        rsum = np.add.reduceat(rl, self.region_read_off[:-1]) if len(rl) else np.zeros(0)
        hsum = np.add.reduceat(hl, self.region_hap_off[:-1]) if len(hl) else np.zeros(0)
        empty_r = self.region_read_off[1:] == self.region_read_off[:-1]
        empty_h = self.region_hap_off[1:] == self.region_hap_off[:-1]
        rsum = np.where(empty_r, 0, rsum)
        hsum = np.where(empty_h, 0, hsum)
        return int(np.sum(rsum.astype(np.int64) * hsum.astype(np.int64)))

    def input_bytes(self) -> int:
        return int(self.read_bases.nbytes + self.read_quals.nbytes + self.read_off.nbytes + self.hap_bases.nbytes
                   + self.hap_off.nbytes + self.region_read_off.nbytes + self.region_hap_off.nbytes)

    def subset(self, regions) -> "Workload":
        """The workload restricted to the given region indices (in that order)."""
        regions = np.asarray(regions, np.int64)
        rb, rq, hb = [], [], []
        roff, hoff, rro, rho = [0], [0], [0], [0]
        for g in regions:
            r0, r1 = self.region_read_off[g], self.region_read_off[g + 1]
            h0, h1 = self.region_hap_off[g], self.region_hap_off[g + 1]
            a, b = self.read_off[r0], self.read_off[r1]
            rb.append(self.read_bases[a:b])
            rq.append(self.read_quals[a:b])
            roff.extend((self.read_off[r0 + 1:r1 + 1] - a + roff[-1]).tolist())
            c, d = self.hap_off[h0], self.hap_off[h1]
            hb.append(self.hap_bases[c:d])
            hoff.extend((self.hap_off[h0 + 1:h1 + 1] - c + hoff[-1]).tolist())
            rro.append(rro[-1] + (r1 - r0))
            rho.append(rho[-1] + (h1 - h0))
        cat = lambda xs: np.concatenate(xs) if xs else np.empty(0, np.uint8)
        return Workload(self.name + "-subset", cat(rb), cat(rq), np.asarray(roff, np.int64), cat(hb),
                        np.asarray(hoff, np.int64), np.asarray(rro, np.int64), np.asarray(rho, np.int64),
                        self.gap, self.ext, self.anchored, dict(self.meta, subset=len(regions)))

    def explicit_pairs(self):
        """(pair_read, pair_hap) of the region batch in output order."""
        rr, hh = self.region_read_off, self.region_hap_off
        nr = np.diff(rr)
        nh = np.diff(hh)
        tot = int(np.sum(nr * nh))
        pr = np.empty(tot, np.int32)
        ph = np.empty(tot, np.int32)
        o = 0
        for g in range(len(nr)):
            k = int(nr[g] * nh[g])
            if k:
                pr[o:o + k] = np.repeat(np.arange(rr[g], rr[g + 1]), nh[g])
                ph[o:o + k] = np.tile(np.arange(hh[g], hh[g + 1]), nr[g])
            o += k
        return pr, ph


def _random_hap(rng, length: int) -> np.ndarray:
    return ALPHABET[rng.integers(0, 4, length)]


def _mutate(rng, hap: np.ndarray, n_snv: int, indel_len: int) -> np.ndarray:
    """hap with n_snv substitutions and one insertion or deletion of indel_len bases."""
    h = hap.copy()
    if len(h) > 2 and n_snv:
        pos = rng.choice(len(h), size=min(n_snv, len(h)), replace=False)
        for p in pos:
            choices = ALPHABET[ALPHABET != h[p]]
            h[p] = choices[rng.integers(0, 3)]
    if indel_len > 0 and len(h) > indel_len + 2:
        p = int(rng.integers(1, len(h) - indel_len))
        if rng.random() < 0.5:
            h = np.concatenate([h[:p], h[p + indel_len:]])
        else:
            h = np.concatenate([h[:p], _random_hap(rng, indel_len), h[p:]])
    return h


def _sim_reads(rng, haps, n_reads, lengths, p_sub, p_indel, quals_fn):
    """Simulate reads from random source haplotypes (vectorised over a region).

    Returns (list of base arrays, list of quality arrays).
    """
    if n_reads == 0:
        return [], []
    hl = np.array([len(h) for h in haps], np.int64)
    hoff = np.concatenate([[0], np.cumsum(hl)])
    flat = np.concatenate(haps)
    src = rng.integers(0, len(haps), n_reads)
    L = np.minimum(np.asarray(lengths, np.int64), hl[src])
    start = (rng.random(n_reads) * (hl[src] - L + 1)).astype(np.int64)
    roff = np.concatenate([[0], np.cumsum(L)])
    total = int(roff[-1])
    idx = np.arange(total, dtype=np.int64) - np.repeat(roff[:-1], L) + np.repeat(hoff[src] + start, L)
    bases = flat[idx]
    if p_sub > 0:
        mask = rng.random(total) < p_sub
        k = int(mask.sum())
        if k:
            codes = np.searchsorted(ALPHABET, bases[mask])
            bases[mask] = ALPHABET[(codes + rng.integers(1, 4, k)) % 4]
    reads = [bases[roff[i]:roff[i + 1]] for i in range(n_reads)]
    if p_indel > 0:
        ev_mask = rng.random(total) < p_indel
        for i in np.unique(np.searchsorted(roff, np.flatnonzero(ev_mask), side="right") - 1):
            r = reads[i]
            n = len(r)
            ev = np.flatnonzero(ev_mask[roff[i]:roff[i + 1]])
            parts = []
            last = 0
            for p in ev:
                parts.append(r[last:p])
                if rng.random() < 0.5:           # deletion of base p
                    last = p + 1
                else:                             # insertion before base p
                    parts.append(_random_hap(rng, 1))
                    last = p
            parts.append(r[last:])
            r = np.concatenate(parts)
            # keep the simulated length
            if len(r) > n:
                r = r[:n]
            elif len(r) < n:
                r = np.concatenate([r, _random_hap(rng, n - len(r))])
            reads[i] = r
    q = quals_fn(total)
    quals = [q[roff[i]:roff[i + 1]] for i in range(n_reads)]
    return reads, quals


def _q_standard(rng):
    return lambda n: Q_LEVELS[rng.choice(4, size=n, p=Q_PROBS)]


def _assemble(name, regions, gap, ext, meta) -> Workload:
    rb, rq, hb = [], [], []
    roff, hoff, rro, rho = [0], [0], [0], [0]
    for haps, reads, quals in regions:
        for r, q in zip(reads, quals):
            rb.append(r)
            rq.append(q)
            roff.append(roff[-1] + len(r))
        for h in haps:
            hb.append(h)
            hoff.append(hoff[-1] + len(h))
        rro.append(rro[-1] + len(reads))
        rho.append(rho[-1] + len(haps))
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.empty(0, dt)
    return Workload(name, cat(rb, np.uint8), cat(rq, np.uint8), np.asarray(roff, np.int64), cat(hb, np.uint8),
                    np.asarray(hoff, np.int64), np.asarray(rro, np.int64), np.asarray(rho, np.int64), gap, ext,
                    False, meta)


def single_region(seed: int = 0, gap: float = GAP_Q45, ext: float = EXT_Q10) -> Workload:
    rng = np.random.default_rng(seed)
    hap0 = _random_hap(rng, 300)
    hap1 = hap0.copy()
    hap1[150] = ALPHABET[ALPHABET != hap0[150]][rng.integers(0, 3)]
    hap1 = np.concatenate([hap1[:220], hap1[223:]])
    reads, quals = _sim_reads(rng, [hap0, hap1], 64, np.full(64, 150), 0.01, 0.001, _q_standard(rng))
    return _assemble("single_region", [([hap0, hap1], reads, quals)], gap, ext, {"seed": seed})


def batched_regions(seed: int = 1, n_regions: int = 10_000, gap: float = GAP_Q45, ext: float = EXT_Q10,
            sigma: float = 1.0) -> Workload:
    rng = np.random.default_rng(seed)
    qf = _q_standard(rng)
    regions = []
    for _ in range(n_regions):
        H = int(rng.integers(2, 17))
        hap0 = _random_hap(rng, int(rng.integers(100, 1001)))
        haps = [hap0] + [_mutate(rng, hap0, int(rng.integers(1, 5)), int(rng.integers(1, 11))) for _ in range(H - 1)]
        nr = int(np.clip(round(rng.lognormal(np.log(60), sigma)), 10, 500))
        reads, quals = _sim_reads(rng, haps, nr, rng.integers(100, 251, nr), 0.01, 0.001, qf)
        regions.append((haps, reads, quals))
    return _assemble("batched_regions", regions, gap, ext, {"seed": seed, "sigma": sigma, "regions": n_regions})


def long_haplotype_stress(seed: int = 2, n_regions: int = 2_000, gap: float = GAP_Q45, ext: float = EXT_Q10) -> Workload:
    rng = np.random.default_rng(seed)
    qf = _q_standard(rng)
    low_q = lambda n: rng.integers(2, 16, n).astype(np.uint8)
    regions = []
    for _ in range(n_regions):
        hap0 = _random_hap(rng, int(rng.integers(1000, 5001)))
        haps = [hap0] + [_mutate(rng, hap0, int(rng.integers(1, 5)), int(rng.integers(1, 11))) for _ in range(3)]
        lengths = rng.integers(150, 301, 50)
        bad = rng.random(50) < 0.2
        good_r, good_q = _sim_reads(rng, haps, int((~bad).sum()), lengths[~bad], 0.01, 0.001, qf)
        bad_r, bad_q = _sim_reads(rng, haps, int(bad.sum()), lengths[bad], 0.05, 0.0, low_q)
        regions.append((haps, good_r + bad_r, good_q + bad_q))
    return _assemble("long_haplotype_stress", regions, gap, ext, {"seed": seed, "regions": n_regions})


PLANTED_Q_GAP = 40.0
PLANTED_Q_EXT = 8.0
PLANTED_OFFSETS = (2.0, -1.0, 0.0, 3.0)


def _quality_bin(q: np.ndarray) -> np.ndarray:
    return np.searchsorted(np.array([15, 25, 35]), q, side="right")


def _sim_hmm_reads(rng, haps, n_reads, lengths, gap, ext, offsets, quals_fn):
    """Reads drawn from the PairHMM generative model (semiglobal, start uniform)."""
    if n_reads == 0:
        return [], []
    src = rng.integers(0, len(haps), n_reads)
    reads, quals = [], []
    for k in range(n_reads):
        hap = haps[src[k]]
        m = len(hap)
        n = int(min(lengths[k], m))
        q = quals_fn(n)
        ph = np.maximum(0.0, np.minimum(q, 60) + np.asarray(offsets)[_quality_bin(q)])
        e = 10.0 ** (-ph / 10.0)
        start = int(rng.integers(0, m - n + 1))
        # one M -> {M, I, D} draw per emitted read base; gaps are rare, so the
        # common all-match read is a straight copy
        u = rng.random(n)
        events = np.flatnonzero(u < 2 * gap)
        if events.size == 0:
            out = hap[start:start + n].copy()
            from_hap = np.ones(n, bool)
        else:
            parts, flags = [], []
            i = j = 0  # read bases emitted, haplotype column
            j = start
            ev = set(events.tolist())
            while i < n:
                if i in ev:
                    run = 1 + int(rng.geometric(1.0 - ext)) - 1
                    if u[i] < gap:       # insertion run: uniform bases
                        take = min(run, n - i)
                        parts.append(_random_hap(rng, take))
                        flags.append(np.zeros(take, bool))
                        i += take
                        if i >= n:
                            break
                    else:                # deletion run: skip haplotype bases
                        j += run
                    ev.discard(i)
                # M emission (past the haplotype end only insertions remain)
                if j < m:
                    parts.append(hap[j:j + 1])
                    flags.append(np.ones(1, bool))
                    j += 1
                else:
                    parts.append(_random_hap(rng, 1))
                    flags.append(np.zeros(1, bool))
                i += 1
            out = np.concatenate(parts)[:n].copy()
            from_hap = np.concatenate(flags)[:n]
        sub = from_hap & (rng.random(n) < e)
        if sub.any():
            codes = np.searchsorted(ALPHABET, out[sub])
            out[sub] = ALPHABET[(codes + rng.integers(1, 4, int(sub.sum()))) % 4]
        reads.append(out)
        quals.append(q)
    return reads, quals


def planted_error_model(seed: int = 3, n_regions: int = 1_000, q_gap: float = PLANTED_Q_GAP, q_ext: float = PLANTED_Q_EXT,
            offsets=PLANTED_OFFSETS, sigma: float = 1.0) -> Workload:
    """batched_regions-shaped regions whose reads follow the model under planted parameters."""
    rng = np.random.default_rng(seed)
    qf = _q_standard(rng)
    gap, ext = 10.0 ** (-q_gap / 10.0), 10.0 ** (-q_ext / 10.0)
    regions = []
    for _ in range(n_regions):
        H = int(rng.integers(2, 17))
        hap0 = _random_hap(rng, int(rng.integers(100, 1001)))
        haps = [hap0] + [_mutate(rng, hap0, int(rng.integers(1, 5)), int(rng.integers(1, 11))) for _ in range(H - 1)]
        nr = int(np.clip(round(rng.lognormal(np.log(60), sigma)), 10, 500))
        reads, quals = _sim_hmm_reads(rng, haps, nr, rng.integers(100, 251, nr), gap, ext, offsets, qf)
        regions.append((haps, reads, quals))
    return _assemble("planted_error_model", regions, GAP_Q45, EXT_Q10,
                     {"seed": seed, "regions": n_regions, "planted": [q_gap, q_ext, *offsets]})


def _concat(parts, name, gap, ext, meta) -> Workload:
    """Join region batches generated separately into one batch."""
    def join(key, off_key=None):
        arrs = [getattr(p, key) for p in parts]
        return np.concatenate(arrs) if arrs else np.empty(0)

    def join_off(key):
        out, base = [np.zeros(1, np.int64)], 0
        for p in parts:
            o = getattr(p, key)
            out.append(o[1:] + base)
            base += int(o[-1])
        return np.concatenate(out)

    return Workload(name, join("read_bases").astype(np.uint8), join("read_quals").astype(np.uint8),
                    join_off("read_off"), join("hap_bases").astype(np.uint8), join_off("hap_off"),
                    join_off("region_read_off"), join_off("region_hap_off"), gap, ext, False, meta)


_MIXED_BLOCK = 2_000


def _mixed_block(args) -> Workload:
    seed, block, count, gap, ext = args
    rng = np.random.default_rng([seed, block])
    return _mixed_regions(rng, count, gap, ext)


def mixed_length_regions(seed: int = 4, n_regions: int = 200_000, gap: float = GAP_Q45, ext: float = EXT_Q10,
            workers: int = 1) -> Workload:
    """Regions are drawn in blocks of 2,000, block b from default_rng([seed, b]), so the
    blocks can be generated on several host processes (workers > 1; 0 = every core).  The
    processes are spawned, so a script that asks for workers != 1 must call this under
    ``if __name__ == "__main__":``."""
    import os
    blocks = [(seed, b, min(_MIXED_BLOCK, n_regions - b * _MIXED_BLOCK), gap, ext)
              for b in range((n_regions + _MIXED_BLOCK - 1) // _MIXED_BLOCK)]
    if workers == 0:
        workers = min(len(blocks), len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else 1)
    if workers > 1 and len(blocks) > 1:
        import multiprocessing as mp
        # spawn: a forked child of a process that holds a CUDA context can hang
        with mp.get_context("spawn").Pool(workers) as pool:
            parts = pool.map(_mixed_block, blocks)
    else:
        parts = [_mixed_block(b) for b in blocks]
    return _concat(parts, "mixed_length_regions", gap, ext, {"seed": seed, "regions": n_regions})


def _mixed_regions(rng, n_regions: int, gap: float, ext: float) -> Workload:
    qf = _q_standard(rng)
    regions = []
    for _ in range(n_regions):
        H = int(rng.integers(2, 33))
        if rng.random() < 0.02:
            nr = int(rng.integers(2, 9))
            lengths = rng.integers(1000, 10001, nr)
            m0 = int(lengths.max() + rng.integers(100, 1000))
            hap0 = _random_hap(rng, m0)
            haps = [hap0] + [_mutate(rng, hap0, int(rng.integers(1, 5)), int(rng.integers(1, 11)))
                             for _ in range(H - 1)]
            reads, quals = _sim_reads(rng, haps, nr, lengths, 0.06, 0.02, qf)
        else:
            m0 = int(np.clip(round(rng.lognormal(np.log(400), 0.6)), 80, 8000))
            hap0 = _random_hap(rng, m0)
            haps = [hap0] + [_mutate(rng, hap0, int(rng.integers(1, 5)), int(rng.integers(1, 11)))
                             for _ in range(H - 1)]
            nr = int(np.clip(round(rng.lognormal(np.log(40), 1.0)), 4, 2000))
            reads, quals = _sim_reads(rng, haps, nr, np.full(nr, 150), 0.01, 0.001, qf)
        regions.append((haps, reads, quals))
    return _assemble("mixed_length_regions", regions, gap, ext, {})


def random_pairs(seed: int, shapes, copies: int, qlo: int = 0, qhi: int = 61, alphabet="ACGT"):
    """Random (read, quals, hap) triples of the given (n, m) shapes, as the reference's tests draw them
    (caller/native/caller/tests/test_accelerator.py:43-47)."""
    rng = np.random.default_rng(seed)
    pairs = []
    for n, m in shapes:
        for _ in range(copies):
            s = "".join(rng.choice(list(alphabet), n))
            h = "".join(rng.choice(list(alphabet), m))
            q = rng.integers(qlo, qhi, n)
            pairs.append((s, q, h))
    return pairs
