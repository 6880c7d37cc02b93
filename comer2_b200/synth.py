"""Seeded synthetic COMER profiles and databases.

No public profile database is used: every workload is generated here from a
seed, with the shapes and value distributions of the benchmark configurations:

* 20 target probabilities per position ~ Dirichlet(0.5 * background), where the
  background is the Robinson & Robinson (1991) amino-acid composition, the
  composition COMER profiles carry by default;
* ENO ~ U[1, 14], printed with one decimal as in the text format;
* 7 transition probabilities (MM, MI, MD, IM, II, DM, DD) ~
  Dirichlet(10, 1, 1, 1, 1, 1, 1), renormalised per source state (M, I, D);
* 3 SS probabilities (C, E, H) ~ Dirichlet(1, 1, 1), state = argmax;
* a 19-entry context vector ~ N(0, 1), its log prior = the N(0, I) log
  density, and its squared norm.

Values are quantised exactly as the COMER text profile format stores them
(integers scaled by 10000; SS probabilities truncated), so the same numbers can
be written as text profiles and read by any COMER reader.  The format stores no
zero target probability for a realistic profile (profiles carry pseudocounts),
so each quantised probability is floored at 1/10000 and the largest entry
absorbs the rounding remainder; the same floor applies to transition
probabilities.

Conversions to the search's working values follow the reference's text reader
(``src/libmycu/cupro/IOProfileModelTxt.cu:336-371,480-515``): probability =
int / 10000 in float32; transition value = logf(p), times 0.4 for IM, II, DM
and DD (``MAIN_TRNPRB_LOGFCT``, ``src/libpro/srcpro/TRANSPROBS.h:10``).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

SCALE = 10000
AA = b"ARNDCQEGHILKMFPSTWYV"
SSCH = b"CEH"
NUMAA = 20
NCV = 19
NTRN = 7          # MM MI MD IM II DM DD
LOG0 = -32768.0   # the reader's value for log(0)
TRN_LOGFCT = np.float32(0.4)

# Robinson, A.B. & Robinson, L.R. (1991) PNAS 88:8880 amino-acid frequencies,
# in the order ARNDCQEGHILKMFPSTWYV
ROBINSON = np.array([
    0.07805, 0.05129, 0.04487, 0.05364, 0.01925, 0.04264, 0.06295, 0.07377, 0.02199, 0.05142,
    0.09019, 0.05744, 0.02243, 0.03856, 0.05203, 0.07120, 0.05841, 0.01330, 0.03216, 0.06441,
], np.float64)


@dataclass
class ProfileSet:
    """Profiles in structure-of-arrays form, concatenated over positions.

    ``trn`` has one extra row per profile: row ``offsets[k] + k + i`` holds the
    transitions into position i of profile k (i = 0 is the beginning state),
    and row ``offsets[k] + k + lengths[k]`` the transitions out of its last
    position -- the reference's ``ptr2DTrnPrbs`` layout.
    """
    lengths: np.ndarray    # int32 [P]
    offsets: np.ndarray    # int64 [P]
    bkg: np.ndarray        # float32 [P, 20]
    eno: np.ndarray        # float32 [P]
    trn: np.ndarray        # float32 [N + P, 7] log-space working values
    trg: np.ndarray        # float32 [N, 20]
    cv: np.ndarray         # float32 [N, 19]
    cvprior: np.ndarray    # float32 [N]
    cvnorm2: np.ndarray    # float32 [N]
    ss: np.ndarray         # float32 [N, 3]
    ssstate: np.ndarray    # uint8 [N]
    aa: np.ndarray         # uint8 [N]
    # integer (text-format) values kept for writing profiles
    trn_int: np.ndarray    # int32 [N + P, 7]
    trg_int: np.ndarray    # int32 [N, 20]

    @property
    def nprofiles(self) -> int:
        return int(self.lengths.shape[0])

    @property
    def npositions(self) -> int:
        return int(self.trg.shape[0])

    def profile(self, k: int) -> "ProfileSet":
        """A one-profile view (copies) of profile k."""
        return self.subset([k])

    def subset(self, idx: Sequence[int]) -> "ProfileSet":
        idx = list(idx)
        pos = [np.arange(self.offsets[k], self.offsets[k] + self.lengths[k]) for k in idx]
        trows = [np.arange(self.offsets[k] + k, self.offsets[k] + k + self.lengths[k] + 1) for k in idx]
        pos = np.concatenate(pos) if pos else np.zeros(0, np.int64)
        trows = np.concatenate(trows) if trows else np.zeros(0, np.int64)
        lens = self.lengths[idx].astype(np.int32)
        offs = np.zeros(len(idx), np.int64)
        if len(idx) > 1:
            offs[1:] = np.cumsum(lens[:-1])
        return ProfileSet(lens, offs, self.bkg[idx].copy(), self.eno[idx].copy(),
                          self.trn[trows].copy(), self.trg[pos].copy(), self.cv[pos].copy(),
                          self.cvprior[pos].copy(), self.cvnorm2[pos].copy(), self.ss[pos].copy(),
                          self.ssstate[pos].copy(), self.aa[pos].copy(),
                          self.trn_int[trows].copy(), self.trg_int[pos].copy())


def concat(sets: List[ProfileSet]) -> ProfileSet:
    lens = np.concatenate([s.lengths for s in sets]).astype(np.int32)
    offs = np.zeros(len(lens), np.int64)
    if len(lens) > 1:
        offs[1:] = np.cumsum(lens[:-1].astype(np.int64))
    cat = lambda name: np.concatenate([getattr(s, name) for s in sets])
    return ProfileSet(lens, offs, cat("bkg"), cat("eno"), cat("trn"), cat("trg"), cat("cv"),
                      cat("cvprior"), cat("cvnorm2"), cat("ss"), cat("ssstate"), cat("aa"),
                      cat("trn_int"), cat("trg_int"))


# ---------------------------------------------------------------------------
def _dirichlet(rng: np.random.Generator, alpha: np.ndarray) -> np.ndarray:
    """Row-wise Dirichlet samples for an [n, k] array of concentrations."""
    g = rng.standard_gamma(alpha)
    s = g.sum(axis=1, keepdims=True)
    bad = s[:, 0] <= 0
    if bad.any():  # all components underflowed: put the mass on the largest alpha
        g[bad] = 0.0
        g[bad, np.argmax(alpha[bad], axis=1)] = 1.0
        s = g.sum(axis=1, keepdims=True)
    return g / s


def _quantise(p: np.ndarray, floor: int = 1) -> np.ndarray:
    """Probabilities -> integers summing to SCALE per row, each >= floor."""
    q = np.rint(p * SCALE).astype(np.int64)
    q = np.maximum(q, floor)
    diff = SCALE - q.sum(axis=1)
    am = np.argmax(q, axis=1)
    q[np.arange(q.shape[0]), am] += diff
    if (q < floor).any():  # pathological rounding: redistribute from the largest
        raise ValueError("quantisation failed")
    return q.astype(np.int32)


def _fval(q: np.ndarray) -> np.ndarray:
    """Text-format integer -> float as the reader does: (float)int / (float)scale."""
    return (q.astype(np.float32) / np.float32(SCALE)).astype(np.float32)


def _trn_values(q: np.ndarray) -> np.ndarray:
    """Integer transition probabilities -> log-space working values."""
    p = _fval(q)
    with np.errstate(divide="ignore"):
        # log in double rounded once to float32 (a correctly rounded logf)
        lg = np.log(p.astype(np.float64)).astype(np.float32)
    lg[:, 3:] = (lg[:, 3:] * TRN_LOGFCT).astype(np.float32)
    lg[q == 0] = np.float32(LOG0)
    return lg


def _draw_transitions(rng, n) -> np.ndarray:
    a = np.array([10, 1, 1, 1, 1, 1, 1], np.float64)
    t = _dirichlet(rng, np.broadcast_to(a, (n, 7)).copy())
    m = _quantise(t[:, 0:3] / t[:, 0:3].sum(1, keepdims=True))
    i = _quantise(t[:, 3:5] / t[:, 3:5].sum(1, keepdims=True))
    d = _quantise(t[:, 5:7] / t[:, 5:7].sum(1, keepdims=True))
    return np.concatenate([m, i, d], axis=1)


def _positions(rng, n, trg_alpha=None):
    """Draw n profile positions; trg_alpha [n,20] overrides the emission prior."""
    if trg_alpha is None:
        trg_alpha = np.broadcast_to(0.5 * ROBINSON, (n, NUMAA)).copy()
    trg_int = _quantise(_dirichlet(rng, trg_alpha))
    cv_int = np.rint(rng.standard_normal((n, NCV)) * SCALE).astype(np.int64)
    cvf = _fval(cv_int)
    v64 = cvf.astype(np.float64)
    norm2 = (v64 * v64).sum(1)
    prior = -0.5 * norm2 - 0.5 * NCV * np.log(2.0 * np.pi)
    ssp = _dirichlet(rng, np.ones((n, 3)))
    ss_int = np.floor(ssp * SCALE).astype(np.int64)
    return trg_int, cv_int, np.rint(prior * SCALE), np.rint(norm2 * SCALE), ss_int


def _assemble(lengths, trg_int, cv_int, prior_int, norm2_int, ss_int, trn_int, eno):
    lengths = np.asarray(lengths, np.int32)
    P = lengths.shape[0]
    offs = np.zeros(P, np.int64)
    if P > 1:
        offs[1:] = np.cumsum(lengths[:-1].astype(np.int64))
    trg = _fval(trg_int)
    ssf = _fval(ss_int)
    return ProfileSet(
        lengths=lengths, offsets=offs,
        bkg=np.broadcast_to(_fval(np.rint(ROBINSON * SCALE)[None, :].astype(np.int64)), (P, NUMAA)).astype(np.float32).copy(),
        eno=np.asarray(eno, np.float32),
        trn=_trn_values(trn_int), trg=trg, cv=_fval(cv_int),
        cvprior=_fval(prior_int.astype(np.int64)), cvnorm2=_fval(norm2_int.astype(np.int64)),
        ss=ssf, ssstate=np.frombuffer(SSCH, np.uint8)[np.argmax(ss_int, axis=1)].copy(),
        aa=np.frombuffer(AA, np.uint8)[np.argmax(trg_int, axis=1)].copy(),
        trn_int=trn_int.astype(np.int32), trg_int=trg_int.astype(np.int32))


def random_profiles(rng: np.random.Generator, lengths: Sequence[int]) -> ProfileSet:
    lengths = np.asarray(lengths, np.int32)
    n = int(lengths.sum())
    P = lengths.shape[0]
    trg_int, cv_int, prior_int, norm2_int, ss_int = _positions(rng, n)
    trn_int = _draw_transitions(rng, n + P)
    eno = np.round(rng.uniform(1.0, 14.0, P), 1)
    return _assemble(lengths, trg_int, cv_int, prior_int, norm2_int, ss_int, trn_int, eno)


def lognormal_lengths(rng, n, median, sigma, lo, hi) -> np.ndarray:
    L = np.rint(np.exp(rng.normal(np.log(median), sigma, n)))
    return np.clip(L, lo, hi).astype(np.int32)


def planted_homolog(rng: np.random.Generator, query: ProfileSet, length: int,
                    seg_lo: int = 60, seg_hi: int = 300, conc: float = 50.0) -> ProfileSet:
    """A db profile holding a perturbed copy of a query segment.

    A query segment of length U[seg_lo, seg_hi] (at most the query length) is
    embedded at a random offset of a random profile; its emissions are drawn
    from Dirichlet(conc * query emissions), and its transitions, SS and context
    vectors are copied from the query segment.
    """
    Lq = int(query.lengths[0])
    ls = int(rng.integers(min(seg_lo, Lq), min(seg_hi, Lq) + 1))
    qs = int(rng.integers(0, Lq - ls + 1))
    L = max(int(length), ls)
    base = random_profiles(rng, [L])
    o = int(rng.integers(0, L - ls + 1))
    qtrg = query.trg_int[qs:qs + ls].astype(np.float64) / SCALE
    pert = _quantise(_dirichlet(rng, conc * qtrg))
    base.trg_int[o:o + ls] = pert
    base.trg[o:o + ls] = _fval(pert)
    base.aa[o:o + ls] = np.frombuffer(AA, np.uint8)[np.argmax(pert, axis=1)]
    for name in ("cv", "cvprior", "cvnorm2", "ss", "ssstate"):
        getattr(base, name)[o:o + ls] = getattr(query, name)[qs:qs + ls]
    # transitions into positions o..o+ls-1 and out of the segment's last one
    base.trn_int[o + 1:o + ls + 1] = query.trn_int[qs + 1:qs + ls + 1]
    base.trn[o + 1:o + ls + 1] = query.trn[qs + 1:qs + ls + 1]
    return base


# ---------------------------------------------------------------------------
# benchmark configurations
@dataclass
class Workload:
    name: str
    queries: List[ProfileSet]
    db: ProfileSet
    homologs: np.ndarray  # indices of planted homologs in db

    @property
    def cells(self) -> int:
        return int(sum(int(q.lengths[0]) for q in self.queries)) * int(self.db.lengths.sum())


def make_db(rng, lengths, query: Optional[ProfileSet] = None, frac_homolog: float = 0.0,
            chunk: int = 2_000_000) -> (ProfileSet, np.ndarray):
    lengths = np.asarray(lengths, np.int32)
    P = lengths.shape[0]
    hom = np.zeros(0, np.int64)
    if query is not None and frac_homolog > 0:
        nh = int(round(frac_homolog * P))
        hom = np.sort(rng.choice(P, nh, replace=False))
    homset = set(hom.tolist())
    parts: List[ProfileSet] = []
    k = 0
    while k < P:
        # a run of random profiles up to the next homolog, in chunks of positions
        j = k
        acc = 0
        while j < P and j not in homset and acc < chunk:
            acc += int(lengths[j])
            j += 1
        if j > k:
            parts.append(random_profiles(rng, lengths[k:j]))
            k = j
        if k < P and k in homset:
            parts.append(planted_homolog(rng, query, int(lengths[k])))
            k += 1
    db = concat(parts)
    return db, hom


def config(n: int, seed: int = 0, scale: float = 1.0) -> Workload:
    """Benchmark configuration n (0..4); ``scale`` shrinks the database size."""
    rng = np.random.default_rng(seed * 1000 + n)
    if n == 0:
        q = random_profiles(rng, [150])
        ndb = max(1, int(2000 * scale))
        db, hom = make_db(rng, rng.integers(50, 501, ndb))
        return Workload("1x150 vs %d profiles U[50,500]" % ndb, [q], db, hom)
    if n == 1:
        q = random_profiles(rng, [400])
        ndb = max(1, int(100_000 * scale))
        db, hom = make_db(rng, lognormal_lengths(rng, ndb, 200, 0.6, 30, 2000), q, 0.02)
        return Workload("1x400 vs %d profiles LN(200,0.6)[30,2000], 2%% homologs" % ndb, [q], db, hom)
    if n == 2:
        nq = max(1, int(64 * min(1.0, scale * 4)))
        qs = [random_profiles(rng, [L]) for L in lognormal_lengths(rng, nq, 250, 0.6, 50, 1500)]
        ndb = max(1, int(20_000 * scale))
        db, hom = make_db(rng, lognormal_lengths(rng, ndb, 200, 0.6, 30, 2000), qs[0], 0.02)
        return Workload("%d queries LN(250,0.6)[50,1500] vs %d profiles" % (nq, ndb), qs, db, hom)
    if n == 3:
        npair = max(1, int(256 * scale))
        qs = [random_profiles(rng, [L]) for L in rng.integers(100, 601, npair)]
        db = random_profiles(rng, rng.integers(100, 601, npair))
        return Workload("%d pairs U[100,600]" % npair, qs, db, np.zeros(0, np.int64))
    if n == 4:
        doms = [random_profiles(rng, [500]) for _ in range(6)]
        q = concat(doms)
        q = ProfileSet(np.array([3000], np.int32), np.zeros(1, np.int64), q.bkg[:1], q.eno[:1],
                       _joined_trn(doms), q.trg, q.cv, q.cvprior, q.cvnorm2, q.ss, q.ssstate, q.aa,
                       _joined_trn_int(doms), q.trg_int)
        ndb = max(1, int(50_000 * scale))
        db, hom = make_db(rng, lognormal_lengths(rng, ndb, 300, 0.6, 30, 2000), q, 0.05)
        return Workload("1x3000 (6 domains) vs %d profiles LN(300,0.6)[30,2000], 5%% homologs" % ndb,
                        [q], db, hom)
    raise ValueError(n)


def _joined_trn(doms):
    rows = [doms[0].trn[0:1]] + [d.trn[1:] for d in doms]
    return np.concatenate(rows)


def _joined_trn_int(doms):
    rows = [doms[0].trn_int[0:1]] + [d.trn_int[1:] for d in doms]
    return np.concatenate(rows)
