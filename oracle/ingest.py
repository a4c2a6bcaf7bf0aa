"""CPU restatement of the reference's alignment ingest (test infrastructure only: the checker
of gems_compress_alignment; never used by the product path).

- convert_state: characters -> state codes, alignment/alignment.cpp:1856-1958 (convertState),
  sequences upper-cased first (:2451);
- build_patterns: one site after another, a new column becomes the next pattern, a repeated
  one adds to its pattern's frequency (buildPattern :1240-1268, addPatternLazy :1511-1543);
- const_char: computeConst :1321-1420 with getAppearance :5567-5600;
- site_stat / site_summary: the pattern flags of computeConst (:1365-1371, :1410-1451), the
  per-site statistic of printSiteInfo (:1455-1477) and the counts of countConstSite
  (:4822-4843) that the program's report prints.
"""
from __future__ import annotations

import numpy as np

DNA_UNKNOWN, PROTEIN_UNKNOWN = 18, 23


def _unknown(n):
    return {4: DNA_UNKNOWN, 20: PROTEIN_UNKNOWN}.get(n, n)


def convert_state(ch: str, n: int) -> int:
    """State code of one character; -1 for a character the reference rejects."""
    c = ch.upper()
    unk = _unknown(n)
    if c in "?-.~":
        return unk
    if n == 4:
        table = {"A": 0, "C": 1, "G": 2, "T": 3, "U": 3, "R": 1 + 4 + 3, "Y": 2 + 8 + 3,
                 "W": 1 + 8 + 3, "S": 2 + 4 + 3, "M": 1 + 2 + 3, "K": 4 + 8 + 3,
                 "B": 2 + 4 + 8 + 3, "H": 1 + 2 + 8 + 3, "D": 1 + 4 + 8 + 3, "V": 1 + 2 + 4 + 3,
                 "O": unk, "N": unk, "X": unk}
        return table.get(c, -1)
    if n == 20:
        special = {"B": 20, "Z": 21, "J": 22, "*": unk, "U": unk, "O": unk, "X": unk}
        if c in special:
            return special[c]
        i = "ARNDCQEGHILKMFPSTWYV".find(c)
        return i if i >= 0 else -1
    raise ValueError("characters are read for 4 and 20 states")


def encode(seqs: list[str], n: int) -> np.ndarray:
    out = np.array([[convert_state(ch, n) for ch in s] for s in seqs], dtype=np.int16)
    if (out < 0).any():
        raise ValueError("unrecognised character")
    return out.astype(np.uint8)


def appearance(code: int, n: int) -> set:
    unk = _unknown(n)
    if code >= unk:
        return set(range(n))
    if code < n:
        return {code}
    if n == 4:
        return {j for j in range(4) if (code - 3) & (1 << j)}
    return {20: {2, 3}, 21: {5, 6}, 22: {9, 10}}[code]


def const_char(column, n: int) -> int:
    unk = _unknown(n)
    app = set(range(n))
    for c in column:
        app &= appearance(int(c), n)
    if len(app) == n:
        return unk
    if len(app) == 1:
        return min(app)
    if len(app) > 1 and n == 4:
        return n - 1 + sum(1 << j for j in app)
    if len(app) > 1 and n == 20:
        return {frozenset({2, 3}): 20, frozenset({5, 6}): 21, frozenset({9, 10}): 22}[frozenset(app)]
    return unk + 1


def build_patterns(codes: np.ndarray, n: int):
    """(patterns [ntaxa][npat], weights [npat], site_pattern [nsites], const_char [npat])."""
    index, cols, weights, site_pattern = {}, [], [], []
    for s in range(codes.shape[1]):
        key = codes[:, s].tobytes()
        p = index.get(key)
        if p is None:
            p = len(cols)
            index[key] = p
            cols.append(codes[:, s].copy())
            weights.append(0)
        weights[p] += 1
        site_pattern.append(p)
    pat = np.stack(cols, axis=1)
    cc = np.array([const_char(pat[:, p], n) for p in range(pat.shape[1])], dtype=np.uint8)
    return pat, np.array(weights, np.float64), np.array(site_pattern, np.int32), cc


# per-site statistic codes, in printSiteInfo's letters: I, C, c, U, -
STAT_INFORMATIVE, STAT_CONST, STAT_CONST_AMBIG, STAT_UNINFORMATIVE, STAT_ALL_GAP = range(5)


def pattern_flags(column, n: int):
    """(is_const, is_informative, const_char) of one pattern: const when some state is
    compatible with every character (is_const and is_invariant coincide there); informative
    when at least two unambiguous states appear at least twice each."""
    cc = const_char(column, n)
    counts = np.bincount(np.asarray([c for c in column if c < n], np.int64), minlength=n)
    informative = int((counts >= 2).sum()) >= 2
    return cc <= _unknown(n), informative, cc


def site_stat(column, n: int) -> int:
    is_const, informative, cc = pattern_flags(column, n)
    if informative:
        return STAT_INFORMATIVE
    if is_const:
        if cc == _unknown(n):
            return STAT_ALL_GAP
        return STAT_CONST if cc < n else STAT_CONST_AMBIG
    return STAT_UNINFORMATIVE


def site_summary(patterns: np.ndarray, weights: np.ndarray, n: int):
    """(constant, invariant, informative, distinct) site counts as countConstSite forms them."""
    const = inform = 0
    for p in range(patterns.shape[1]):
        is_const, informative, _ = pattern_flags(patterns[:, p], n)
        const += int(weights[p]) if is_const else 0
        inform += int(weights[p]) if informative else 0
    return const, const, inform, patterns.shape[1]
