"""Seeded synthetic workloads for the likelihood path.

Builds the inputs the kernels run on, with the shapes and value distributions of the
benchmark configurations: random unrooted binary trees with exponential branch lengths,
reversible models (GTR for DNA, a symmetric 20x20 exchangeability matrix for protein, a
Goldman-Yang style codon model for 61 sense codons), discrete-Gamma or free-rate categories,
sequences simulated down the tree, gap cells coded as the all-ones tip state, and pattern
compression with integer weights.  The heavy loops live in ``csrc/synth.c``.

Nothing here computes likelihoods; it only prepares data.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

from . import _lib

# state codes of the converted alignment (tip state bytes)
DNA_UNKNOWN = 18      # alignment.cpp: STATE_UNKNOWN for DNA (4 + 14 ambiguity codes)
PROTEIN_UNKNOWN = 23  # 20 amino acids + B, Z, J
CODON_UNKNOWN = 61    # number of sense codons of the standard code


def state_unknown(nstates: int) -> int:
    return {4: DNA_UNKNOWN, 20: PROTEIN_UNKNOWN}.get(nstates, nstates)


@dataclasses.dataclass
class Model:
    nstates: int
    exch_upper: np.ndarray   # n(n-1)/2 exchangeabilities, row-major upper triangle
    freq: np.ndarray         # n state frequencies
    rates: np.ndarray        # category rates (mean 1)
    props: np.ndarray        # category proportions
    eval: np.ndarray = None
    evec: np.ndarray = None
    inv_evec: np.ndarray = None
    p_invar: float = 0.0
    gamma_shape: float = 0.0

    def __post_init__(self):
        if self.eval is None:
            self.eval, self.evec, self.inv_evec = eigensystem(self.exch_upper, self.freq)

    @property
    def ncat(self) -> int:
        return len(self.rates)


@dataclasses.dataclass
class Tree:
    ntaxa: int
    eu: np.ndarray   # int32 edge endpoints
    ev: np.ndarray
    length: np.ndarray

    @property
    def nedges(self) -> int:
        return len(self.eu)

    @property
    def nnodes(self) -> int:
        return len(self.eu) + 1

    def newick(self, names=None, prec: int = 17) -> str:
        """Newick string rooted at the internal node ``ntaxa`` (a trifurcation)."""
        n = self.nnodes
        adj = [[] for _ in range(n)]
        for u, v, l in zip(self.eu, self.ev, self.length):
            adj[u].append((v, l))
            adj[v].append((u, l))
        names = names or [f"T{i}" for i in range(self.ntaxa)]
        root = self.ntaxa if n > self.ntaxa else 0

        def rec(u, parent):
            kids = [(v, l) for v, l in adj[u] if v != parent]
            if not kids:
                return names[u]
            return "(" + ",".join(f"{rec(v, u)}:{l:.{prec}g}" for v, l in kids) + ")"

        return rec(root, -1) + ";"


@dataclasses.dataclass
class Alignment:
    ntaxa: int
    nstates: int
    nsites: int
    patterns: np.ndarray  # uint8 [ntaxa][npat]
    weights: np.ndarray   # float64 [npat]

    @property
    def npat(self) -> int:
        return self.patterns.shape[1]

    def const_char(self) -> np.ndarray:
        """Constant state of each pattern (reference Pattern::const_char): the common state
        when all known states agree, STATE_UNKNOWN when all are unknown, else unknown+1."""
        unk = state_unknown(self.nstates)
        pat = self.patterns
        known = pat < self.nstates
        out = np.full(self.npat, unk + 1, dtype=np.uint8)
        anyk = known.any(axis=0)
        first = np.where(known, pat, 255).min(axis=0)
        same = np.all(np.where(known, pat == first[None, :], True), axis=0)
        out[anyk & same] = first[anyk & same]
        out[~anyk] = unk
        return out


def eigensystem(exch_upper, freq):
    """Eigensystem of the reversible rate matrix normalised to one substitution per site:
    Q = S diag(pi) with zero row sums, symmetrised as diag(sqrt pi) Q diag(1/sqrt pi).
    Returns (eval, evec, inv_evec) with Q = evec diag(eval) inv_evec, row-major."""
    freq = np.asarray(freq, dtype=np.float64)
    freq = freq / freq.sum()
    n = len(freq)
    s = np.zeros((n, n))
    iu = np.triu_indices(n, 1)
    s[iu] = exch_upper
    s = s + s.T
    q = s * freq[None, :]
    np.fill_diagonal(q, 0.0)
    rowsum = q.sum(axis=1)
    q -= np.diag(rowsum)
    q /= float(rowsum @ freq)
    sq = np.sqrt(freq)
    a = (sq[:, None] * q) / sq[None, :]
    a = 0.5 * (a + a.T)
    w, v = np.linalg.eigh(a)
    evec = v / sq[:, None]
    inv_evec = v.T * sq[None, :]
    return w.copy(), np.ascontiguousarray(evec), np.ascontiguousarray(inv_evec)


def gamma_rates(alpha: float, ncat: int) -> np.ndarray:
    """Discrete Gamma(alpha, alpha) category rates by the mean method (Yang 1994)."""
    from scipy.special import gammainc, gammaincinv
    if ncat == 1:
        return np.ones(1)
    cuts = gammaincinv(alpha, np.arange(1, ncat) / ncat) / alpha
    cdf = np.concatenate([[0.0], gammainc(alpha + 1, cuts * alpha), [1.0]])
    return np.diff(cdf) * ncat


def dna_gtr(rng: np.random.Generator, ncat=4, alpha=0.5) -> Model:
    exch = rng.uniform(0.5, 2.0, 6)
    exch = exch / exch[5]          # GT = 1, as in the GTR{a,b,c,d,e} parameterisation
    freq = rng.dirichlet(np.ones(4))
    return Model(4, exch, freq, gamma_rates(alpha, ncat), np.full(ncat, 1.0 / ncat),
                 gamma_shape=alpha)


def protein(rng: np.random.Generator, ncat=4, alpha=0.8) -> Model:
    exch = rng.lognormal(0.0, 1.0, 190)
    freq = rng.dirichlet(np.ones(20))
    return Model(20, exch, freq, gamma_rates(alpha, ncat), np.full(ncat, 1.0 / ncat),
                 gamma_shape=alpha)


_BASES = "TCAG"
_AA = "FFLLSSSSYY**CC*WLLLLPPPPHHQQRRRRIIIMTTTTNNKKSSRRVVVVAAAADDEEGGGG"


def codon_sense():
    """Standard genetic code: the 61 sense codons (TCAG order) and their amino acids."""
    cods, aas = [], []
    for i, a in enumerate(_AA):
        if a != "*":
            cods.append(_BASES[i // 16] + _BASES[(i // 4) % 4] + _BASES[i % 4])
            aas.append(a)
    return cods, aas


def gy_exchangeabilities(omega: float, kappa: float) -> np.ndarray:
    """Goldman-Yang exchangeabilities over the 61 sense codons (upper triangle, row-major):
    kappa for a transition, times omega for a non-synonymous change, 0 for codons differing
    at more than one position (model/modelcodon.cpp:366, GY with fixed kappa and omega)."""
    cods, aas = codon_sense()
    n = len(cods)
    purine = set("AG")
    exch = []
    for i in range(n):
        for j in range(i + 1, n):
            diff = [k for k in range(3) if cods[i][k] != cods[j][k]]
            if len(diff) != 1:
                exch.append(0.0)
                continue
            a, b = cods[i][diff[0]], cods[j][diff[0]]
            r = kappa if ((a in purine) == (b in purine)) else 1.0
            if aas[i] != aas[j]:
                r *= omega
            exch.append(r)
    return np.array(exch)


def codon_gy(rng: np.random.Generator, ncat=4, alpha=0.5, freerate=False) -> Model:
    """Goldman-Yang style codon model: omega ~ U[0.1,1], kappa ~ U[1,5], frequencies
    ~ Dirichlet(1^61); +G (mean rates) or a free-rate model with ncat categories."""
    n = len(codon_sense()[0])
    omega = rng.uniform(0.1, 1.0)
    kappa = rng.uniform(1.0, 5.0)
    freq = rng.dirichlet(np.ones(n))
    exch = gy_exchangeabilities(omega, kappa)
    if freerate:
        props = rng.dirichlet(np.ones(ncat))
        rates = np.sort(rng.gamma(1.0, 1.0, ncat))
        rates = rates / float(rates @ props)
    else:
        props = np.full(ncat, 1.0 / ncat)
        rates = gamma_rates(alpha, ncat)
    return Model(n, exch, freq, rates, props, gamma_shape=alpha)


def random_tree(ntaxa: int, mean_len: float, seed: int) -> Tree:
    ne = 2 * ntaxa - 3
    eu = np.zeros(ne, np.int32)
    ev = np.zeros(ne, np.int32)
    ln = np.zeros(ne, np.float64)
    got = _lib.synth().gems_synth_tree(ntaxa, ctypes.c_double(mean_len), ctypes.c_uint64(seed),
                                       _ptr(eu), _ptr(ev), _ptr(ln))
    assert got == ne
    return Tree(ntaxa, eu, ev, ln)


def simulate(tree: Tree, model: Model, nsites: int, seed: int, gap_frac=0.0) -> Alignment:
    n = model.nstates
    out = np.empty((tree.ntaxa, nsites), np.uint8)
    rc = _lib.synth().gems_synth_simulate(
        tree.ntaxa, tree.nedges, _ptr(tree.eu), _ptr(tree.ev), _ptr(tree.length), n, model.ncat,
        _ptr(np.ascontiguousarray(model.rates, np.float64)),
        _ptr(np.ascontiguousarray(model.props, np.float64)),
        _ptr(model.eval), _ptr(model.evec), _ptr(model.inv_evec),
        _ptr(np.ascontiguousarray(model.freq, np.float64)), ctypes.c_longlong(nsites),
        ctypes.c_double(gap_frac), state_unknown(n), ctypes.c_uint64(seed), _ptr(out))
    assert rc == 0
    return compress(out, n)


def compress(aln: np.ndarray, nstates: int) -> Alignment:
    ntaxa, nsites = aln.shape
    aln = np.ascontiguousarray(aln, np.uint8)
    pat = np.empty((ntaxa, nsites), np.uint8)
    w = np.empty(nsites, np.float64)
    npat = _lib.synth().gems_synth_compress(ntaxa, ctypes.c_longlong(nsites), _ptr(aln),
                                            _ptr(pat), _ptr(w))
    pat = np.ascontiguousarray(pat.reshape(-1)[: ntaxa * npat].reshape(ntaxa, npat))
    return Alignment(ntaxa, nstates, nsites, pat, w[:npat].copy())


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------------------
# the benchmark configurations (seeded)
# ---------------------------------------------------------------------------------------

def config_dna16(seed=1, nsites=10_000):
    """FP64 DNA GTR+G4 on 16 taxa, lengths ~Exp(0.1), 10,000 sites."""
    rng = np.random.default_rng(seed)
    model = dna_gtr(rng, 4, 0.5)
    tree = random_tree(16, 0.1, seed + 11)
    aln = simulate(tree, model, nsites, seed + 23)
    return tree, model, aln


def config_dna512(seed=2, nsites=1_000_000, gap_frac=0.05):
    """DNA GTR+G4 on 512 taxa, lengths ~Exp(0.05), 1,000,000 sites, 5% gap cells."""
    rng = np.random.default_rng(seed)
    model = dna_gtr(rng, 4, 0.5)
    tree = random_tree(512, 0.05, seed + 11)
    aln = simulate(tree, model, nsites, seed + 23, gap_frac=gap_frac)
    return tree, model, aln


def config_protein128(seed=3, nsites=100_000):
    """20-state protein +G4 (shape 0.8) on 128 taxa, lengths ~Exp(0.15), 100,000 sites."""
    rng = np.random.default_rng(seed)
    model = protein(rng, 4, 0.8)
    tree = random_tree(128, 0.15, seed + 11)
    aln = simulate(tree, model, nsites, seed + 23)
    return tree, model, aln


def config_codon200(seed=4, nsites=4000, freerate=False):
    """61-state codon model (+G4 or +R8) on 200 taxa, 4,000 sites."""
    rng = np.random.default_rng(seed)
    model = codon_gy(rng, 8 if freerate else 4, 0.5, freerate=freerate)
    tree = random_tree(200, 0.1, seed + 11)
    aln = simulate(tree, model, nsites, seed + 23)
    return tree, model, aln


def write_fasta(path, aln_cols: np.ndarray, nstates: int, names=None):
    """Write an alignment [ntaxa][nsites] of state bytes as FASTA (DNA or protein letters,
    '-' for the unknown state)."""
    letters = {4: "ACGT", 20: "ARNDCQEGHILKMFPSTWYV"}[nstates]
    unk = state_unknown(nstates)
    lut = np.frombuffer((letters + "?" * (256 - len(letters))).encode(), np.uint8).copy()
    lut[unk] = ord("-")
    names = names or [f"T{i}" for i in range(aln_cols.shape[0])]
    with open(path, "w") as f:
        for i, row in enumerate(aln_cols):
            f.write(f">{names[i]}\n{lut[row].tobytes().decode()}\n")


def expand_patterns(aln: Alignment) -> np.ndarray:
    """Alignment columns from patterns and integer weights (pattern order)."""
    reps = aln.weights.astype(np.int64)
    return np.repeat(aln.patterns, reps, axis=1)


if os.environ.get("GEMS_SYNTH_SELFTEST"):
    t = random_tree(5, 0.1, 1)
    print(t.newick())
