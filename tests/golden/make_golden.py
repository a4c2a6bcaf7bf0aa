"""Generate the golden fixtures under tests/golden/ by running the reference program.

The reference IQ-TREE ships a prebuilt IQ-TREE 2.4.0 executable
(test_scripts/iqtree2/Linux-intel/iqtree2) that runs on this kind of host.  It is executed
as a black box -- never inspected -- on seeded synthetic cases and on the reference's own
test data (test_scripts/test_data/turtle.fa, turtle.trees), with every model parameter fixed
and `-prec 12` so the report prints 12 decimals:

  * `-blfix`      : log-likelihood of the tree at the given branch lengths, the discrete
                    Gamma category rates, and per-site log-likelihoods (`-wsl`, 6 digits);
  * no `-blfix`   : log-likelihood and branch lengths after the program's branch-length
                    optimisation (optimizeAllBranches to convergence);
  * `-safe`       : the same with the SAFE (per-category) scaling kernel.

Each case is saved as <name>.npz holding the inputs (compressed patterns, tree, model
parameters) and the program's outputs.  A 61-state codon case (GY with omega and kappa fixed,
`-st CODON`) pins the codon model and the 61-state kernels the same way.

The ingest fixtures under ingest/ pin the alignment reading and pattern compression on the
reference's own test alignments (turtle.fa, turtle_aa.fasta, example.phy): the raw
characters, the program's distinct-pattern count and site summary counts, its per-site
statistic (`-alninfo`: informative / constant / ambiguous-constant / uninformative / all-gap)
and its per-site log-likelihoods at a fixed model and tree.

Re-run with

    python tests/golden/make_golden.py --ref <iqtree source tree> [--only name ...]

or with the source tree in the IQTREE_SOURCE environment variable.  This script needs the
reference tree; the committed .npz fixtures do not.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gems_b200 import synth  # noqa: E402
from oracle import oracle as orc  # noqa: E402

IUPAC = {1: "A", 2: "C", 4: "G", 8: "T", 5: "R", 10: "Y", 6: "S", 9: "W", 12: "K", 3: "M",
         14: "B", 13: "D", 11: "H", 7: "V"}
DNA = "ACGT"
AA = "ARNDCQEGHILKMFPSTWYV"


def dna_letter(state):
    if state < 4:
        return DNA[state]
    if state == 18:
        return "-"
    return IUPAC[state - 3]  # ambiguity code: bitmask = state - 3


def write_fasta(path, cols, nstates, names):
    with open(path, "w") as f:
        for i, row in enumerate(cols):
            if nstates == 4:
                s = "".join(dna_letter(int(x)) for x in row)
            else:
                s = "".join(AA[x] if x < 20 else "-" for x in row)
            f.write(f">{names[i]}\n{s}\n")


def parse_newick(s):
    """Returns (names, edges) with edges as (parent_index, child_index, length); nodes are
    numbered in parse order."""
    s = s.strip().rstrip(";")
    pos = 0
    nodes = []  # name or None
    edges = []

    def parse():
        nonlocal pos
        me = len(nodes)
        nodes.append(None)
        if s[pos] == "(":
            pos += 1
            while True:
                child = parse()
                ln = 0.0
                if pos < len(s) and s[pos] == ":":
                    pos += 1
                    m = re.match(r"[-+0-9.eE]+", s[pos:])
                    ln = float(m.group(0))
                    pos += len(m.group(0))
                edges.append((me, child, ln))
                if s[pos] == ",":
                    pos += 1
                    continue
                if s[pos] == ")":
                    pos += 1
                    break
            m = re.match(r"[^:,();]*", s[pos:])  # internal label / support
            pos += len(m.group(0))
        else:
            m = re.match(r"[^:,();]+", s[pos:])
            nodes[me] = m.group(0)
            pos += len(m.group(0))
        return me

    parse()
    return nodes, edges


def splits_to_lengths(nodes, edges, names):
    """Map each edge of a parsed Newick tree to its split (frozenset of taxon names on the
    child side) -> length."""
    kids = {}
    for p, c, ln in edges:
        kids.setdefault(p, []).append((c, ln))
    out = {}

    def below(u):
        if nodes[u] is not None:
            return {nodes[u]}
        acc = set()
        for c, ln in kids.get(u, []):
            b = below(c)
            out[frozenset(b)] = ln
            acc |= b
        return acc

    allset = below(0)
    canon = {}
    for sp, ln in out.items():
        other = frozenset(allset - sp)
        key = min(sp, other, key=lambda x: sorted(x))
        canon[key] = canon.get(key, 0.0) + ln  # root edges of a bifurcating root merge
    return canon


def tree_splits(tree, names):
    """Split key of each edge of a synth.Tree (same canonical form)."""
    n = tree.nnodes
    adj = [[] for _ in range(n)]
    for e, (u, v) in enumerate(zip(tree.eu, tree.ev)):
        adj[u].append((v, e))
        adj[v].append((u, e))
    allset = frozenset(names[:tree.ntaxa])
    keys = [None] * tree.nedges

    def side(u, parent):
        if u < tree.ntaxa:
            return {names[u]}
        acc = set()
        for v, e in adj[u]:
            if v == parent:
                continue
            b = side(v, u)
            sp = frozenset(b)
            keys[e] = min(sp, frozenset(allset - sp), key=lambda x: sorted(x))
            acc |= b
        return acc

    root = tree.ntaxa
    side(root, -1)
    return keys


def run_iqtree(binary, aln_path, tree_path, model, workdir, prefix, extra=()):
    cmd = [binary, "-s", aln_path, "-te", tree_path, "-m", model, "-T", "1", "-prec", "12",
           "-redo", "-pre", os.path.join(workdir, prefix), "-seed", "1"] + list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    rep = open(os.path.join(workdir, prefix + ".iqtree")).read()
    log = r.stdout
    lnl = float(re.search(r"Log-likelihood of the tree: (-?[0-9.]+)", rep).group(1))
    rates = [float(x) for x in re.findall(r"^\s+\d+\s+([0-9.eE+-]+)\s+[0-9.eE+-]+\s*$", rep,
                                          re.M)]
    out = {"lnl": lnl, "rates": rates, "log": log, "report": rep}
    sl = os.path.join(workdir, prefix + ".sitelh")
    if os.path.exists(sl):
        lines = open(sl).read().split("\n")
        out["site_lnl"] = np.array([float(x) for x in lines[1].split()[1:]])
    tf = os.path.join(workdir, prefix + ".treefile")
    out["treefile"] = open(tf).read().strip()
    return out


def paml_file(path, model):
    n = 20
    s = np.zeros((n, n))
    iu = np.triu_indices(n, 1)
    s[iu] = model.exch_upper
    s = s + s.T
    with open(path, "w") as f:
        for i in range(1, n):
            f.write(" ".join(f"{s[i, j]:.17g}" for j in range(i)) + "\n")
        f.write("\n" + " ".join(f"{x:.17g}" for x in model.freq) + "\n")


def codon_case(binary, workdir, name="codon12_g4"):
    """GY codon model with omega, kappa, the 61 frequencies and the Gamma shape fixed; 12 taxa,
    1,500 codon sites with 3% gap codons; the program runs it with -st CODON."""
    rng = np.random.default_rng(606)
    omega, kappa = rng.uniform(0.1, 1.0), rng.uniform(1.0, 5.0)
    cods, _ = synth.codon_sense()
    freq = rng.dirichlet(np.ones(len(cods)))
    alpha, ncat = 0.6, 4
    model = synth.Model(61, synth.gy_exchangeabilities(omega, kappa), freq,
                        orc.gamma_rates(alpha, ncat), np.full(ncat, 1.0 / ncat),
                        gamma_shape=alpha)
    tree = synth.random_tree(12, 0.15, 611)
    aln = synth.simulate(tree, model, 1500, 623, gap_frac=0.03)
    names = [f"T{i}" for i in range(tree.ntaxa)]
    cols = synth.expand_patterns(aln)
    fa = os.path.join(workdir, name + ".fa")
    with open(fa, "w") as f:
        for i, row in enumerate(cols):
            f.write(f">{names[i]}\n" + "".join(cods[x] if x < 61 else "---" for x in row) + "\n")
    nwk = os.path.join(workdir, name + ".nwk")
    open(nwk, "w").write(tree.newick(names))
    # the program orders codons by nucleotides A < C < G < T
    order = sorted(range(61), key=lambda i: ["ACGT".index(c) for c in cods[i]])
    mstr = (f"GY{{{omega:.17g},{kappa:.17g}}}+F{{" +
            ",".join(f"{freq[i]:.17g}" for i in order) + f"}}+G{ncat}{{{alpha:.17g}}}")
    extra = ["-st", "CODON", "-safe"]
    fixed = run_iqtree(binary, fa, nwk, mstr, workdir, name + "_fix", ["-blfix", "-wsl"] + extra)
    if "not present" in fixed["log"]:
        raise RuntimeError("a codon state is absent: the program would drop it from the model")
    # With every model parameter fixed the program does not re-optimise the branch lengths of
    # a codon model given by -te (its report shows one round and the input lengths), so this
    # case carries no optimised lengths.
    reps = aln.weights.astype(np.int64)
    first = np.concatenate([[0], np.cumsum(reps)[:-1]])
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        nstates=61, ntaxa=tree.ntaxa, eu=tree.eu, ev=tree.ev, length=tree.length,
        exch_upper=model.exch_upper, freq=freq, alpha=alpha, ncat=ncat, p_invar=0.0,
        rates=model.rates, props=model.props, patterns=aln.patterns, weights=aln.weights,
        const_char=aln.const_char(), safe=1, omega=omega, kappa=kappa,
        ref_lnl_fixed=fixed["lnl"], ref_rates=np.array(fixed["rates"]),
        ref_pattern_lnl_6sig=fixed["site_lnl"][first], model_string=mstr)
    print(f"{name}: npat={aln.npat} lnl_fixed={fixed['lnl']!r}")


def read_phylip(path):
    """Sequential PHYLIP: a header 'ntaxa nsites', then a name and its sequence per taxon."""
    lines = [ln.rstrip("\n") for ln in open(path)]
    ntaxa, nsites = (int(x) for x in lines[0].split()[:2])
    names, seqs = [], []
    for ln in lines[1:]:
        if not ln.strip():
            continue
        if len(names) < ntaxa and (not seqs or len(seqs[-1]) >= nsites):
            parts = ln.split()
            names.append(parts[0])
            seqs.append("".join(parts[1:]))
        else:
            seqs[-1] += "".join(ln.split())
    assert len(names) == ntaxa and all(len(x) == nsites for x in seqs)
    return names, seqs


def tree_from_treefile(treefile, names):
    """A program-written Newick tree as a synth.Tree with leaves numbered in sequence order."""
    nd, ed = parse_newick(treefile)
    leaf_idx = {nm: i for i, nm in enumerate(names)}
    ntaxa = len(names)
    mp, nxt = {}, ntaxa
    for i, nm in enumerate(nd):
        if nm is not None:
            mp[i] = leaf_idx[nm]
        else:
            mp[i] = nxt
            nxt += 1
    eu = np.array([mp[p] for p, c, ln in ed], np.int32)
    ev = np.array([mp[c] for p, c, ln in ed], np.int32)
    ln = np.array([l for p, c, l in ed])
    return synth.Tree(ntaxa, eu, ev, ln)


STAT_CODE = {"I": 0, "C": 1, "c": 2, "U": 3, "-": 4}


def ingest_case(binary, ref, workdir, fname, nstates, seed):
    """One of the reference's test alignments: raw characters, the program's pattern and site
    statistics, and its per-site lnL at a fixed seeded model on the tree the program builds
    for the file (`-n 0`)."""
    path = os.path.join(ref, "test_scripts", "test_data", fname)
    names, seqs = read_phylip(path) if fname.endswith(".phy") else read_fasta_raw(path)
    start = run_iqtree_plain(binary, path, "JC" if nstates == 4 else "LG", workdir,
                             "start_" + fname, ["-n", "0"])
    tree = tree_from_treefile(start["treefile"], names)
    tree_path = os.path.join(workdir, "tree_" + fname + ".nwk")
    open(tree_path, "w").write(start["treefile"])
    rng = np.random.default_rng(seed)
    alpha, ncat = 0.7, 4
    if nstates == 4:
        m = synth.dna_gtr(rng, ncat, alpha)
        ex = m.exch_upper / m.exch_upper[5]
        mstr = ("GTR{" + ",".join(f"{x:.17g}" for x in ex[:5]) + "}+F{" +
                ",".join(f"{x:.17g}" for x in m.freq) + "}")
    else:
        m = synth.protein(rng, ncat, alpha)
        pf = os.path.join(workdir, fname + ".paml")
        paml_file(pf, m)
        mstr = pf
    mstr += f"+G{ncat}{{{alpha:.17g}}}"
    out = run_iqtree(binary, path, tree_path, mstr, workdir, "fix_" + fname,
                     ["-blfix", "-wsl", "-alninfo"])
    rep = out["report"]

    def count(label):
        return int(re.search(label + r": (\d+)", rep).group(1))

    stat_lines = open(os.path.join(workdir, "fix_" + fname + ".alninfo")).read().split("\n")
    stats = [ln.split("\t") for ln in stat_lines if ln and not ln.startswith("#")][1:]
    site_stat = np.array([STAT_CODE[st] for _, st in stats], np.uint8)
    raw = np.array([np.frombuffer(s.encode(), np.uint8) for s in seqs])
    key = os.path.splitext(fname)[0]
    np.savez_compressed(
        os.path.join(HERE, "ingest", key + ".npz"),
        source=fname, nstates=nstates, chars=raw, ntaxa=len(names), eu=tree.eu, ev=tree.ev,
        length=tree.length, exch_upper=m.exch_upper, freq=m.freq, alpha=alpha,
        rates=orc.gamma_rates(alpha, ncat), props=np.full(ncat, 1.0 / ncat),
        ref_lnl=out["lnl"], ref_site_lnl_6sig=out["site_lnl"], ref_site_stat=site_stat,
        ref_distinct=count("Number of distinct site patterns"),
        ref_const=count("Number of constant sites"),
        ref_invariant=count(r"Number of invariant \(constant or ambiguous constant\) sites"),
        ref_informative=count("Number of parsimony informative sites"), model_string=mstr)
    print(f"ingest/{key}: sites={raw.shape[1]} distinct={count('Number of distinct site patterns')}"
          f" lnl={out['lnl']!r}")


def read_fasta_raw(path):
    """FASTA with the characters as written (no case change)."""
    names, seqs = [], []
    for line in open(path):
        line = line.strip()
        if line.startswith(">"):
            names.append(line[1:].split()[0])
            seqs.append([])
        elif line:
            seqs[-1].append(line)
    return names, ["".join(s) for s in seqs]


def run_iqtree_plain(binary, aln_path, model, workdir, prefix, extra=()):
    cmd = [binary, "-s", aln_path, "-m", model, "-T", "1", "-prec", "12", "-redo", "-pre",
           os.path.join(workdir, prefix), "-seed", "1"] + list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])
    return {"treefile": open(os.path.join(workdir, prefix + ".treefile")).read().strip()}


def model_arrays(model, alpha, ncat, pinv=0.0):
    """Category rates and proportions as IQ-TREE forms them for +G (and +I+G)."""
    r = orc.gamma_rates(alpha, ncat)
    if pinv > 0:
        r = r * (ncat / (1.0 - pinv)) / r.sum()
        props = np.full(ncat, (1.0 - pinv) / ncat)
    else:
        props = np.full(ncat, 1.0 / ncat)
    return r, props


def make_case(binary, name, tree, model, aln, workdir, safe=False, pinv=0.0, protein=False):
    names = [f"T{i}" for i in range(tree.ntaxa)]
    cols = synth.expand_patterns(aln)
    fa = os.path.join(workdir, name + ".fa")
    write_fasta(fa, cols, model.nstates, names)
    nwk = os.path.join(workdir, name + ".nwk")
    open(nwk, "w").write(tree.newick(names))
    alpha = model.gamma_shape
    ncat = model.ncat
    if protein:
        pf = os.path.join(workdir, name + ".paml")
        paml_file(pf, model)
        mstr = f"{pf}+G{ncat}{{{alpha:.17g}}}"
    else:
        ex = model.exch_upper / model.exch_upper[5]
        mstr = ("GTR{" + ",".join(f"{x:.17g}" for x in ex[:5]) + "}+F{" +
                ",".join(f"{x:.17g}" for x in model.freq) + "}")
        if pinv > 0:
            mstr += f"+I{{{pinv:.17g}}}"
        mstr += f"+G{ncat}{{{alpha:.17g}}}"
    extra = ["-safe"] if safe else []
    fixed = run_iqtree(binary, fa, nwk, mstr, workdir, name + "_fix", ["-blfix", "-wsl"] + extra)
    opt = run_iqtree(binary, fa, nwk, mstr, workdir, name + "_opt", extra)
    keys = tree_splits(tree, names)
    nd, ed = parse_newick(opt["treefile"])
    canon = splits_to_lengths(nd, ed, names)
    opt_len = np.array([canon[k] for k in keys])
    # per-site -> per-pattern (sites were written in pattern order)
    reps = aln.weights.astype(np.int64)
    first = np.concatenate([[0], np.cumsum(reps)[:-1]])
    site = fixed.get("site_lnl")
    ptn_lnl = site[first] if site is not None else np.zeros(aln.npat)
    rates, props = model_arrays(model, alpha, ncat, pinv)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        nstates=model.nstates, ntaxa=tree.ntaxa, eu=tree.eu, ev=tree.ev, length=tree.length,
        exch_upper=model.exch_upper, freq=model.freq, alpha=alpha, ncat=ncat, p_invar=pinv,
        rates=rates, props=props, patterns=aln.patterns, weights=aln.weights,
        const_char=aln.const_char(), safe=int(safe),
        ref_lnl_fixed=fixed["lnl"], ref_rates=np.array(fixed["rates"]),
        ref_pattern_lnl_6sig=ptn_lnl, ref_lnl_opt=opt["lnl"], ref_len_opt=opt_len,
        model_string=mstr)
    print(f"{name}: npat={aln.npat} lnl_fixed={fixed['lnl']!r} lnl_opt={opt['lnl']!r}")


def read_fasta(path):
    names, seqs = [], []
    for line in open(path):
        line = line.strip()
        if line.startswith(">"):
            names.append(line[1:].split()[0])
            seqs.append([])
        elif line:
            seqs[-1].append(line)
    return names, ["".join(s).upper() for s in seqs]


def turtle_case(binary, ref, workdir):
    """The reference's own test data: turtle.fa with the first tree of turtle.trees."""
    td = os.path.join(ref, "test_scripts", "test_data")
    names, seqs = read_fasta(os.path.join(td, "turtle.fa"))
    code = {c: i for i, c in enumerate(DNA)}
    for bm, c in IUPAC.items():
        if bm not in (1, 2, 4, 8):
            code[c] = bm + 3
    for c in "-N?":
        code[c] = 18
    cols = np.array([[code[c] for c in s] for s in seqs], np.uint8)
    nwk = open(os.path.join(td, "turtle.trees")).read().split(";")[0] + ";"
    nd, ed = parse_newick(nwk)
    # renumber: leaves 0..ntaxa-1 in FASTA order, internal nodes after
    leaf_idx = {nm: i for i, nm in enumerate(names)}
    ntaxa = len(names)
    mp, nxt = {}, ntaxa
    for i, nm in enumerate(nd):
        if nm is not None:
            mp[i] = leaf_idx[nm]
        else:
            mp[i] = nxt
            nxt += 1
    # root of the parse may have degree 3 (unrooted) -- keep it as an internal node
    eu = np.array([mp[p] for p, c, ln in ed], np.int32)
    ev = np.array([mp[c] for p, c, ln in ed], np.int32)
    ln = np.array([max(l, 1e-6) for p, c, l in ed])
    tree = synth.Tree(ntaxa, eu, ev, ln)
    freq = np.array([0.3, 0.2, 0.2, 0.3])
    exch = np.array([1.0, 2.0, 1.0, 1.0, 2.0, 1.0])
    model = synth.Model(4, exch, freq, orc.gamma_rates(0.5, 4), np.full(4, 0.25),
                        gamma_shape=0.5)
    aln = synth.compress(cols, 4)
    # run the program on the original files (names as in the reference data)
    mstr = "GTR{1,2,1,1,2}+F{0.3,0.2,0.2,0.3}+G4{0.5}"
    tree_path = os.path.join(workdir, "turtle.nwk")
    with open(tree_path, "w") as f:
        f.write(nwk)
    fixed = run_iqtree(binary, os.path.join(td, "turtle.fa"), tree_path, mstr, workdir,
                       "turtle_fix", ["-blfix"])
    np.savez_compressed(
        os.path.join(HERE, "turtle_ref.npz"),
        nstates=4, ntaxa=ntaxa, eu=tree.eu, ev=tree.ev, length=tree.length,
        exch_upper=exch, freq=freq, alpha=0.5, ncat=4, p_invar=0.0,
        rates=model.rates, props=model.props, patterns=aln.patterns, weights=aln.weights,
        const_char=aln.const_char(), safe=0, ref_lnl_fixed=fixed["lnl"],
        ref_rates=np.array(fixed["rates"]), model_string=mstr)
    print(f"turtle_ref: npat={aln.npat} lnl_fixed={fixed['lnl']!r}")


CASES = ("dna16_g4", "dna24_gaps_amb", "dna160_deep", "dna12_inv_g4", "prot12_g4", "turtle_ref",
         "codon12_g4", "ingest")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("IQTREE_SOURCE"),
                    help="IQ-TREE source tree holding test_scripts/ (or set IQTREE_SOURCE)")
    ap.add_argument("--only", nargs="*", choices=CASES, default=list(CASES),
                    help="regenerate only these cases")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set IQTREE_SOURCE")
    binary = os.path.join(args.ref, "test_scripts", "iqtree2", "Linux-intel", "iqtree2")
    only = set(args.only)
    with tempfile.TemporaryDirectory() as wd:
        if "dna16_g4" in only:
            # DNA GTR+G4, 16 taxa (the small FP64 configuration, 2,000 sites)
            rng = np.random.default_rng(101)
            m = synth.dna_gtr(rng, 4, 0.5)
            m = synth.Model(4, m.exch_upper, m.freq, orc.gamma_rates(0.5, 4), np.full(4, 0.25),
                            gamma_shape=0.5)
            t = synth.random_tree(16, 0.1, 111)
            a = synth.simulate(t, m, 2000, 123)
            make_case(binary, "dna16_g4", t, m, a, wd)
            make_case(binary, "dna16_g4_safe", t, m, a, wd, safe=True)
        if "dna24_gaps_amb" in only:
            # gaps and IUPAC ambiguity codes, 24 taxa
            rng = np.random.default_rng(202)
            m = synth.dna_gtr(rng, 4, 0.7)
            m = synth.Model(4, m.exch_upper, m.freq, orc.gamma_rates(0.7, 4), np.full(4, 0.25),
                            gamma_shape=0.7)
            t = synth.random_tree(24, 0.08, 211)
            a = synth.simulate(t, m, 1500, 223, gap_frac=0.05)
            cols = synth.expand_patterns(a)
            amb = np.random.default_rng(5).random(cols.shape) < 0.03
            cols[amb] = np.random.default_rng(6).integers(4, 18, amb.sum())
            cols[:, 0] = 18  # an all-gap column
            a = synth.compress(cols, 4)
            make_case(binary, "dna24_gaps_amb", t, m, a, wd)
        if "dna160_deep" in only:
            # deep tree: underflow scaling events (NORM and SAFE)
            rng = np.random.default_rng(303)
            m = synth.dna_gtr(rng, 4, 0.5)
            m = synth.Model(4, m.exch_upper, m.freq, orc.gamma_rates(0.5, 4), np.full(4, 0.25),
                            gamma_shape=0.5)
            t = synth.random_tree(160, 0.3, 311)
            a = synth.simulate(t, m, 400, 323)
            make_case(binary, "dna160_deep", t, m, a, wd)
            make_case(binary, "dna160_deep_safe", t, m, a, wd, safe=True)
        if "dna12_inv_g4" in only:
            # +I+G4 (invariant sites)
            rng = np.random.default_rng(404)
            m = synth.dna_gtr(rng, 4, 0.6)
            t = synth.random_tree(12, 0.1, 411)
            a = synth.simulate(t, m, 1200, 423)
            make_case(binary, "dna12_inv_g4", t, m, a, wd, pinv=0.25)
        if "prot12_g4" in only:
            # 20-state protein +G4 with a user exchangeability matrix (PAML format)
            rng = np.random.default_rng(505)
            m = synth.protein(rng, 4, 0.8)
            m = synth.Model(20, m.exch_upper, m.freq, orc.gamma_rates(0.8, 4), np.full(4, 0.25),
                            gamma_shape=0.8)
            t = synth.random_tree(12, 0.15, 511)
            a = synth.simulate(t, m, 800, 523)
            make_case(binary, "prot12_g4", t, m, a, wd, protein=True)
        if "turtle_ref" in only:
            turtle_case(binary, args.ref, wd)
        if "codon12_g4" in only:
            codon_case(binary, wd)
        if "ingest" in only:
            os.makedirs(os.path.join(HERE, "ingest"), exist_ok=True)
            ingest_case(binary, args.ref, wd, "turtle.fa", 4, 701)
            ingest_case(binary, args.ref, wd, "turtle_aa.fasta", 20, 702)
            ingest_case(binary, args.ref, wd, "example.phy", 4, 703)


if __name__ == "__main__":
    main()
