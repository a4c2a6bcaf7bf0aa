"""computePartialLikelihood in packets, from a C++ caller.

tests/cpp/packet_driver.cpp is compiled with g++ against include/gems_b200.h and linked to
libgems_b200.so.  It splits the patterns into packets as the reference's computeBounds does and
calls gems_compute_partial for every (packet, traversal entry), as the reference's
computeTraversalInfo loop does (tree/phylokernelnew.h:1274-1281); a second session runs the
whole op list with gems_traverse.  Every slot (partials and scale counters) and the branch lnL
must be identical, bit for bit, for every kernel family: 4- and 20-state CUDA-core forms,
the tcgen05 20- and 61-state forms, the FP64 61-state GEMM forms (NORM and SAFE)."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from gems_b200 import GemsError, Session, synth
from gems_b200.api import PREC, SCALING, full_traversal, op_array

pytestmark = pytest.mark.gpu

CASES = [  # (states, categories, precision, scaling)
    (4, 4, "fp64", "norm"),
    (4, 4, "fp64", "safe"),
    (4, 4, "mixed", "norm"),
    (20, 4, "fp64", "norm"),
    (20, 4, "mixed", "norm"),
    (61, 4, "fp64", "safe"),
    (61, 4, "fp64", "norm"),
    (61, 4, "mixed", "safe"),
]
IDS = [f"n{n}-c{c}-{p}-{s}" for n, c, p, s in CASES]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("cpp") / "packet_driver")
    lib = os.path.join(ROOT, "gems_b200")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "packet_driver.cpp"), "-L" + lib,
                    "-lgems_b200", "-Wl,-rpath," + lib, "-o", out], check=True)
    return out


def _case(n, ncat, seed):
    rng = np.random.default_rng(seed)
    model = {4: lambda: synth.dna_gtr(rng, ncat, 0.5), 20: lambda: synth.protein(rng, ncat, 0.8),
             61: lambda: synth.codon_gy(rng, ncat, 0.6)}[n]()
    tree = synth.random_tree(24, 0.15, seed + 1)
    aln = synth.simulate(tree, model, {4: 5000, 20: 3000, 61: 1500}[n], seed + 2, gap_frac=0.03)
    return tree, model, aln


def _write_input(path, tree, model, aln, precision, scaling):
    ops, br = full_traversal(tree)
    arr, nops = op_array(ops)
    hdr = np.array([tree.ntaxa, aln.npat, model.nstates, model.ncat, tree.ntaxa - 2,
                    PREC[precision], SCALING[scaling], nops], np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(aln.patterns, np.uint8).tobytes())
        for a in (aln.weights, model.eval, model.evec, model.inv_evec, model.rates, model.props):
            f.write(np.ascontiguousarray(a, np.float64).tobytes())
        f.write(bytes(arr)[: nops * ctypes.sizeof(arr[0])])
        f.write(bytes(br))


@pytest.mark.parametrize("n,ncat,precision,scaling", CASES, ids=IDS)
@pytest.mark.parametrize("threads", [3, 8])
def test_packets_from_cpp_match_whole_traversal(gpu, driver, tmp_path, n, ncat, precision,
                                                scaling, threads):
    tree, model, aln = _case(n, ncat, 40 + n)
    inp = str(tmp_path / "input.bin")
    _write_input(inp, tree, model, aln, precision, scaling)
    r = subprocess.run([driver, inp, str(threads)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr


def test_misaligned_or_out_of_range_packet_refused(gpu):
    tree, model, aln = _case(61, 4, 7)
    s = Session(tree.ntaxa, aln.npat, 61, 4, tree.ntaxa - 2, "mixed", "safe")
    s.upload_tips(aln.patterns)
    s.upload_patterns(aln.weights)
    s.set_model(model.eval, model.evec, model.inv_evec, model.rates, model.props)
    assert s.pattern_granule() == 128
    ops, _ = full_traversal(tree)
    for lo, hi in ((64, 256), (0, 100), (0, aln.npat + 1), (128, 128), (-128, 128)):
        with pytest.raises(GemsError) as e:
            s.compute_partial(ops[0], lo, hi)
        assert e.value.status == 5
    s.compute_partial(ops[0], 0, 128)
    s.compute_partial(ops[0], 128, aln.npat)
    s.close()
