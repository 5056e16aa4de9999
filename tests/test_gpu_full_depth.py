"""Full-depth parity on the benchmark circuits, against digests of the unmodified reference engine.

The final stores are too large to commit (up to ~4.4e7 terms), so each fixture
(``tests/golden/full_<name>.npz``, written by ``tests/golden/make_golden.py --full-depth``) keeps a
bucketed digest of the reference's raw export: the SHA-256 of the sorted key set (compared bit-exactly),
per-bucket term counts, sums of |c| and two pseudo-random projections of the coefficients (each within
1e-10 of its bucket's sum |c|, which holds when every coefficient agrees to 1e-10 relative), the 4096
largest coefficients term by term (1e-10 relative), and <0|O|0> (1e-10 relative).

* the 100-qubit kicked Ising circuit (5600 gates, Pauli weight <= 10, lower_atol 1e-5): ~3.1e7 terms;
* the 6x6 spinful Hubbard circuit (2208 gates, Majorana length <= 8, lower_atol 1e-5);
* two instances of the batched 50-qubit workload, depths 24 and 12 (Pauli weight <= 8), through a plain
  engine and, for the depth-12 one, through the batch runner with an export per instance;
* the 20-qubit line circuit (390 gates) in the Schrodinger picture with schrodinger_cutoff 4: the
  evolved state's ~6.4e7 paired monomials.
"""

import numpy as np
import pytest

from monoprop_b200 import _native
from monoprop_b200.batch import BatchConfig, run_batch
from oracle import golden

pytestmark = pytest.mark.gpu


def _run(wl):
    eng = _native.engine_for(wl)
    try:
        eng.propagate(wl.gen_words(), wl.angles())
        keys, coefs = eng.export()
        ev = eng.expectation()
    finally:
        eng.close()
    return keys, coefs, ev


@pytest.mark.parametrize("name", sorted(golden.FULL_DEPTH))
def test_full_depth_matches_reference_digest(name):
    g = golden.load("full_" + name)
    wl = golden.FULL_DEPTH[name]()
    assert wl.n_layers == int(g["n_layers"])
    keys, coefs, ev = _run(wl)
    bitwise = golden.check_digest(g, keys, coefs, ev)
    print(f"{name}: {keys.shape[0]} terms, <O> = {ev!r}, coefficients bit-identical to the reference: {bitwise}")


def test_batch_instance_full_depth_matches_reference_digest():
    g = golden.load("full_ising50_b12")
    wl = golden.FULL_DEPTH["ising50_b12"]()
    cap = int(g["n"]) + 16
    r = run_batch([wl], BatchConfig(workers=1), export_caps=[cap])
    keys, coefs = r.exports[0]
    assert int(r.final_terms[0]) == int(g["n"])
    golden.check_digest(g, keys, coefs, float(r.expectations[0]))
