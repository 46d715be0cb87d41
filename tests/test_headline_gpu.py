"""GPU parity on the full-size timed workloads, against digests of the reference's own results
(tests/golden/headline_digests.json, written by tests/golden/make_headline_digests.py from the reference
compiled from its sources):

* the batched comparison, 4096 pairs of lengths log-uniform in [256, 65536]: every braid of the batched
  persistent launch (tuned band heights, and every band forced to 1024 rows) and of the per-pair launches
  against OpenMPIterativeCombing<int,false>(1) (R:include/SemiLocal/SemiLocalLCS.h:231-306);
* the 2^20 single pair: wavefront and hybrid braids against OpenMPHybridIterative<int,false>
  (R:include/SemiLocal/SemiLocalLCS.h:594-794), semi-local scores read from the GPU braid, and the
  bit-parallel score against nary::llcs_nary_symbol_smart_combing<uint64_t>
  (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736) on the reference routine's domain.

Bar: bit-exact (sha256 of every int32 braid)."""
import hashlib
import json
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
DIGESTS = os.path.join(os.path.dirname(__file__), "golden", "headline_digests.json")


def _digest(r2c) -> str:
    return hashlib.sha256(np.ascontiguousarray(r2c, dtype="<i4").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def digests():
    with open(DIGESTS) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def batch():
    return gen.batch_pairs(4096, 256, 65536, seed=5)


@pytest.fixture(scope="module")
def pair_2p20():
    return gen.hybrid_pair(1 << 20, seed=4)


def _check_batch(res, sc, ref):
    got = [_digest(r) for r in res]
    bad = [i for i, d in enumerate(got) if d[:16] != ref["pair_sha256_16"][i]]
    assert not bad, f"{len(bad)} braids differ from the reference, first pairs {bad[:8]}"
    h = hashlib.sha256()
    for d in got:
        h.update(bytes.fromhex(d))
    assert h.hexdigest() == ref["batch_sha256"]
    assert np.array_equal(np.asarray(sc), np.asarray(ref["global_scores"]))


@pytest.mark.parametrize("mode,band_rows", [(0, 0), (0, 1024), (1, 0)],
                         ids=["batched-tuned", "batched-bands1024", "per-pair-tuned"])
def test_batch_4096_vs_reference(engine, digests, batch, mode, band_rows):
    """The whole timed batch; band heights from the tuner as in the benchmark (band_rows 0), or forced to 1024
    rows, which pads the last band of most pairs."""
    engine.autotune(cache=os.environ.get("SLCS_TUNING_CACHE") or None)
    ref = digests["batch_4096"]
    assert sum(len(a) * len(b) for a, b in batch) == ref["cells"]
    res, sc = engine.batch_comb(batch, mode=mode, band_rows=band_rows)
    _check_batch(res, sc, ref)


@pytest.mark.parametrize("algo", ["wavefront", "hybrid", "hybrid_65536", "auto"])
def test_pair_2p20_vs_reference(engine, digests, pair_2p20, algo):
    a, b = pair_2p20
    ref = digests["hybrid_2p20"]
    assert (len(a), len(b)) == (ref["m"], ref["n"])
    if algo == "hybrid":
        r2c, score = engine.comb(a, b, algo=engine.ALGO_HYBRID, tile=4096)
    elif algo == "hybrid_65536":
        r2c, score = engine.comb(a, b, algo=engine.ALGO_HYBRID, tile=65536)
    elif algo == "auto":
        r2c, score = engine.comb(a, b)
    else:
        r2c, score = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
    assert _digest(r2c) == ref["sha256"]
    assert score == ref["global_score"]
    q = engine.scores(r2c, len(a), len(b), [(k, i, j) for k, i, j, _ in ref["queries"]])
    assert [int(x) for x in q] == [v for *_, v in ref["queries"]]


def test_bit_2p20_vs_reference(engine, digests, pair_2p20):
    a, b = pair_2p20
    ref = digests["bit_2p20"]
    la, lb = (len(a) // 32) * 32, (len(b) // 32) * 32
    ta, tb = a[:la], b[:lb]
    if not ref["a_is_first"]:
        ta, tb = tb, ta
    assert (len(ta), len(tb)) == (ref["len_a"], ref["len_b"])
    assert engine.bitcomb_llcs(ta, tb) == ref["llcs"]
    assert engine.hyyro_llcs(ta, tb) == ref["llcs"]
    # the untrimmed pair (outside the reference routine's domain) against the reference braid's score
    assert engine.bitcomb_llcs(a, b) == digests["hybrid_2p20"]["global_score"]
    assert engine.hyyro_llcs(a, b) == digests["hybrid_2p20"]["global_score"]
