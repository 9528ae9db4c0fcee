"""Digest of the oracle's proof of the mixed-size lookup workload.

The workload: 40 plonk-like modules whose log2 row counts are drawn
uniformly from 10..20 with seed 0xC4 (loom_b200.plonk.mixed_sizes), each
with a copy constraint and a range lookup into a shared 2^8 table
(arguments.Range, arguments/lookup.go:31-46), proved with 200 FRI queries
(prover/prover.go:655-719).  The proof is several tens of MB, so the
fixture keeps its length and SHA-256 only; tests/test_gpu_parity.py proves
the same program on the GPU, batched and plain, and compares.

The oracle (oracle/, CPU) takes minutes on a few cores.  Run:
    python tests/golden/make_c4_digest.py
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEED = 0xC4
MODULES, LOG_MIN, LOG_MAX = 40, 10, 20
QUERIES = 200
OUT = os.path.join(HERE, "c4_mixed_lookup_digest.json")


def main():
    import oracle
    from loom_b200 import field as F, plonk
    sizes = plonk.mixed_sizes(MODULES, LOG_MIN, LOG_MAX, SEED)
    compiled, wit = plonk.build_mixed(sizes, seed=SEED)
    mont = [F.to_mont(w) for w in wit]
    t = time.time()
    proof = oracle.prove(compiled.words, mont, QUERIES)
    secs = time.time() - t
    oracle.verify(compiled.words, proof, QUERIES, compiled.logup_buses)
    rec = {"workload": "plonk.build_mixed(plonk.mixed_sizes(40, 10, 20, 0xC4), seed=0xC4)",
           "seed": SEED, "log_sizes": sizes, "rows": int(sum(1 << s for s in sizes)), "queries": QUERIES,
           "program_sha256": hashlib.sha256(compiled.words.astype("<u4").tobytes()).hexdigest(),
           "proof_len": len(proof), "proof_sha256": hashlib.sha256(proof).hexdigest(),
           "oracle_seconds": round(secs, 1), "oracle_threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))}
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
