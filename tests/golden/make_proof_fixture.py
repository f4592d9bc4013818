"""Writes tests/golden/proof_k10.json: one proof of the config-3 circuit at
k = 10 made by this library on a GPU (transcript on), with what a verifier
needs beside it: the verifying key (fixed and permutation commitments, the
transcript scalar), the public inputs and the synthetic SRS's trapdoor (from
which [s]_2 = tau [1]_2).  The CPU test suite verifies the proof from these
bytes with the pairing check and rejects changed copies of it
(tests/test_proof_fixture.py).

Run on a machine with a CUDA device:  python tests/golden/make_proof_fixture.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import load_package  # noqa: E402

K, SRS_SEED, PROOF_SEED = 10, 11, 21


def main():
    import importlib
    import torch
    h2b = load_package()
    P = importlib.import_module(h2b.__name__ + ".prover")
    V = importlib.import_module(h2b.__name__ + ".verify")
    res = P.Resident(h2b, SRS_SEED)
    vk = res.verifying_key(K)
    st = torch.cuda.Stream()
    w = P.ProofWorkload(res, K, PROOF_SEED, transcript=True)
    w.run(st)
    st.synchronize()
    assert V.verify_proof(vk, w.public, w.proof, res.verifier_params())
    pt = lambda p: None if p is None else [hex(p[0]), hex(p[1])]  # noqa: E731
    out = {
        "k": K, "srs_seed": SRS_SEED, "proof_seed": PROOF_SEED, "tau": hex(res.tau),
        "fixed_commitments": [pt(p) for p in vk.fixed_commitments],
        "permutation_commitments": [pt(p) for p in vk.permutation_commitments],
        "transcript_repr": hex(vk.transcript_repr),
        "public": [hex(v) for v in w.public],
        "proof": w.proof.hex(),
    }
    with open(os.path.join(HERE, "proof_k10.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
