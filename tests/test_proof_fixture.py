"""A proof made by this library on a GPU (tests/golden/proof_k10.json, from
tests/golden/make_proof_fixture.py) verifies on the host from its bytes:
transcript replay, the vanishing argument at x and the SHPLONK opening
ending in the pairing check e(W', [s]_2) e(F + u W', -[1]_2) == 1
(poly/kzg/msm.rs:159-176 in the reference).  Changed copies fail: one
evaluation, one commitment, W', a public input, the G2 element [s]_2, or a
truncated proof."""
import importlib
import json
import os

import pytest

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "proof_k10.json")


@pytest.fixture(scope="module")
def fx(h2b):
    if not os.path.exists(FIXTURE):
        pytest.skip("proof fixture not generated (tests/golden/make_proof_fixture.py needs a GPU)")
    d = json.load(open(FIXTURE))
    V = importlib.import_module(h2b.__name__ + ".verify")
    T = importlib.import_module(h2b.__name__ + ".transcript")
    pt = lambda p: None if p is None else (int(p[0], 16), int(p[1], 16))  # noqa: E731
    vk = V.VerifyingKey(d["k"], [pt(p) for p in d["fixed_commitments"]],
                        [pt(p) for p in d["permutation_commitments"]], int(d["transcript_repr"], 16))
    return V, T, vk, [int(v, 16) for v in d["public"]], bytes.fromhex(d["proof"]), int(d["tau"], 16)


def test_gpu_proof_verifies_on_the_host(fx):
    V, _, vk, public, proof, tau = fx
    assert len(proof) == 1248
    assert V.verify_proof(vk, public, proof, V.params_from_tau(tau))


def test_changed_proofs_fail(h2b, fx):
    V, T, vk, public, proof, tau = fx
    F = h2b.fields
    params = V.params_from_tau(tau)
    bad = bytearray(proof)
    bad[32 * 13 + 64] ^= 1                                     # an advice evaluation
    assert not V.verify_proof(vk, public, bytes(bad), params)
    bad = bytearray(proof)
    bad[32:64] = T.compress(F.G1_GENERATOR)                    # advice commitment 1
    assert not V.verify_proof(vk, public, bytes(bad), params)
    bad = bytearray(proof)
    bad[-32:] = T.compress(F.G1_GENERATOR)                     # W'
    assert not V.verify_proof(vk, public, bytes(bad), params)
    assert not V.verify_proof(vk, [public[0] + 1] + public[1:], proof, params)
    assert not V.verify_proof(vk, public, proof, V.params_from_tau(tau + 1))
    assert not V.verify_proof(vk, public, proof[:-32], params)
