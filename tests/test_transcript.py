"""Fiat-Shamir transcript and proof wire format (halo2's Blake2bWrite /
Blake2bRead with Challenge255, restated in halo2-gpu_b200/transcript.py).
No reference output pins these bytes (the crates are absent); the tests check
the construction against independent restatements with hashlib and Python
integers, the point encoding against the curve, and that a reader replays a
writer's proof to the same challenges."""
import hashlib
import importlib

import pytest


@pytest.fixture()
def T(h2b):
    return importlib.import_module(h2b.__name__ + ".transcript")


def _points(F, count):
    pts, P = [], F.G1_GENERATOR
    for i in range(count):
        pts.append(P)
        P = F.g1_add(F.g1_mul(P, 0x1F3D5B79 + i), F.G1_GENERATOR)
    return pts


def test_compress_round_trip_and_flags(h2b, T):
    F = h2b.fields
    for pt in _points(F, 12):
        b = T.compress(pt)
        assert len(b) == 32 and T.decompress(b) == pt
        assert bool(b[31] & 0x80) == bool(pt[1] & 1)
        neg = (pt[0], F.Q_MOD - pt[1])
        assert T.decompress(T.compress(neg)) == neg and T.compress(neg) != b
    g = T.compress(F.G1_GENERATOR)
    assert g == (1).to_bytes(32, "little")              # y = 2 is even: no sign bit
    inf = T.compress(None)
    assert inf == bytes(31) + b"\x40" and T.decompress(inf) is None


def test_decompress_rejects_bad_encodings(h2b, T):
    F = h2b.fields
    with pytest.raises(T.TranscriptError):
        T.decompress(F.Q_MOD.to_bytes(32, "little"))     # x not canonical
    x = next(x for x in range(2, 100) if pow((x ** 3 + 3) % F.Q_MOD, (F.Q_MOD - 1) // 2, F.Q_MOD) != 1)
    with pytest.raises(T.TranscriptError):
        T.decompress(x.to_bytes(32, "little"))            # not on the curve
    with pytest.raises(T.TranscriptError):
        T.decompress(bytes(31) + b"\xc0")                 # infinity with a sign bit
    with pytest.raises(T.TranscriptError):
        T.decompress((5).to_bytes(32, "little")[:31] + b"\x40")
    with pytest.raises(T.TranscriptError):
        T.decompress(bytes(31))


def test_challenges_follow_the_blake2b_construction(h2b, T):
    F = h2b.fields
    pt, s = _points(F, 1)[0], 0x1234567890ABCDEF
    w = T.Blake2bWrite()
    w.write_point(pt)
    w.write_scalar(s)
    c1 = w.squeeze_challenge()
    c2 = w.squeeze_challenge()
    ref = hashlib.blake2b(digest_size=64, person=b"Halo2-Transcript")
    ref.update(b"\x01" + pt[0].to_bytes(32, "little") + pt[1].to_bytes(32, "little"))
    ref.update(b"\x02" + s.to_bytes(32, "little"))
    ref.update(b"\x00")
    assert c1 == int.from_bytes(ref.copy().digest(), "little") % F.R_MOD
    ref.update(b"\x00")                                   # the running state continues
    assert c2 == int.from_bytes(ref.copy().digest(), "little") % F.R_MOD
    assert w.finalize() == T.compress(pt) + s.to_bytes(32, "little")


def test_reader_replays_writer(h2b, T):
    F = h2b.fields
    pts = _points(F, 5)
    scal = [3, F.R_MOD - 1, 0, 1 << 200]
    w = T.Blake2bWrite()
    w.common_scalar(77)
    got = []
    for i, p in enumerate(pts):
        w.write_point(p)
        if i % 2:
            got.append(w.squeeze_challenge())
    for s in scal:
        w.write_scalar(s)
    got.append(w.squeeze_challenge())
    proof = w.finalize()
    assert len(proof) == 32 * (len(pts) + len(scal))
    r = T.Blake2bRead(proof)
    r.common_scalar(77)
    again = []
    for i, p in enumerate(pts):
        assert r.read_point() == p
        if i % 2:
            again.append(r.squeeze_challenge())
    assert [r.read_scalar() for _ in scal] == scal
    again.append(r.squeeze_challenge())
    assert again == got and r.remaining() == 0
    # a changed byte changes what the reader absorbs, so the challenges differ
    bad = bytearray(proof)
    bad[32 * len(pts) + 3] ^= 1
    r2 = T.Blake2bRead(bytes(bad))
    r2.common_scalar(77)
    for i in range(len(pts)):
        r2.read_point()
        if i % 2:
            r2.squeeze_challenge()
    [r2.read_scalar() for _ in scal]
    assert r2.squeeze_challenge() != got[-1]


def test_transcript_rejects_infinity_and_non_canonical(h2b, T):
    F = h2b.fields
    w = T.Blake2bWrite()
    with pytest.raises(T.TranscriptError):
        w.write_point(None)
    with pytest.raises(T.TranscriptError):
        w.write_scalar(F.R_MOD)
    r = T.Blake2bRead(F.R_MOD.to_bytes(32, "little"))
    with pytest.raises(T.TranscriptError):
        r.read_scalar()
    with pytest.raises(T.TranscriptError):
        T.Blake2bRead(b"\x00" * 10).read_scalar()


def test_commitment_image_to_affine(h2b, T):
    import numpy as np
    F = h2b.fields
    pt = _points(F, 2)[1]
    img = np.concatenate([F.fq_mont_limbs([pt[0]]), F.fq_mont_limbs([pt[1]]), F.fq_mont_limbs([1])], axis=1)
    assert T.commitment_to_affine(img.reshape(-1)) == pt
    inf = np.concatenate([F.fq_mont_limbs([0]), F.fq_mont_limbs([1]), F.fq_mont_limbs([0])], axis=1)
    assert T.commitment_to_affine(inf.reshape(-1)) is None
