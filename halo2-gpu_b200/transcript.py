"""Fiat-Shamir transcript and proof wire format of the prover (host side).

The reference proves with halo2's `Blake2bWrite<_, G1Affine, Challenge255>`
and verifies with `Blake2bRead` (halo2-axiom @ 5e4f0e5,
`halo2_proofs/src/transcript.rs`, a dependency absent from the reference
tree; its call sites are `halo2_proofs/src/plonk/prover.rs:56-482` and the
tests' `Blake2bWrite::<_, G1Affine, Challenge255<_>>::init(vec![])`, e.g.
`halo2_proofs/tests/phase5_prove_verify_lookup_permutation.rs:258-283`).
This module restates that transcript's published construction:

* the state is one BLAKE2b hash with a 64-byte digest and the 16-byte
  personalisation "Halo2-Transcript";
* a point is absorbed as the byte 1 followed by its affine x and y, each the
  32-byte little-endian canonical integer (the point at infinity cannot be
  absorbed); a scalar as the byte 2 followed by its 32-byte little-endian
  canonical value;
* a challenge absorbs the byte 0, then finalises a COPY of the state (the
  running state continues) and maps the 64-byte digest, read as a
  little-endian 512-bit integer, to Fr by reduction mod r (Challenge255,
  `from_uniform_bytes`);
* `write_point` / `write_scalar` absorb and append the wire form to the
  proof: a scalar as its 32-byte little-endian canonical value, a G1 point
  compressed to 32 bytes (x little-endian; BN254's p < 2^254 leaves the top
  two bits of the last byte free, and they carry the sign of y (0x80: y odd)
  and the point at infinity (0x40, every other bit zero)).

Parity is unpinned: the BLAKE2b hash itself is the standard one
(`hashlib.blake2b`), but halo2-axiom and halo2curves-axiom are not vendored
and no Rust toolchain exists here, so the byte layout above is a
restatement that no reference output has checked.
"""
import hashlib

from . import fields as F

PREFIX_CHALLENGE, PREFIX_POINT, PREFIX_SCALAR = 0, 1, 2
PERSONAL = b"Halo2-Transcript"
SIGN_MASK, IDENTITY_MASK = 0x80, 0x40
_SQRT_EXP = (F.Q_MOD + 1) // 4          # p = 3 mod 4


class TranscriptError(ValueError):
    pass


def compress(pt):
    """Affine G1 point (x, y) as plain ints, or None for infinity -> 32 bytes."""
    if pt is None:
        out = bytearray(32)
        out[31] = IDENTITY_MASK
        return bytes(out)
    x, y = pt
    out = bytearray(x.to_bytes(32, "little"))
    if y & 1:
        out[31] |= SIGN_MASK
    return bytes(out)


def decompress(b):
    """32 bytes -> (x, y) or None; raises TranscriptError when the bytes are
    not the encoding of a point on y^2 = x^3 + 3."""
    if len(b) != 32:
        raise TranscriptError("compressed point must be 32 bytes")
    flags = b[31] & (SIGN_MASK | IDENTITY_MASK)
    raw = bytearray(b)
    raw[31] &= 0x3F
    x = int.from_bytes(raw, "little")
    if flags & IDENTITY_MASK:
        if x != 0 or flags & SIGN_MASK:
            raise TranscriptError("malformed encoding of the point at infinity")
        return None
    if x >= F.Q_MOD:
        raise TranscriptError("x is not canonical")
    rhs = (x * x * x + 3) % F.Q_MOD
    y = pow(rhs, _SQRT_EXP, F.Q_MOD)
    if y * y % F.Q_MOD != rhs:
        raise TranscriptError("x is not on the curve")
    if (y & 1) != bool(flags & SIGN_MASK):
        y = F.Q_MOD - y
    if y == 0 and flags & SIGN_MASK:
        raise TranscriptError("sign bit set for y = 0")
    return (x, y)


def commitment_to_affine(jac96):
    """The library's 96-byte MSM result (Jacobian image {X, Y, Z}, Montgomery
    Fq limbs) as a plain affine point, or None for infinity."""
    return F.jac_to_affine_ints(jac96)


class _Base:
    def __init__(self):
        self._state = hashlib.blake2b(digest_size=64, person=PERSONAL)

    def common_point(self, pt):
        if pt is None:
            raise TranscriptError("cannot write points at infinity to the transcript")
        x, y = pt
        self._state.update(bytes([PREFIX_POINT]) + x.to_bytes(32, "little") + y.to_bytes(32, "little"))

    def common_scalar(self, s):
        if not 0 <= s < F.R_MOD:
            raise TranscriptError("scalar is not canonical")
        self._state.update(bytes([PREFIX_SCALAR]) + s.to_bytes(32, "little"))

    def squeeze_challenge(self):
        self._state.update(bytes([PREFIX_CHALLENGE]))
        return int.from_bytes(self._state.copy().digest(), "little") % F.R_MOD


class Blake2bWrite(_Base):
    """Prover side: absorbs what it writes and accumulates the proof bytes."""

    def __init__(self):
        super().__init__()
        self._proof = bytearray()

    def write_point(self, pt):
        self.common_point(pt)
        self._proof += compress(pt)

    def write_scalar(self, s):
        self.common_scalar(s)
        self._proof += s.to_bytes(32, "little")

    def finalize(self):
        return bytes(self._proof)


class Blake2bRead(_Base):
    """Verifier side: reads the proof in the order it was written, absorbing
    the same bytes, so its challenges equal the prover's."""

    def __init__(self, proof):
        super().__init__()
        self._proof = memoryview(bytes(proof))
        self._at = 0

    def _take(self, n):
        if self._at + n > len(self._proof):
            raise TranscriptError("proof is too short")
        b = bytes(self._proof[self._at:self._at + n])
        self._at += n
        return b

    def read_point(self):
        pt = decompress(self._take(32))
        self.common_point(pt)
        return pt

    def read_scalar(self):
        s = int.from_bytes(self._take(32), "little")
        if s >= F.R_MOD:
            raise TranscriptError("scalar is not canonical")
        self.common_scalar(s)
        return s

    def remaining(self):
        return len(self._proof) - self._at
