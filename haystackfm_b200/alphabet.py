"""IUPAC nucleotide alphabet: host-side encoding, mirroring haystackfm's
`src/alphabet.rs` API (codes, `encode_byte`, `encode_char`, `decode_char`,
`iupac_bases`, `compatible_symbols`, `DnaSequence`, `concatenate_sequences`).

Codes 0..15: $ A C G T N R Y S W K M B D H V (src/alphabet.rs:3-52).
"""
from __future__ import annotations

import numpy as np

from .errors import FmIndexError

ALPHABET_SIZE = 16
SENTINEL, A, C, G, T, N, R, Y, S, W, K, M, B, D, H, V = range(16)

_SYMBOLS = "$ACGTNRYSWKMBDHV"

# 256-entry ASCII -> code table (src/alphabet.rs:54-94); -1 = invalid.  U/u map to T.
ENCODE_LUT = np.full(256, -1, dtype=np.int16)
for _code, _ch in enumerate(_SYMBOLS):
    ENCODE_LUT[ord(_ch)] = _code
    ENCODE_LUT[ord(_ch.lower())] = _code
ENCODE_LUT[ord("$")] = SENTINEL
ENCODE_LUT[ord("U")] = T
ENCODE_LUT[ord("u")] = T

# compatible_symbols (src/alphabet.rs:174-193), same slice order.
IUPAC_COMPAT = (
    (),
    (A, N, R, W, M, D, H, V),
    (C, N, Y, S, M, B, H, V),
    (G, N, R, S, K, B, D, V),
    (T, N, Y, W, K, B, D, H),
    (A, C, G, T, N, R, Y, S, W, K, M, B, D, H, V),
    (A, G, N, R, S, W, K, M, B, D, H, V),
    (C, T, N, Y, S, W, K, M, B, D, H, V),
    (C, G, N, R, Y, S, K, M, B, D, H, V),
    (A, T, N, R, Y, W, K, M, B, D, H, V),
    (G, T, N, R, Y, S, W, K, B, D, H, V),
    (A, C, N, R, Y, S, W, M, B, D, H, V),
    (C, G, T, N, R, Y, S, W, K, M, B, D, H, V),
    (A, G, T, N, R, Y, S, W, K, M, B, D, H, V),
    (A, C, T, N, R, Y, S, W, K, M, B, D, H, V),
    (A, C, G, N, R, Y, S, W, K, M, B, D, H, V),
)
# ExactDna::compatible (src/alphabet.rs:286-294)
EXACT_COMPAT = ((), (A,), (C,), (G,), (T,)) + ((),) * 11

_IUPAC_BASES = {
    A: (A,), C: (C,), G: (G,), T: (T,), N: (A, C, G, T), R: (A, G), Y: (C, T), S: (G, C),
    W: (A, T), K: (G, T), M: (A, C), B: (C, G, T), D: (A, G, T), H: (A, C, T), V: (A, C, G),
}

TAG_IUPAC = 0   # IupacDna (src/alphabet.rs:262-272)
TAG_EXACT = 1   # ExactDna (src/alphabet.rs:282-305)


def encode_byte(b: int):
    v = int(ENCODE_LUT[b & 0xFF])
    return None if v < 0 else v


def encode_char(ch: str):
    if len(ch) != 1 or ord(ch) > 127:
        return None
    return encode_byte(ord(ch))


def decode_char(code: int):
    return _SYMBOLS[code] if 0 <= code < 16 else None


def iupac_bases(code: int):
    return _IUPAC_BASES.get(code, ())


def compatible_symbols(code: int):
    return IUPAC_COMPAT[code] if 0 <= code < 16 else ()


def compat_table(tag: int):
    return EXACT_COMPAT if tag == TAG_EXACT else IUPAC_COMPAT


def encode(s: str) -> np.ndarray:
    """Encode an ASCII IUPAC string to codes (raises on invalid characters)."""
    raw = np.frombuffer(s.encode("ascii"), dtype=np.uint8)
    codes = ENCODE_LUT[raw]
    if (codes < 0).any():
        i = int(np.argmax(codes < 0))
        raise FmIndexError.invalid_character(s[i], i)
    return codes.astype(np.uint8)


class DnaSequence:
    """Encoded DNA sequence plus FASTA header (src/alphabet.rs:310-370)."""

    __slots__ = ("_bases", "_header")

    def __init__(self, bases, header: str = ""):
        self._bases = np.ascontiguousarray(bases, dtype=np.uint8)
        self._header = header

    @classmethod
    def from_str(cls, s: str) -> "DnaSequence":
        if not s:
            raise FmIndexError.empty_sequence()
        codes = encode(s)
        bad = np.nonzero(codes == SENTINEL)[0]
        if len(bad):
            raise FmIndexError.invalid_character(s[int(bad[0])], int(bad[0]))
        return cls(codes)

    @classmethod
    def from_str_with_header(cls, s: str, header: str) -> "DnaSequence":
        seq = cls.from_str(s)
        seq._header = header
        return seq

    @classmethod
    def from_encoded(cls, bases) -> "DnaSequence":
        return cls(bases)

    def __len__(self):
        return len(self._bases)

    def is_empty(self) -> bool:
        return len(self._bases) == 0

    def header(self) -> str:
        return self._header

    def as_slice(self) -> np.ndarray:
        return self._bases

    def __eq__(self, other):
        return isinstance(other, DnaSequence) and self._header == other._header and \
            np.array_equal(self._bases, other._bases)


def concatenate_sequences(sequences):
    """s1 $ s2 $ ... sn $ and the cumulative exclusive ends (src/alphabet.rs:375-393)."""
    total = sum(len(s) + 1 for s in sequences)
    if total > 0xFFFFFFFF:
        raise FmIndexError.text_too_large(total)
    text = np.zeros(total, dtype=np.uint8)
    bounds = np.zeros(len(sequences), dtype=np.uint32)
    pos = 0
    for i, s in enumerate(sequences):
        b = s.as_slice()
        text[pos:pos + len(b)] = b
        pos += len(b) + 1
        bounds[i] = pos
    return text, bounds
