"""Error type mirroring haystackfm's `FmIndexError` (src/error.rs:5-30), plus the
status codes of the C ABI (include/hfm.h)."""
from __future__ import annotations

HFM_OK = 0
HFM_E_CUDA = -1
HFM_E_OOM = -2
HFM_E_FORMAT = -3
HFM_E_ARG = -4
HFM_E_TIMEOUT = -5
HFM_E_OVERFLOW = -6
HFM_E_WALK = -7
HFM_E_CHAR = -8

STATUS_NAMES = {
    HFM_E_CUDA: "E_CUDA", HFM_E_OOM: "E_OOM", HFM_E_FORMAT: "E_FORMAT", HFM_E_ARG: "E_ARG",
    HFM_E_TIMEOUT: "E_TIMEOUT", HFM_E_OVERFLOW: "E_OVERFLOW", HFM_E_WALK: "E_WALK", HFM_E_CHAR: "E_CHAR",
}


class FmIndexError(Exception):
    """kind is one of: InvalidCharacter, EmptySequence, TextTooLarge, DeserializeError,
    SerializeError, GpuError (the reference enum's variants)."""

    def __init__(self, kind: str, message: str, status: int = 0):
        super().__init__(message)
        self.kind = kind
        self.status = status

    @classmethod
    def invalid_character(cls, ch, pos):
        return cls("InvalidCharacter", f"invalid DNA character '{ch}' at position {pos}")

    @classmethod
    def empty_sequence(cls):
        return cls("EmptySequence", "empty sequence")

    @classmethod
    def text_too_large(cls, n):
        return cls("TextTooLarge", f"text too large: {n} bytes exceeds u32::MAX")

    @classmethod
    def from_status(cls, status: int, message: str):
        if status == HFM_E_FORMAT:
            return cls("DeserializeError", f"deserialization failed: {message}", status)
        if status == HFM_E_CHAR:
            return cls("InvalidCharacter", message, status)
        if status == HFM_E_ARG and message.startswith("empty"):
            return cls("EmptySequence", message, status)
        return cls("GpuError", f"GPU error: {STATUS_NAMES.get(status, status)}: {message}", status)
