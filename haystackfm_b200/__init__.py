"""haystackfm_b200: B200-native (sm_100a) batched FM-index query path."""
from .alphabet import (ALPHABET_SIZE, DnaSequence, compatible_symbols, concatenate_sequences,  # noqa: F401
                       decode_char, encode, encode_byte, encode_char, iupac_bases)
from .errors import FmIndexError  # noqa: F401
