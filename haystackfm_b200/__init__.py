"""haystackfm_b200: B200-native (sm_100a) batched FM-index query path of haystackfm.

IUPAC backward search with sampled-SA locate, and the bidirectional SMEM/MEM pipeline,
behind the C ABI in include/hfm.h (libhfm.so).  The Python classes mirror the
reference's FmIndex / BidirFmIndex API.
"""
from .alphabet import (ALPHABET_SIZE, DnaSequence, compatible_symbols, concatenate_sequences,  # noqa: F401
                       decode_char, encode, encode_byte, encode_char, iupac_bases)
from .errors import FmIndexError  # noqa: F401
from .fm_index import (BidirFmIndex, ExactDna, FmIndex, FmIndexConfig, IupacDna, MemHit,  # noqa: F401
                       OccEncoding)
