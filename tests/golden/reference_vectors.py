"""Golden vectors and known-answer cases transcribed from haystackfm's own tests.

Each entry cites the reference test it comes from.  The reference is Rust and cannot
run here, so these are the expected values its tests assert, copied as data; the
oracle (oracle/hfm_oracle.cpp) is pinned against them in tests/test_oracle_golden.py.
"""

# tests/common/mod.rs:47-66 — (text, pattern, expected_count)
COUNT_VECTORS = [
    ("ACGT", "A", 1), ("ACGT", "C", 1), ("ACGT", "G", 1), ("ACGT", "T", 1),
    ("ACGT", "AC", 1), ("ACGT", "ACGT", 1), ("ACGTACGT", "ACGT", 2), ("ACGTACGT", "A", 2),
    ("AAAA", "A", 4), ("AAAA", "AA", 3), ("AAAA", "AAA", 2), ("AAAA", "AAAA", 1), ("AAAA", "C", 0),
    ("ACGTTAGCCAGTACGT", "GT", 3), ("ACGTTAGCCAGTACGT", "AGC", 1), ("ACGTTAGCCAGTACGT", "TAG", 1),
]

# src/c_array.rs:76-119 — (text codes, expected C array)
C_ARRAY_VECTORS = [
    ([1, 2, 3, 4, 0], [0, 1, 2, 3, 4, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5]),
    ([1, 1, 2, 2, 0], [0, 1, 3, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5, 5]),
    ([1, 5, 5, 0], [0, 1, 2, 2, 2, 2, 4, 4, 4, 4, 4, 4, 4, 4, 4, 4]),
]

# src/alphabet.rs:546-610 — COMPAT_LEN and COMPAT rows (0 = padding)
COMPAT_LEN = [0, 8, 8, 8, 8, 15, 12, 12, 12, 12, 12, 12, 14, 14, 14, 14]
COMPAT_ROWS = [
    [0] * 16,
    [1, 5, 6, 9, 11, 13, 14, 15, 0, 0, 0, 0, 0, 0, 0, 0],
    [2, 5, 7, 8, 11, 12, 14, 15, 0, 0, 0, 0, 0, 0, 0, 0],
    [3, 5, 6, 8, 10, 12, 13, 15, 0, 0, 0, 0, 0, 0, 0, 0],
    [4, 5, 7, 9, 10, 12, 13, 14, 0, 0, 0, 0, 0, 0, 0, 0],
    [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0],
    [1, 3, 5, 6, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0, 0, 0],
    [2, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0, 0, 0],
    [2, 3, 5, 6, 7, 8, 10, 11, 12, 13, 14, 15, 0, 0, 0, 0],
    [1, 4, 5, 6, 7, 9, 10, 11, 12, 13, 14, 15, 0, 0, 0, 0],
    [3, 4, 5, 6, 7, 8, 9, 10, 12, 13, 14, 15, 0, 0, 0, 0],
    [1, 2, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15, 0, 0, 0, 0],
    [2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0],
    [1, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0],
    [1, 2, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0],
    [1, 2, 3, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 0, 0],
]

# src/alphabet.rs:532-539 — concatenate "ACG","TT"
CONCAT_VECTOR = (["ACG", "TT"], [1, 2, 3, 0, 4, 4, 0], [4, 7])

# src/fm_index/query.rs:505-646 (sample rate 1 unless given) — (seqs, rate, pattern, kind, expected)
# kind "count": int; "locate": sorted [(seq_idx, pos)]; "map": {text_pos: (seq, off)}
QUERY_CASES = [
    (["ACGTACGT"], 1, "ACGT", "count", 2),
    (["ACGTACGT"], 1, "ACG", "count", 2),
    (["ACGTACGT"], 1, "CGT", "count", 2),
    (["ACGTACGT"], 1, "ACGTACGT", "count", 1),
    (["ACGTACGT"], 1, "A", "count", 2),
    (["ACGTACGT"], 1, "C", "count", 2),
    (["ACGTACGT"], 1, "G", "count", 2),
    (["ACGTACGT"], 1, "T", "count", 2),
    (["AAAA"], 1, "C", "count", 0),
    (["AAAA"], 1, "AC", "count", 0),
    (["ACGTACGT"], 1, "ACGT", "locate", [(0, 0), (0, 4)]),
    (["ACGTACGT"], 1, "ACGTACGT", "locate", [(0, 0)]),
    (["AAAA"], 1, "C", "locate", []),
    (["ACGTACGTACGT"], 4, "ACGT", "count", 3),
    (["ACGTACGTACGT"], 4, "ACGT", "locate", [(0, 0), (0, 4), (0, 8)]),
    (["ACGT", "TGCA"], 1, "ACGT", "count", 1),
    (["ACGT", "TGCA"], 1, "TGCA", "count", 1),
]
MAP_POSITION_CASE = (["ACGT", "TGCA"], {0: (0, 0), 3: (0, 3), 5: (1, 0), 8: (1, 3)})   # query.rs:637-646

# src/fm_index/query.rs:447-493 — multi-sequence locate at every sample rate equals rate 1
MULTI_SEQ_RATE_SEQS = ["ACGTACGTACGTTTTTACGGGACACAC", "TTTTGGGGCCCCAAAATTTTACGTACGT",
                       "ACACACACGTGTGTGTACGTACGTACGT", "GGGGGGGGTTTTTTTTCCCCCCCCAAAA"]
MULTI_SEQ_RATE_PATTERNS = ["A", "ACGT", "ACAC", "TTTT", "GGGG", "CCCCAAAA", "ACGTACGT"]
MULTI_SEQ_RATES = [2, 3, 4, 8, 16, 32]

# tests/query_tests.rs:182-209 — multi_sequence_queries
MULTI_SEQ_QUERIES = (["ACGTACGT", "TGCATGCA", "AAACCC"], {"ACGT": 2, "TGCA": 2, "AAA": 1, "CCC": 1})

# src/fm_index/lookup.rs:150-304 — lookup-table consistency cases: (text, depth, patterns)
LOOKUP_CASES = [
    ("ACGTTAGCCAGTACGT", 3, ["ACG", "CGT", "GCC", "TAG", "ACGT", "TTA", "AAA"]),
    ("ACGTACGTACGT", 4, ["ACGT"]),
    ("ACGTNACGT", 3, ["ACG", "CGT", "N", "ACGT"]),
]
LOOKUP_SHORT_PATTERN = ("ACGTACGT", 4, "ACG", 2)            # lookup.rs:194-200
EXACT_N_ZERO = ("ACGTNACGT", 3, "N")                        # lookup.rs:204-227

# src/fm_index/smem.rs:405-728 and tests/bidir_correctness.rs:204-294 — SMEM/MEM known answers
# (reference, query, min_len, mode, expected list of (qs, qe, match_count or None))
SMEM_CASES = [
    ("ACGTACGT", "ACGT", 1, "smem", [(0, 4, 2)]),                 # smem.rs:414-422
    ("ACGTACGT", "A", 2, "smem", []),                             # smem.rs:439-445
    ("AAAA", "CCCC", 1, "smem", []),                              # smem.rs:406-411
    ("ACGT", "N", 1, "smem", [(0, 1, 4)]),                        # smem.rs:628-638
    ("AACAAGAAT", "ANT", 1, "smem", [(0, 3, None)]),              # smem.rs:641-651
    ("ACGT", "NN", 1, "smem", [(0, 2, 3)]),                       # smem.rs:689-698
    ("ANCGT", "AC", 2, "mem", [(0, 2, 2)]),                       # smem.rs:701-716
    ("AAAA", "NA", 2, "smem", [(0, 2, None)]),                    # smem.rs:719-728
    ("ACGTACGTACGT", "ACGT", 1, "smem", [(0, 4, 3)]),             # smem.rs:518-533
]
# brute-force MEM comparison cases (bidir_correctness.rs:204-229, smem.rs:447-560)
BRUTE_FORCE_CASES = [
    ("ACGTACGT", "ACGT"), ("ACGTTAGCCAGTACGT", "CGTTAGC"), ("AAAACCCCC", "AACCC"),
    ("ACGT", "TGCA"), ("ACGT", "ACGT"), ("TTTTTTTT", "TTTTT"),
]

# src/fm_index/smem.rs:749-799 — SMEM-drop regression query
SMEM_DROP_QUERY = ("CGTTCTGGAAGCAATGGCTTTCCTTGAGGAATCCCACCCAGGGATCTTTGAAAACTCTTGT"
                   "CTTGAAACGATGGAAGTTGTTCAGCAAACAAGAGTGGACAAACTAACTCAAGGTCGCCAGA"
                   "CTTATGACTGGACATTGAATAGAAACCAACCAGCTGCAACTGCTTTGGCCAACA")

# tests/locate_iupac_parity.rs — (references, query) pairs
LOCATE_IUPAC_CASES = [
    (["ACGT"], q) for q in ["N", "R", "Y", "S", "W", "K", "M", "B", "D", "H", "V", "NN"]
] + [
    (["AAAGGG"], "RR"), (["ACGTACGT"], "NNN"), (["ACGACA"], "ACR"), (["ACGTACGT"], "RCG"),
    (["ACGT", "TGCA"], "N"), (["AAGG", "CCTT"], "R"), (["AAAA"], "S"),
    (["ACGTACGT"], "ACG"), (["ACGTACGT"], "RY"), (["ACGTACGT"], "ACGT"),
]
# tests/locate_gpu_parity.rs
LOCATE_GPU_CASES = [
    (["ACGTACGT"], "ACGT"), (["ACGTACGT"], "TTTT"), (["ACGT"], ""), (["AAAACCCGGG"], "A"),
    (["AAAACCCGGG"], "C"), (["AAAACCCGGG"], "G"), (["ACGT", "TGCA"], "A"),
    (["ACGTACGT", "NNNACGTNNN"], "ACG"), (["ACGTACGT", "NNNACGTNNN"], "ACGT"), (["ACNGT"], "N"),
    (["ACGT", "TTTT", "CCCC", "GGGG", "ACGTACGT"], "ACGT"),
] + [(["ACGTACGTACGTACGT"], q) for q in ["A", "C", "G", "T", "AC", "CG", "GT", "ACG"]]

# tests/mem_iupac_parity.rs — (references, query, min_len, mode)
MEM_IUPAC_CASES = [
    (["ACGTACGT"], "NACGT", 1, 0), (["ACGTACGT"], "RCGT", 1, 0), (["ACGTACGT"], "AYGT", 1, 0),
    (["ACGT"], "NN", 1, 0), (["ACGT", "TGCA", "GGGG"], "RNGT", 1, 0), (["ACGT"], "NA", 3, 0),
    (["ACGTACGT"], "ACYN", 1, 0),
    (["ACGTACGT"], "NACGT", 1, 1), (["ACGTACGT"], "RCGT", 1, 1), (["ACGTACGT"], "ANGT", 1, 1),
    (["ACGT"], "NNN", 1, 1), (["ACGT", "TGCA", "GGGG"], "RNGT", 1, 1), (["AAAA"], "SSS", 1, 1),
    (["ACGTACGT"], "ACYN", 1, 1),
]
# tests/gpu_mem_positions_parity.rs — (references, queries, min_len, mode, max_hits)
MEM_POSITION_CASES = [
    (["ACGTACGT"], ["ACGT"], 1, 0, 1024),
    (["ACGTACGT", "ACGT", "TTTTACGT"], ["ACGT"], 1, 0, 1024),
    (["ACGTACGT"], ["ACGT"], 1, 1, 1024),
    (["ACGTACGT", "CGTTAGCC", "AAACGT"], ["ACGT", "CGT", "AAA"], 1, 1, 1024),
    (["ACGTACGT"], ["A"], 4, 1, 1024),
    (["ACGTACGTACGTACGT"], ["ACGT"], 1, 1, 1),          # truncation flag, :492-507
]
