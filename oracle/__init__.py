"""CPU oracle for haystackfm's query path (test infrastructure only)."""
