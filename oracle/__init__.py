"""CPU oracle package (test infrastructure; see mfs_oracle.c)."""
