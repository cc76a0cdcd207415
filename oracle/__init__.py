"""CPU FP64 oracle (test infrastructure only; see euv_oracle.py)."""
