"""CPU FP64 oracle (test infrastructure only; see ``stenpy_oracle``)."""
