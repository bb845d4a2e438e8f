"""CPU oracle for the SPEEDY column physics (test infrastructure only; see speedy_oracle)."""
