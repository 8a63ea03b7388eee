"""CPU oracle for the banded pair-HMM path (test infrastructure only; never on the product path)."""
