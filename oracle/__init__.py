"""CPU oracle for the SuperCountingBloom hot path (test infrastructure only)."""
