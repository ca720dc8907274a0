"""CPU oracle for parity tests and the CPU baseline (test infrastructure only)."""
