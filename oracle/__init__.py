"""Test infrastructure: CPU oracle for the finite-volume hot path (see fvm_oracle)."""
