"""CPU checker for the cross-section path (test infrastructure only)."""
