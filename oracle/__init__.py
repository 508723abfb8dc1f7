"""Oracle: a CPU restatement of the reference's simulation step (test infrastructure only)."""
