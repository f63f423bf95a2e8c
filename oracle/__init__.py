"""ORACLE — test infrastructure (CPU restatement of the reference's step)."""
