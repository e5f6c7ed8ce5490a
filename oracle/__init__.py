"""Oracle: FP64 CPU restatement of the reference path (test infrastructure only)."""
