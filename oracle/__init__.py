"""CPU oracle (test infrastructure only): a restatement of gbasis's ERI algorithm."""
