"""CPU oracle (test infrastructure): a C restatement of numax.linalg."""
