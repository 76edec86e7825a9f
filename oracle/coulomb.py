"""Oracle restatement of the Coulomb matrix elements (test infrastructure); see functions."""
