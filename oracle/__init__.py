"""CPU oracle of the GGDT (test infrastructure only; see ggdt_oracle.c)."""
