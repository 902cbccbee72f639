"""CPU oracle of the explicit step (test infrastructure; see oracle.h)."""
