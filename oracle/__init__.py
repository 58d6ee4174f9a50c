"""CPU oracle of the solve path (test infrastructure only)."""
