"""CPU oracle of the reconstruction path (test infrastructure only)."""
