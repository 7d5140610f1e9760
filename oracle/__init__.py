"""CPU oracle of the bake path (test infrastructure only)."""
