"""CPU oracle of the multi-density Woodcock tracker (test infrastructure only)."""
