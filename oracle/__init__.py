"""CPU oracle of the mechanics timestep (test infrastructure only)."""
