"""CPU oracle of the energy-game solver: test infrastructure only (see oracle.py)."""
