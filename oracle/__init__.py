"""CPU oracle of the Barnes-Hut step -- test infrastructure only (see oracle.py)."""
