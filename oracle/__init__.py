"""CPU oracle of the HiPIMS step (test infrastructure only)."""
