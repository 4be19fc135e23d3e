"""CPU FP64 oracle of the jspsr reconstruction path (test infrastructure only)."""
