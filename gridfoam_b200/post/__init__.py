"""Post-processing on the device (gridfoam ``post/``): immersed-surface forces."""
