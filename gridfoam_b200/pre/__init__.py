"""Pre-processing on the device (gridfoam ``pre/``): potential-flow initialisation."""
