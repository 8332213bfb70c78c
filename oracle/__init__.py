"""CPU oracle of the ED-MRDT per-timestep path — test infrastructure only."""
