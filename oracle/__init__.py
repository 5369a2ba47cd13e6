"""CPU oracle of the pmlib3d particle-mesh step: test infrastructure only."""
