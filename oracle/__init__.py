"""CPU oracle of RELAX's relaxation loop -- test infrastructure only."""
