"""CPU oracle of the ICAR advection step: test infrastructure, never product."""
