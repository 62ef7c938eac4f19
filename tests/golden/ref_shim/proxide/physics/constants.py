"""Stand-in for proxide.physics.constants (TEST INFRASTRUCTURE ONLY).

proxide 0.1.0a9 is not installed.  The values prolix's GB code reads from it
are set to those the benchmark configurations state: the Coulomb constant
332.0637 kcal A / (mol e^2) (prolix's own direct-Coulomb literal,
physics/system.py:135; prolix's test pins proxide's value only to 1e-4,
tests/physics/test_constants.py:17-21), solute dielectric 1, solvent 78.5,
probe radius 1.4 A.
"""

COULOMB_CONSTANT = 332.0637
COULOMB_CONSTANT_KCAL = COULOMB_CONSTANT
DIELECTRIC_WATER = 78.5
DIELECTRIC_PROTEIN = 1.0
PROBE_RADIUS = 1.4
BOLTZMANN_KCAL = 0.0019872041
