"""The parity bar for the tests: oracle/parity.py holds it (the oracle's
checker), so that the tests and the benchmark's accuracy report apply the
same tolerances."""
from oracle.parity import (EDGE_SLACK, FRACTION_TOL, IRRADIANCE_FLOOR, IRRADIANCE_TOL, WORD_AGREEMENT,  # noqa: F401
                           accuracy, bits, compare, flat)
