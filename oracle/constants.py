"""Physical constants, restated from src/half_constants.F90:5-14."""
import math

PI = math.pi
TWOPI = 2.0 * PI
AUTOA = 0.529177249           # Bohr radius in Angstrom (half_constants.F90:8)
RYTOEV = 13.605826            # Rydberg in eV (half_constants.F90:9)
HATOEV = 2.0 * RYTOEV         # Hartree in eV (half_constants.F90:10)
FELECT = 2.0 * RYTOEV * AUTOA  # e^2 in eV*Angstrom (half_constants.F90:11)
EDEPS = 4.0 * PI * FELECT     # (half_constants.F90:12)
HSQDTM = RYTOEV * AUTOA * AUTOA  # hbar^2/2m in eV*Angstrom^2 (half_constants.F90:14)
