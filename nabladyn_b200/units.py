"""Units and physical constants: nm, ps, Da (g/mol), kJ/mol, K.

The same unit system and constants as the reference (src/nabladyn/units.py:12-28): SI 2019
exact values, so results in these units compare directly.
"""

AVOGADRO = 6.02214076e23  # 1/mol
BOLTZMANN = 0.00831446261815324  # kJ/(mol K): k_B N_A, the molar gas constant
ANGSTROM = 0.1  # nm
FS = 0.001  # ps
BAR = 0.0602214076  # kJ/(mol nm^3): 1e5 Pa x 1e-27 m^3/nm^3 x N_A
ATM = 1.01325 * BAR  # kJ/(mol nm^3)

__all__ = ("AVOGADRO", "BOLTZMANN", "ANGSTROM", "FS", "BAR", "ATM")
