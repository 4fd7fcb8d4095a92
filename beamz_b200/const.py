"""Physical constants and units, with the reference's values.

beamz uses non-CODATA vacuum constants (beamz/const.py:1-10); the update
coefficients depend on them, so they are kept exactly.
"""
LIGHT_SPEED = 299792458.0  # m/s
VAC_PERMITTIVITY = 8.85e-12
VAC_PERMEABILITY = 1.256e-6
EPS_0 = 8.85e-12
MU_0 = 1.256e-6

um = 1e-6
µm = 1e-6
μm = 1e-6
nm = 1e-9
