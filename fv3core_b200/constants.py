"""Physical constants of the acoustic substep.

The values are those of FV3 (the reference's ``fv3core/utils/global_constants.py``
1-17 lists the same numbers); results can only match the reference if the
constants do, so they are kept identical.
"""
RADIUS = 6.3712e6  # Earth radius [m]
PI = 3.1415926535897931
OMEGA = 7.2921e-5  # Earth rotation rate [1/s]
GRAV = 9.80665  # gravity [m/s^2]
RDGAS = 287.05  # dry-air gas constant [J/kg/K]
RVGAS = 461.50  # water-vapour gas constant [J/kg/K]
CP_AIR = 1004.6  # dry-air heat capacity at constant pressure [J/kg/K]
KAPPA = RDGAS / CP_AIR
DZ_MIN = 2.0  # minimum layer thickness [m]
CV_AIR = CP_AIR - RDGAS
RDG = -RDGAS / GRAV
CNST_0P20 = 0.2
ZVIR = RVGAS / RDGAS - 1
RGRAV = 1.0 / GRAV
SDAY = 86400.0

# moist thermodynamics of the step preamble and epilogue (the same file, 7-8, 21-37)
HLV = 2.5e6  # latent heat of evaporation [J/kg]
HLF = 3.3358e5  # latent heat of fusion [J/kg]
CV_VAP = 3.0 * RVGAS
C_ICE = 1972.0
C_LIQ = 4.1855e3
CP_VAP = 4.0 * RVGAS
TICE = 273.16
DC_ICE = C_LIQ - C_ICE
LI0 = HLF - DC_ICE * TICE
