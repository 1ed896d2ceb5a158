"""Physical constants and unit conversions, identical to the reference's
(Constants.cpp:12-18, Constants.h:21)."""

bohr = 0.52917721092            # Angstrom per bohr
autocm = 2.194746313e5          # cm^-1 per hartree
autoK = 315775.0428639057
Hmass = 1837.15137              # electron masses
Dmass = 2.0 * Hmass
Cmass = 21891.6543
Omass = Cmass * 15.9994 / 12.0107
autokcalpmol = 627.509474277194  # kcal/mol per hartree

NUCLEAR_MASS = {"H": Hmass, "D": Dmass, "C": Cmass, "O": Omass}   # DiskIO.cpp:22-40

PES_QTIP4PF = 0
PES_TTM3F = 1
PES_IDS = {"qtip4pf": PES_QTIP4PF, "ttm3f": PES_TTM3F}
