"""detray's internal unit system (core/include/detray/definitions/units.hpp):
lengths in mm, energies in GeV, charges in e; a field of 1 T is
0.000299792458 GeV / (e mm)."""
um = 1e-3
mm = 1.0
cm = 10.0
m = 1000.0
MeV = 1e-3
GeV = 1.0
T = 0.000299792458
cm2 = cm * cm
g = 1.0 / 1.782662e-24  # GeV / c^2
