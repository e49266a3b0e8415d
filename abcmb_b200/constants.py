"""Physical constants in the units of abcmb/constants.py:8-39 (eV, cm, s, Mpc).

The kernels and the host code must use the same FP64 values as the
reference, so they are restated here verbatim.
"""
import math

c = 29979245800.0                 # speed of light, cm/s
c_Mpc_over_s = 9.71561e-15        # speed of light, Mpc/s
H0_over_h = 3.24078e-18           # 100 km/s/Mpc in 1/s
hbar = 6.582119569509e-16         # eV s
G = 1.18980205e-40                # G/c^2 in cm^3 eV^-1 s^-2
kB = 8.617343e-5                  # eV/K
mp = 938271999.0                  # eV
mn = 939565413.0                  # eV
me = 510998.9461                  # eV
TCMB_today = 2.34865418e-4        # eV
mH = mp + me + 13.5982860719383   # eV
mHe = 3.72839e9                   # eV
thomson_xsec = 6.652458734e-25    # cm^2
stef_bolt = math.pi ** 2 / (60.0 * hbar ** 3 * c ** 2)
rydberg = 13.598286071938324      # eV
E21 = 10.198714553953742          # eV
RHO_CRIT_UNIT = 3.0 * H0_over_h ** 2 / 8.0 / math.pi / G   # omega -> eV cm^-3
