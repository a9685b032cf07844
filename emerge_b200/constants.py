"""Physical constants with the values EMerge uses (``src/emerge/_emerge/const.py``)."""
C0 = 299792458.0
Z0 = 376.73031366857
EPS0 = 8.854187818814e-12
MU0 = 1.0 / (C0 * C0 * EPS0)
