"""Physical constants, same values as the reference (constants.pyx:3-12)."""
import sys

c = 299792458.0
elementary_charge = 1.602176565e-19
m_e = 9.10938291e-31
m_p = 1.672621777e-27
epsilon_0 = 8.85418781762e-12
pi = 3.141592653589793
machineEpsilon = sys.float_info.epsilon
doubleMaxVal = sys.float_info.max
doubleMinVal = sys.float_info.min
