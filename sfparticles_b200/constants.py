"""Physical constants: scipy.constants (CODATA 2022) values, the same numbers
the reference imports (sfparticles/particles.py:5), written exactly."""
import math

C = 299792458.0
M_E = float.fromhex("0x1.279dcc922bcd9p-100")      # 9.1093837139e-31 kg
E_CHARGE = float.fromhex("0x1.7a4da290c1653p-63")  # 1.602176634e-19 C
HBAR = float.fromhex("0x1.185a7057c690dp-113")     # 1.0545718176461565e-34 J s
EPSILON_0 = float.fromhex("0x1.37876f1591150p-37")  # 8.8541878188e-12 F/m
PI = math.pi
ALPHA = float.fromhex("0x1.de3d429c6dc9dp-8")      # 0.0072973525643

# names the reference exports from sfparticles.particles
c, m_e, e, hbar, epsilon_0, pi = C, M_E, E_CHARGE, HBAR, EPSILON_0, PI
