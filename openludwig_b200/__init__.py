"""openludwig_b200 -- B200-native (sm_100a) lattice Boltzmann time step with the
capabilities of OpenLUDWIG's solver path: D3Q27 cumulant / regularized-BGK +
WALE/WMLES stream-collide over sparse 8^3 blocks, Bouzidi walls, 2:1
multi-level sub-cycling, O(u^4) equilibrium + thermal DDF, and surface-stress
Cd/Cl/Cm -- all hand-written CUDA behind the C ABI in include/openludwig_b200.h.
"""
__version__ = "0.1.0"
