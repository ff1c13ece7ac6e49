"""B200-native SELM fluctuating-hydrodynamics step (monomers coupled to a
periodic Stokes fluid).  Compute runs in libselm_b200.so (hand-written
sm_100a CUDA); this package is the host-side binding."""
from .selm import Params, Topology, Selm, op_interp, op_spread, op_rfft3, op_irfft3  # noqa: F401

__all__ = ["Params", "Topology", "Selm", "op_interp", "op_spread", "op_rfft3", "op_irfft3"]
