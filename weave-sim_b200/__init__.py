"""weavesim_b200 — B200-native dynamic relaxation of woven (Kagome) timber gridshells.

The hot path (one DR iteration: Cosserat rod forces, Coulomb stick-slip crossings, conflict-free gather, kinetic
damping) runs as hand-written sm_100a CUDA behind the C ABI of include/weavesim.h; this package is the Python mirror
of the reference's solver interface (web/js/solver_gpu.js GpuSolver) over that ABI.
"""
from ._lib import Model, default_params, kagome, polylines, mask, lib, last_error  # noqa: F401
from .scenefile import load_scene  # noqa: F401
from . import configs  # noqa: F401
from .solver import GpuSolver, device_count  # noqa: F401,E402
