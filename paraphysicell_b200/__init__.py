"""B200-native mechanics timestep of paraPhysiCell.

The CUDA library (libppc.so, C ABI in include/ppc.h) holds the agent state in
HBM and runs the mechanics step; `paraphysicell_b200.device` binds it.
"""
from .abi import AgentArrays, Mesh, Params  # noqa: F401
