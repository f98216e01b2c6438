"""B200-native Digital Twin Brain time-step path.

The conductance-based LIF block update (four receptor channels, Poisson
noise, CSR spike propagation) and the Balloon-Windkessel BOLD model as
hand-written sm_100a CUDA kernels behind a C ABI (``include/dtb.h``,
``libdtb.so``), with drop-in Python classes mirroring the reference's
``models/block.py`` and ``models/bold_model_pytorch.py``.
"""
from .network import BoldModel, Network  # noqa: F401
from .synthetic import NetworkSpec, single_block, whole_brain  # noqa: F401

__all__ = ["Network", "BoldModel", "NetworkSpec", "single_block", "whole_brain"]
