"""gear_b200: B200-native (sm_100a) CROWN bound propagation and BaB select/split/prune
for GEAR's NLP global solver hot path. See include/gear_b200.h for the C ABI."""
from .graph import Graph, GraphError, trace
from .bounded import BoundedModule, BoundedTensor, PerturbationLpNorm

__all__ = ["Graph", "GraphError", "trace", "BoundedModule", "BoundedTensor", "PerturbationLpNorm"]
