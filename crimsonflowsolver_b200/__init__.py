"""crimsonflowsolver_b200: B200 (sm_100a) ElmGMR assembly + memLS NS solve.

The CUDA library is built in-tree with :func:`build`; every compute entry point
runs on the GPU through the C ABI in include/crimson_b200.h.
"""
from ._native import build, lib  # noqa: F401
from .problem import RCR, FlowParams, NetlistBC, NetlistLoopBC, time_params  # noqa: F401

__all__ = ["build", "lib", "FlowParams", "RCR", "NetlistBC", "NetlistLoopBC", "time_params", "mesh", "solver", "netlist"]


def __getattr__(name):
    if name in ("mesh", "solver", "problem", "netlist"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
