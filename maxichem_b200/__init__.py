"""maxichem_b200: the per-call chemistry solve of imalsky/maxichem, built for NVIDIA B200 (sm_100a).

``CudaSolver(net, device, photo=True)`` / ``solver(x, T, P, dt, h, J=J) -> (x, h, done, steps)`` / ``solver.check()``
as in the reference; ``VulcanNetwork`` reads a VULCAN network. Importing the package does not import torch; the
solver module does, on first use.
"""

from .network import VulcanNetwork

__all__ = ["ADSolver", "CudaSolver", "CallResult", "Cotangents", "JvpResult", "LaunchResult", "VjpResult",
           "VulcanNetwork"]


def __getattr__(name: str):
    if name in ("CudaSolver", "CallResult", "LaunchResult"):
        from . import solver

        return getattr(solver, name)
    if name in ("ADSolver", "Cotangents", "JvpResult", "VjpResult"):
        from . import ad

        return getattr(ad, name)
    raise AttributeError(name)
