"""EosTypes (src/eos.jl:1-22): the ideal-gas polytrope used by every solver."""
from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass(frozen=True)
class Polytrope:
    """Polytrope{T}(gamma), src/eos.jl:7-9."""

    gamma: float


def Pressure(u: float, eos: Polytrope) -> float:
    """src/eos.jl:11-13"""
    return (eos.gamma - 1) * u


def SoundSpeed(rho: float, u: float, eos) -> float:
    """src/eos.jl:15-21 (eos may be a Polytrope or gamma)."""
    g = eos.gamma if isinstance(eos, Polytrope) else float(eos)
    return math.sqrt((g * (g - 1) * u) / (rho + g * u))
