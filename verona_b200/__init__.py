"""verona_b200: B200-native SRHD step (reconstruction, HLL/HLLC fluxes,
con2prim, RK update, ghost fill) behind a C ABI, with Python mirrors of
Wesenheit/Verona's Verona1D/2D/3D HARM_HLL interface."""
from . import EosTypes
from ._lib import VBError, default_options, lib
from .solver import Solver

__all__ = ["EosTypes", "Solver", "VBError", "default_options", "lib"]
