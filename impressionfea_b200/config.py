"""Input decks of the forging path (mirrors SimulationConfig3D / SimulationConfig of ImpressionFEA.Core).

Field names follow the reference records; defaults are the reference's defaults
(ThreeD/SimulationConfig3D.cs:19-76, Simulation/SimulationConfig.cs:14-39, Forging3DSolver.cs:27-50, :1048).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Forging3DConfig:
    """Material law, friction, press kinematics and numerics of one 3D forging case."""
    C: float = 100.0              # FlowStressLaw C (MPa)
    N: float = 0.0                # strain-hardening exponent n
    M: float = 0.1                # strain-rate sensitivity m
    eps0: float = 1.0             # strain offset eps0
    friction: float = 0.3         # shear friction factor m_f (tau = m_f * k)
    ram: float = 50.0             # ram speed, mm/s
    h: float = 3.0                # ElementSize, mm
    ds: float = 0.5               # StrokeIncrement, mm
    tol: float = 1e-3             # Tolerance on |dv|/|v|
    max_iter: int = 70            # MaxIterations
    auto_step: bool = True        # AutoStep
    max_cutbacks: int = 5         # MaxCutbacks
    remesh_quality: float = 0.12  # RemeshQuality
    size: float = 40.0            # billet size setting rateRef = ram / size (height of a vertical cylinder)
    sym_x: bool = True            # quarter model: x >= 0
    sym_y: bool = True            # y >= 0
    sym_factor: int = 4
    penalty_factor: float = 1e4   # Forging3DSolver.PenaltyFactor
    newton_blend: float = 0.6     # NewtonBlend
    quadratic_ls: bool = True     # QuadraticLineSearch
    extrapolate_start: bool = False
    adaptive_newton: bool = True
    sticky_secant: bool = False
    pcg_budget: int = 15          # PcgBudget


@dataclass
class Forging2DConfig:
    """2D axisymmetric / plane-strain upsetting case (SimulationConfig + DieSet)."""
    C: float = 120.0
    N: float = 0.05
    M: float = 0.15
    eps0: float = 0.01
    friction: float = 0.3
    ram: float = 10.0
    ds: float = 0.15
    tol: float = 1e-6
    max_iter: int = 60
    axisymmetric: bool = True
    length: float = 100.0
    radius: float = 10.0
    height: float = 30.0
    nx: int = 20
    nz: int = 60
    bottom_profile: np.ndarray = field(default_factory=lambda: np.array([[0.0, 0.0], [200.0, 0.0]]))
    top_profile: np.ndarray = field(default_factory=lambda: np.array([[0.0, 15.0], [200.0, 15.0]]))
