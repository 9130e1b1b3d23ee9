"""B200-native time step of the Fourier contour cell model.

Drop-in for the hot path of FourierContourCells.jl (its public names,
src/FourierContourCells.jl:55-76): ``Simulation``, ``step``/``run`` (Julia's
``step!``/``run!``), ``compute_gradients``, ``BodyType``, ``Tension``,
``Overlap``, ``PerimeterElasticity``, ``LinearRepulsion``, ``HarmonicBond``,
``OnTypes``, ``shape_index`` and the observables, over the C ABI of
include/fcc.h implemented by hand-written sm_100a CUDA kernels
(csrc/, built into lib/libfcc_b200.so).

The directory name is not a Python identifier; load it with
``importlib`` under the name ``fcc_b200`` (see ``load`` in the repository's
``__graft_entry__.py``).
"""

from .model import (ArgumentError, DimensionMismatch, DeviceError, PoolFull, BodyType, EnergyTerm, BodyTerm, ContactTerm,
                    BondTerm, Tension, PerimeterElasticity, Overlap, LinearRepulsion, HarmonicBond, OnTypes,
                    UserTerm, UserBodyTerm, UserContactTerm, UserBondTerm, Bending, ShapeIndexElasticity, Adhesion,
                    QuarticBond,
                    Bodies, PeriodicBox, vcat, nbodies, hexagonal_monolayer, with_nuclei, parent_bonds,
                    polydisperse_monolayer, minimum_image, wrap)
from .simulation import (Simulation, NativeSimulation, native_library, step, run, compute_gradients,
                         update_neighbors, perimeters, areas, shape_index, body_energy, positions,
                         unwrapped_positions, contours, protrusion, Gradients, Geometry, NeighborInfo,
                         pinned_bodies, pinned_copy)
from .ops import philox_noise, build_neighbors, barrier_selftest
from .pool import Pool
from .serving import Request, Result, Server

__all__ = [
    "ArgumentError", "DimensionMismatch", "DeviceError", "PoolFull", "Pool", "Request", "Result", "Server", "BodyType", "EnergyTerm", "BodyTerm", "ContactTerm",
    "BondTerm", "Tension", "PerimeterElasticity", "Overlap", "LinearRepulsion", "HarmonicBond", "OnTypes",
    "Bodies", "PeriodicBox", "vcat", "nbodies", "hexagonal_monolayer", "with_nuclei", "parent_bonds",
    "polydisperse_monolayer", "minimum_image", "wrap", "Simulation", "NativeSimulation", "native_library", "step",
    "run", "compute_gradients", "update_neighbors", "perimeters", "areas", "shape_index", "body_energy",
    "positions", "unwrapped_positions", "contours", "protrusion", "Gradients", "Geometry", "NeighborInfo",
    "philox_noise", "build_neighbors", "barrier_selftest", "pinned_bodies", "pinned_copy", "UserTerm",
    "UserBodyTerm", "UserContactTerm", "UserBondTerm", "Bending", "ShapeIndexElasticity", "Adhesion", "QuarticBond",
]
