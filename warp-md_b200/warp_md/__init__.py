"""warp_md (B200 build) -- drop-in for warp-md's RMSD plans on sm_100a.

Mirrors the reference's Python surface for this path
(python/warp_md/__init__.py:17,232-240 re-exporting the PyO3 classes of
crates/traj-py/src/io.rs):

    system = System.from_arrays(atom_table, positions0=coords[0])
    traj = Trajectory.from_numpy(coords)               # (frames, atoms, 3)
    sel = system.select("name CA")
    RmsdPlan(sel, reference="frame0", align=True).run(traj, system, device="cuda:0")
    PairwiseRmsdPlan(sel, metric="rms").run(traj, system)
    AlignPlan(sel, mass=True).run(traj, system)           # (frames, 12): R, t
    SuperposePlan(sel).run(traj, system)                   # every atom superposed

Every plan runs on the CUDA library in ``_native/libwarpmd_rmsd.so``; there is
no CPU path.  ``device="cpu"`` raises, ``"auto"`` means ``"cuda:0"``.
"""
from __future__ import annotations

__version__ = "0.4.30"

from ._native import WarpMdError  # noqa: F401
from .core import Selection, System, Trajectory  # noqa: F401
from .plans import (AlignPlan, AtomicAdpPlan, AtomicFluctPlan, BfactorsPlan, PairwiseRmsdPlan,  # noqa: F401
                    RmsdPerResPlan, RmsdPlan, RmsfPlan, RotationMatrixPlan, SuperposePlan, SuperposeTrajectoryPlan,
                    TrajectoryClusterPlan)
from . import synth  # noqa: F401

__rust_cuda_enabled__ = True
__rust_build_profile__ = "b200-sm100a"


def native_version() -> str:
    from ._native import version

    return version()


__all__ = ["System", "Selection", "Trajectory", "RmsdPlan", "PairwiseRmsdPlan", "AlignPlan", "RotationMatrixPlan",
           "SuperposePlan", "SuperposeTrajectoryPlan", "RmsfPlan", "AtomicFluctPlan", "BfactorsPlan", "AtomicAdpPlan",
           "RmsdPerResPlan", "TrajectoryClusterPlan", "WarpMdError", "synth"]
