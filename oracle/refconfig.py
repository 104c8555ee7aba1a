"""The reference's parameters for the oracle, derived without the engine library.

TEST INFRASTRUCTURE ONLY (the CPU baseline's configuration).  The reference fixes its parameters
as macros in B.h; this module holds B.h's values for the parameters the oracle's MLP and DROP
restatements read, lets a workload override the independent ones, and derives the dependent ones
with B.h's own expressions (B.h:373-411):
    RECON_CYL_HEIGHT = SSD_V_SIZE - 1.0
    COLUMNS = int(2 * RECON_CYL_RADIUS / VOXEL_WIDTH)    ROWS = int(2 * RECON_CYL_RADIUS / VOXEL_HEIGHT)
    SLICES = int(RECON_CYL_HEIGHT / SLICE_THICKNESS)      NUM_VOXELS = COLUMNS * ROWS * SLICES
    MLP_U_STEP = VOXEL_WIDTH / 2 (unless a workload sets it)
The result is the pct_config structure of include/pct_api.h (its ctypes layout), which the oracle
takes; only the layout is shared with the engine, no code of it runs.
"""
from __future__ import annotations

import ctypes as C

from pct_reconstruction_b200._abi import pct_config  # the C structure layout only (no library load)

# B.h values (B.h:335, 351, 373, 389-392, 409, 419-423, 464-465; PROJECTION_ALGORITHM DROP = 2)
B_H = dict(VOXEL_WIDTH=0.0625, VOXEL_HEIGHT=0.0625, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=8.0, SSD_V_SIZE=9.0,
           MIN_MLP_LENGTH=30, LAMBDA=0.0001, DROP_BLOCK_SIZE=204800, HISTORIES_PER_BLOCK=640, ITERATIONS=10,
           PROJECTION_ALGORITHM=2, PSI_SIGN=1, ETA=2.5, IDENTIFY_X_N_AIR=0, X_N_AIR_THRESHOLD=0.1)
# parameters of other stages that a workload may name; they do not enter the MLP or DROP
IGNORED = {"T_BIN_SIZE", "V_BIN_SIZE", "ANGULAR_BIN_SIZE"}


class ReferenceConfig:
    """pct_config with B.h's values and derivations; attributes read like the structure's."""

    def __init__(self, **params):
        unknown = set(params) - set(B_H) - IGNORED - {"MLP_U_STEP"}
        if unknown:
            raise KeyError(f"not a parameter of the MLP/DROP path: {sorted(unknown)}")
        v = dict(B_H)
        v.update({k: p for k, p in params.items() if k not in IGNORED})
        c = pct_config()
        for k, x in v.items():
            if k != "MLP_U_STEP":
                setattr(c, k, x)
        c.RECON_CYL_HEIGHT = c.SSD_V_SIZE - 1.0
        slice_thickness = c.VOXEL_THICKNESS  # SLICE_THICKNESS, equal to VOXEL_THICKNESS in B.h
        c.COLUMNS = int(2 * c.RECON_CYL_RADIUS / c.VOXEL_WIDTH)
        c.ROWS = int(2 * c.RECON_CYL_RADIUS / c.VOXEL_HEIGHT)
        c.SLICES = int(c.RECON_CYL_HEIGHT / slice_thickness)
        c.NUM_VOXELS = c.COLUMNS * c.ROWS * c.SLICES
        c.MLP_U_STEP = params.get("MLP_U_STEP", c.VOXEL_WIDTH / 2)
        self._c = c

    def __getattr__(self, name):
        c = self.__dict__.get("_c")
        if c is not None and hasattr(c, name):
            return getattr(c, name)
        raise AttributeError(name)

    @property
    def struct(self) -> pct_config:
        return self._c


def reference_config(**params) -> ReferenceConfig:
    return ReferenceConfig(**params)


__all__ = ["reference_config", "ReferenceConfig", "B_H", "C"]
