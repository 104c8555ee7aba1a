"""Test configuration: the `gpu` marker, import paths and shared fixtures.

`-m "not gpu"` runs on a CPU-only machine: the oracle against known answers and golden
fixtures, host-side logic, and a load/symbol check of libpct_b200.so (no device calls).
`-m gpu` runs the parity tests proper through the C ABI on a CUDA device.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine through the C ABI")


def pytest_sessionstart(session):
    # Build what is missing (the engine library and the CPU oracle); an up-to-date tree is a no-op.
    from pct_reconstruction_b200 import _abi
    if not _abi.LIB_PATH.exists():
        from pct_reconstruction_b200 import build
        build.build()
    import oracle
    oracle.build()  # make: a no-op when up to date, a rebuild after a header change


@pytest.fixture(scope="session")
def c1_params():
    """Plain-pipeline small configuration: 128x128x16 voxels of 1x1x2.5 mm (radius 6.4 cm,
    SSD_V_SIZE 5 cm -> height 4 cm), 3200-history DROP blocks, lambda 1e-4, 1 mm MLP step."""
    return dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
                T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0, DROP_BLOCK_SIZE=3200,
                HISTORIES_PER_BLOCK=640, ITERATIONS=6, MLP_U_STEP=0.1)


@pytest.fixture(scope="session")
def c2_params():
    """Plain-pipeline head-size configuration: 200x200x32 voxels of 1x1x2.5 mm (radius 10 cm,
    SSD_V_SIZE 9 cm -> height 8 cm), 60000-history DROP blocks, MLP step VOXEL_WIDTH/2."""
    return dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=10.0, SSD_V_SIZE=9.0,
                T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0, DROP_BLOCK_SIZE=60000,
                HISTORIES_PER_BLOCK=480, ITERATIONS=12)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
