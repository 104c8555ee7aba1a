"""Configuration: reference defaults, derived values and settings.cfg parsing (CPU only)."""
from pathlib import Path

import pytest

from pct_reconstruction_b200 import Config, PCTError

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_defaults_derive_like_reference_header():
    # B.h:333-480 defaults: 16 cm / 0.0625 cm = 256 columns, (9-1)/0.25 = 32 slices,
    # T_BINS = int(35/0.0625 + 0.5) = 560, V_BINS = 36, ANGULAR_BINS = int(360/3 + 0.5) = 120.
    c = Config()
    assert (c.COLUMNS, c.ROWS, c.SLICES) == (256, 256, 32)
    assert c.NUM_VOXELS == 256 * 256 * 32
    assert c.RECON_CYL_HEIGHT == 8.0
    assert (c.T_BINS, c.V_BINS, c.ANGULAR_BINS) == (560, 36, 120)
    assert c.NUM_BINS == 560 * 36 * 120
    assert c.MLP_U_STEP == 0.0625 / 2
    assert c.MIN_MLP_LENGTH == 30 and c.HISTORIES_PER_BLOCK == 640 and c.DROP_BLOCK_SIZE == 204800
    import numpy as np
    assert c.LAMBDA == np.float32(0.0001)  # float global in the reference


def test_head_grid(c2_params):
    c = Config(**c2_params)
    assert (c.COLUMNS, c.ROWS, c.SLICES, c.NUM_VOXELS) == (200, 200, 32, 1_280_000)
    assert c.MLP_U_STEP == 0.1 / 2


def test_settings_cfg_parse():
    c = Config(str(GOLDEN / "settings_c1.cfg"))
    assert c.DROP_BLOCK_SIZE == 3200 and c.ITERATIONS == 6 and c.SIGMAS_TO_KEEP == 3
    assert c.VOXEL_THICKNESS == 0.25 and c.COLUMNS == 128 and c.MSC_DIFF_THRESH == 50
    assert c.SINOGRAM_FILTER == 1  # FBP_FILTER_TYPE alias


def test_bad_values_rejected():
    with pytest.raises(PCTError):
        Config(COLUMNS="abc")
    with pytest.raises(PCTError):
        Config(NOT_A_KEY=1)
    with pytest.raises(PCTError):
        Config(THREADS_PER_HISTORY=3)
    with pytest.raises(PCTError):
        Config(VOXEL_WIDTH=-1.0)


@pytest.mark.parametrize("params,reason", [
    (dict(COLUMNS="abc"), "COLUMNS: not an integer"),
    (dict(LAMBDA="1e-4x"), "LAMBDA: not a number"),
    (dict(NOT_A_KEY=1), "unknown key NOT_A_KEY"),
    (dict(THREADS_PER_HISTORY=3), "THREADS_PER_HISTORY must be 0 or 32"),
    (dict(VOXEL_WIDTH=-1.0), "VOXEL_WIDTH, VOXEL_HEIGHT and VOXEL_THICKNESS must be positive"),
    (dict(S_CURVE_ON=1, PRECISION="MIXED"), "S_CURVE_ON needs PRECISION EXACT"),
    (dict(SCATTER_MODE="DETERMINISTIC", PROJECTION_ALGORITHM="ROBUSTB"), "not built for PROJECTION_ALGORITHM ROBUSTB"),
])
def test_rejections_carry_their_reason(params, reason):
    """pct_config_last_error names why pct_config_set / pct_config_finalize refused a value."""
    with pytest.raises(PCTError, match=reason):
        Config(**params)


def test_settings_file_errors_carry_their_reason(tmp_path):
    with pytest.raises(PCTError, match="cannot open"):
        Config(str(tmp_path / "missing.cfg"))
    cfg = tmp_path / "bad.cfg"
    # keys of other subsystems are skipped; the malformed known key is the reported error
    cfg.write_text("OUTPUT_DIRECTORY = \"out\"\nSOME_HOST_OPTION = 3\nLAMBDA = fast // comment\nOTHER = 1\n")
    with pytest.raises(PCTError, match=r"bad\.cfg: LAMBDA: not a number: fast"):
        Config(str(cfg))



def test_create_failure_keeps_its_reason():
    """pct_create destroys the context it was building when it fails; pct_last_error(NULL) keeps why."""
    from pct_reconstruction_b200 import Context
    c = Config()
    c.struct.THREADS_PER_HISTORY = 3  # past the binding's own check: pct_create validates its copy
    with pytest.raises(PCTError, match="configuration: THREADS_PER_HISTORY must be 0 or 32"):
        Context(c)


def test_create_without_a_gpu_names_the_cuda_call():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pct_reconstruction_b200 import Context
    with pytest.raises(PCTError, match=r"cudaSetDevice\(0\)"):
        Context(Config())
