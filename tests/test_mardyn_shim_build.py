"""The MarDyn shim harness (madpac_b200/mardyn_shim) compiles against the reference's headers and
objects, reads a configuration with the reference's own reader, and, on a machine without a CUDA
device, stops where the device container is created with the reference's error convention
(global_log->error, exit with the status code: MDGPU_ERR_CUDA = 2). CPU only."""
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT, system_from_golden
from madpac_b200 import workloads as W

DRIVER = os.path.join(ROOT, "madpac_b200", "mardyn_shim", "_build", "shim_driver")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="the shim harness was not built (no reference sources)")
@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_shim_reads_the_configuration_and_reports_a_missing_device():
    system, _, _ = system_from_golden("fcc864_unshifted")
    tmp = tempfile.mkdtemp(prefix="mdshim_")
    W.write_inp(system, os.path.join(tmp, "sys.inp"))
    W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
    r = subprocess.run([DRIVER, "sys.cfg", "2", ".", "0"], cwd=tmp, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2
    assert "GpuLinkedCells: mdgpu_create failed" in r.stdout + r.stderr
