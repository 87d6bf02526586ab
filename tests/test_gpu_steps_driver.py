"""The profiling driver (python -m nodals_b200.steps) runs each of its
configurations for a few SIMPLE iterations and reports the last one."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config", ["fast", "fp64", "amg_fp32"])
def test_steps_driver_runs(native, capsys, config):
    from nodals_b200 import steps
    steps.main(["--mesh", "pipe_tiny", "--steps", "2", "--config", config])
    out = capsys.readouterr().out
    assert f"mesh pipe_tiny config {config}: iteration 2," in out
