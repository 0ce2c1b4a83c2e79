"""The bounded-wait path of the TMA pipeline kernels, made to run out on purpose.

The pipeline kernels wait on an mbarrier for each tile copy with a bound of one
second of the GPU's global timer; on expiry they flag the instance (status 2),
wait (again bounded) for the copies they did issue, and return, and the run
reports ESC_ETIMEOUT.  The test knob ESC_PIPE_DROP_COPY=1, read when a batch is
created, makes those kernels withhold their first copy: its wait runs out with
nothing in flight, and no fault, trap or hang is involved.  Afterwards an
ordinary batch in the same process must still give the oracle's results.
"""
import time

import numpy as np
import pytest

import esc
from esc import fields
from oracle import core_shell_oracle as orc

pytestmark = pytest.mark.gpu


def test_pipeline_wait_runs_out_then_the_process_recovers(monkeypatch):
    monkeypatch.setenv("ESC_ROWS", "pipe")
    monkeypatch.setenv("ESC_COLS", "block")
    c0, phi = fields.initial_fields(64, radius=16.0)
    monkeypatch.setenv("ESC_PIPE_DROP_COPY", "1")
    t0 = time.time()
    with esc.Batch([phi], precision="fp64") as b:
        assert b.describe()[0]["rows"] == "tma-pipeline"
        with pytest.raises(esc.EscError) as ei:
            b.run([c0], dt=0.01, steps=1)
    assert ei.value.status == esc.ESC_ETIMEOUT, str(ei.value)
    assert time.time() - t0 < 60
    monkeypatch.delenv("ESC_PIPE_DROP_COPY")
    with esc.Batch([phi], precision="fp64") as b:
        assert b.describe()[0]["rows"] == "tma-pipeline"
        cs, hs, bad = b.run([c0], dt=0.01, steps=5)
    co, ho = orc.run_simulation(c0, phi, dt=0.01, steps=5)
    assert bad == [-1]
    assert np.max(np.abs(cs[0] - co)) / np.max(np.abs(co)) < 1e-12
