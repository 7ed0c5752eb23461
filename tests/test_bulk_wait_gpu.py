"""The bounded waits of the bulk-copy linear kernel give up cleanly.

Each warp of the "bulk" step kernel waits on a ring slot's mbarrier for its
rows' bulk copies.  SWALS_TEST_BULK_EXTRA_TX adds bytes to every slot's
expected count that no copy delivers, so no slot ever completes -- a wait on
something that never arrives -- while the copies themselves land normally.
Every warp must then give up after SWALS_BULK_WAIT_CYCLES SM clocks, count
the expiry, wait (bounded) for its other slots and leave; synchronize reports
SWALS_ERR_CUDA with the count, the next synchronize is clean, and the same
context goes on to run a correct step.  Run in a child process so that the
environment switches apply to it alone.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

CHILD = r"""
import os
import numpy as np
from ptha_b200 import Domain, SwalsError, workloads

kw, U, _ = workloads.linear_gaussian_basin(n=256, dx=1000.0)


def one_step(kernel):
    os.environ["SWALS_LINEAR_KERNEL"] = kernel
    d = Domain(**kw)
    d.set_U(U)
    d.evolve_one_step(dt)
    return d


probe = Domain(**kw)
probe.set_U(U)
dt = probe.linear_timestep_max()
ref = one_step("wide16")
ref.synchronize()
expect = ref.get_U()[:3]
d = one_step("bulk")
try:
    d.synchronize()
    print("RESULT no-error")
except SwalsError as e:
    print("RESULT error", e.code, str(e).replace("\n", " "))
d.synchronize()
print("RESULT cleared")
# the context is usable: a fresh domain steps the same state correctly
d2 = one_step("wide16")
d2.synchronize()
print("RESULT usable", all(np.array_equal(a, b) for a, b in zip(d2.get_U()[:3], expect)))
"""


def test_bulk_wait_gives_up_and_reports():
    env = dict(os.environ, SWALS_LINEAR_KERNEL="bulk", SWALS_TEST_BULK_EXTRA_TX="16",
               SWALS_BULK_WAIT_CYCLES="200000")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env["PYTHONPATH"] = root + os.pathsep + env.get("PYTHONPATH", "")
    out = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=root, capture_output=True, text=True,
                         timeout=300)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("RESULT")]
    assert out.returncode == 0, (out.stdout, out.stderr)
    assert lines[0].startswith("RESULT error 4 "), lines
    assert "bounded waits for bulk-copied rows ran out" in lines[0], lines
    assert lines[1] == "RESULT cleared", lines
    assert lines[2] == "RESULT usable True", lines
