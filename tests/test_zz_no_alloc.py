"""ns_collide_pairs_noalloc: the batch narrowphase for hosts that cannot allocate device memory
while they run (an engine whose GPU memory is all reserved by its own pool, or a frame loop that
cannot afford the device-wide synchronisation of cudaMalloc/cudaFree). It works in a fixed
scratch area inside the library, so it takes at most 4096 pairs per call, and its results must be
the same bits as the allocating entry point's, which is the tolerance every narrowphase test here
uses. This file is collected last on purpose."""
import numpy as np
import pytest

from natsel_b200 import narrowphase
from natsel_b200.world import NsError

import _pairgen

pytestmark = pytest.mark.gpu


def test_matches_the_allocating_entry_point_on_two_calls_in_a_row():
    jobs = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, 4000, 77, 1.2)
    with_alloc, without = jobs.copy(), jobs.copy()
    for _ in range(2):  # the second call starts from the caches the first wrote back
        expected = narrowphase.collide_pairs(with_alloc)
        got = narrowphase.collide_pairs_noalloc(without)
        assert got.tobytes() == expected.tobytes()
        assert without.tobytes() == with_alloc.tobytes()
    assert (got["point_count"] > 0).sum() > 400


def test_a_small_call_after_a_full_one_reads_nothing_stale():
    full = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, narrowphase.NOALLOC_MAX_PAIRS, 78, 1.0)
    narrowphase.collide_pairs_noalloc(full)
    small = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, 10, 79, 1.0)
    ref = small.copy()
    got = narrowphase.collide_pairs_noalloc(small)
    expected = narrowphase.collide_pairs(ref)
    assert got.tobytes() == expected.tobytes() and small.tobytes() == ref.tobytes()


def test_batches_over_the_limit_are_rejected_before_any_work():
    jobs = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, narrowphase.NOALLOC_MAX_PAIRS + 1, 80, 1.0)
    before = jobs.tobytes()
    with pytest.raises(NsError) as err:
        narrowphase.collide_pairs_noalloc(jobs)
    assert err.value.code == 3 and "4096" in str(err.value)
    assert jobs.tobytes() == before
    assert len(narrowphase.collide_pairs_noalloc(jobs[:0].copy())) == 0


FIRST_CALL_SCRIPT = r"""
import sys
sys.path[:0] = [{root!r}, {tests!r}]
import numpy as np
from natsel_b200 import narrowphase
from oracle import pyoracle
import _pairgen
jobs = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, 3000, 81, 1.2)
ref = jobs.copy().view(pyoracle.PAIR_JOB_DTYPE)
got = narrowphase.collide_pairs_noalloc(jobs)        # the first library call of this process
want = pyoracle.collide_pairs(ref)
assert got.tobytes() == want.tobytes(), "results differ from the oracle"
assert jobs.tobytes() == ref.tobytes(), "written-back caches differ from the oracle"
again = narrowphase.collide_pairs_noalloc(jobs)       # second call, from the written-back caches
assert again.tobytes() == pyoracle.collide_pairs(ref).tobytes()
print("first-call ok", int((got["point_count"] > 0).sum()))
"""


def test_first_call_in_a_fresh_process_matches_the_oracle():
    """A host that cannot allocate makes this its first call into the library, at start-up:
    the device set-up that call does (stack limit, module load) must leave correct results.
    Runs in a new process, so nothing else has touched the device before it."""
    import os
    import subprocess
    import sys
    from conftest import ROOT, TESTS
    script = FIRST_CALL_SCRIPT.format(root=ROOT, tests=TESTS)
    out = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ))
    assert out.returncode == 0, out.stdout + out.stderr
    assert "first-call ok" in out.stdout
    assert int(out.stdout.split()[-1]) > 300
