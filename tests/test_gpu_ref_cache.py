"""The reference entry point's table cache past its capacity.

gpu_batch_bls_verify keeps the distinct key tables of earlier calls on the
device; when a call's new tables do not fit beside them, the cache is emptied
and that call's tables are registered afresh.  The capacity is read from
BLS_REF_TABLE_CACHE when the first reference call creates its context, so the
calls run in a fresh process with a capacity of six tables: key sets of four
alternate (each change empties the cache), a subset of the resident set does
not, a call with more distinct tables than the capacity takes the path that
copies the tables with the call, and two new tables fit beside four.  Every
result is checked against the workload's known answer."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
import bls_gpu as G
import workload as WL

wl = WL.config_keyset(960, 8, seed=77)
g2 = np.array(json.loads(sys.argv[1]), dtype=np.uint64)
out = []

def call(keys):
    ix = np.nonzero(np.isin(wl["pk_index"], keys))[0]
    tabs = np.ascontiguousarray(wl["pk_tables"][wl["pk_index"][ix]])
    got = G.batch_bls_verify(wl["sigs"][ix], wl["nhms"][ix], g2, tabs)
    ok = [int(x) for x in got] == [int(x) for x in wl["expect"][ix]]
    out.append({"keys": keys, "items": int(len(ix)), "ok": ok, "stats": list(G.ref_cache_stats())})

call([0, 1, 2, 3])
call([4, 5, 6, 7])
call([0, 1, 2, 3])
call([1, 2])
call([0, 1, 2, 3, 4, 5, 6])
call([0, 1, 2, 3, 4, 5])
print("RESULT " + json.dumps(out))
"""


def test_reference_cache_empties_when_full(golden):
    env = dict(os.environ)
    env["BLS_REF_TABLE_CACHE"] = "6"
    env["PYTHONPATH"] = os.pathsep.join(
        [os.path.join(ROOT, "icp-gpu_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
        + ([env["PYTHONPATH"]] if env.get("PYTHONPATH") else []))
    g2 = json.dumps([int(v) for v in golden["g2_gen_coeffs"]])
    p = subprocess.run([sys.executable, "-c", CHILD, g2], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [s for s in p.stdout.splitlines() if s.startswith("RESULT ")][-1]
    calls = json.loads(line[len("RESULT "):])
    assert all(c["ok"] for c in calls), calls
    assert all(c["items"] > 0 for c in calls)
    # (resident tables, capacity, flushes) after each call
    stats = [tuple(c["stats"]) for c in calls]
    assert stats[0] == (4, 6, 0)    # four new tables fit
    assert stats[1] == (4, 6, 1)    # four more do not: emptied, then the new four
    assert stats[2] == (4, 6, 2)    # the first four again: emptied again
    assert stats[3] == (4, 6, 2)    # two of the resident tables: nothing changes
    assert stats[4] == (4, 6, 2)    # seven distinct tables exceed the capacity: copied with the call
    assert stats[5] == (6, 6, 2)    # two new tables fit beside the four resident ones
