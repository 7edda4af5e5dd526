"""The critical-path walk over per-task traces (chompack_b200.trace), on
synthetic traces and on the exported programs, without a GPU."""
import numpy as np

from chompack_b200 import _native as N
from chompack_b200 import trace
from chompack_b200.plan import Plan
import golden_cases as G


def _tasks(ops, groups, waits_of, ntasks):
    tasks = np.zeros(ntasks, dtype=trace.TASK)
    waits = []
    for i in range(ntasks):
        tasks["op"][i] = ops[i]
        tasks["group"][i] = groups[i]
        tasks["wait_off"][i] = len(waits)
        tasks["nwait"][i] = len(waits_of[i])
        waits.extend(waits_of[i])
    return tasks, np.array(waits, dtype=np.int32).reshape(-1, 2)


def test_walk_follows_the_last_met_wait():
    # 0 -> {1, 2} -> group 5 (members 1, 2) -> 3; 4 independent and short
    ops = [1, 0, 0, 2, 0]
    groups = [-1, 5, 5, -1, -1]
    waits_of = [[], [(0, 1)], [(0, 1)], [(5, 2)], []]
    tasks, waits = _tasks(ops, groups, waits_of, 5)
    tr = np.zeros((5, 4), dtype=np.int64)
    #            claim  start   end
    tr[0, :3] = (1000, 1000, 11000)
    tr[1, :3] = (11500, 12000, 15000)
    tr[2, :3] = (13000, 13000, 20000)   # ends last of the group
    tr[3, :3] = (19000, 21000, 30000)   # claimed before the group ended
    tr[4, :3] = (1000, 1000, 2000)
    r = trace.critical_path(tasks, waits, tr)
    assert [p["task"] for p in r["path"]] == [0, 2, 3]
    assert r["span_ms"] == 0.029
    assert r["path_exec_ms"] == {"GEMM": 0.007, "POTRF": 0.01, "ASM": 0.009}
    # task 2 was claimed 2 us after task 0 ended; task 3 waited 1 us after the group
    assert r["path"][1]["claim_delay_ns"] == 2000 and r["path"][1]["wait_ns"] == 0
    assert r["path"][2]["claim_delay_ns"] == 0 and r["path"][2]["wait_ns"] == 1000
    assert r["cta_time_ms"] == round((10000 + 3000 + 7000 + 9000 + 1000) / 1e6, 2)


def test_exported_program_matches_the_plan():
    d, A, s = G.load("numeric31")
    pl = Plan(s, device=-1)
    tasks, waits = trace.program(pl, N.OP_CHOLESKY)
    info = pl.program_info(N.OP_CHOLESKY)
    assert len(tasks) == info["tasks"] and len(waits) == info["waits"]
    assert np.all(tasks["wait_off"][1:] >= tasks["wait_off"][:-1])
    assert int(tasks["wait_off"][-1]) + int(tasks["nwait"][-1]) == len(waits)
    # a trace that runs the list in order with unit durations: the path ends
    # at the last task and every task on it starts when its last wait is met
    nt = len(tasks)
    end = np.zeros(nt, dtype=np.int64)
    for i in range(nt):
        w0, nw = int(tasks["wait_off"][i]), int(tasks["nwait"][i])
        st = 0
        for cid, _ in waits[w0:w0 + nw]:
            if cid < nt:
                st = max(st, end[cid])
            else:
                m = np.nonzero(tasks["group"][:i] == cid)[0]
                st = max(st, end[m].max() if len(m) else 0)
        end[i] = st + 1000
    tr = np.zeros((nt, 4), dtype=np.int64)
    tr[:, 0] = tr[:, 1] = end - 1000
    tr[:, 2] = end
    r = trace.critical_path(tasks, waits, tr)
    assert r["path_claim_delay_ms"] == 0 and r["path_wait_ms"] == 0
    assert r["span_ms"] == r["path_tasks"] * 0.001
