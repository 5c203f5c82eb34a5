"""Failure paths of the lane-protocol sessions (sessions.cu), made on the host.

The reference host drives calculator_retrieval_expand_sqmd_run and
calculator_retrieval_pure_pq_sqmd_run through rpcmem control blocks
(retrieval_db_common.h:56-190, retrieval_sqmd_pure_pq.h:57-163) from a thread
of its own.  These tests stand in for that host with ctypes: a session whose
host writes nothing must end by itself after ROVER_SESSION_IDLE_MS, a
shutdown or abort written into the block must end it, the index it serves
must refuse to unload while it runs, and a buffer with too much work or an
id outside the index must come back as DSP_ABORT with the reference's status
(sqmd_process_lane_buffer_payload_with_cap, retrieval_sqmd_common.c:215-252).
No kernel waits on the host, so nothing here can hang a GPU: every wait is a
host-side poll with a time limit.

Each scenario runs in a fresh process (the library's state is process-wide).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

AEE_SUCCESS, AEE_EFAILED, AEE_EBADPARM = 0, 1, 14

# SqControl offsets (search-branch layout, static_asserts in sessions.cu)
SQ_CTRL_STATE, SQ_LANE_COUNT, SQ_SESSION_STATE = 0, 4, 12
SQ_LANES, SQ_LANE_BYTES, SQ_BUF_BYTES = 128, 1792, 768
SQ_WORK, SQ_RESULT = 16, 272
SQ_QUERY_SLOT, SQ_QUERY_FLOATS = 14720, 1040
SQ_STARTUP = 19968
SQ_CONTROL_BYTES = 20096
SESS_RUNNING, SESS_SHUTDOWN, SESS_ABORT = 1, 2, 3
BUF_CPU_READY, BUF_DSP_DONE, BUF_DSP_ABORT = 1, 2, 3


def _scenario(name: str) -> dict:
    """Runs one scenario of this file in a child process and returns its report."""
    env = dict(os.environ, ROVER_SESSION_IDLE_MS="800")
    p = subprocess.run([sys.executable, __file__, name], capture_output=True, text=True, env=env, timeout=240,
                       cwd=ROOT)
    assert p.returncode == 0, (p.stdout + p.stderr)[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_sqmd_session_ends_when_the_host_goes_quiet():
    r = _scenario("idle")
    assert r["rc"] == AEE_EFAILED
    assert 0.7 <= r["seconds"] < 30, r
    assert r["unload_while_live"] == AEE_EFAILED and "SQMD session" in r["busy_error"]
    assert r["session_state"] == SESS_ABORT
    assert "idle limit" in r["error"]
    assert r["unload_after"] == AEE_SUCCESS


def test_sqmd_session_shutdown_and_abort_written_by_the_host():
    r = _scenario("shutdown")
    assert r["shutdown_rc"] == AEE_SUCCESS and r["shutdown_seconds"] < 0.7, r
    assert r["abort_rc"] == AEE_EFAILED and r["abort_seconds"] < 0.7, r


def test_sqmd_buffer_failures_come_back_as_dsp_abort():
    r = _scenario("bad_buffers")
    assert r["good_state"] == BUF_DSP_DONE and r["good_count"] == 3
    assert r["good_ids"] == [5, 9, 2]
    assert all(d >= 0 for d in r["good_dists"])
    assert r["too_much"] == [BUF_DSP_ABORT, -3]
    assert r["bad_id"] == [BUF_DSP_ABORT, -1]


def test_session_argument_checks():
    r = _scenario("args")
    assert r["pq_no_lanes"] == AEE_EBADPARM
    assert r["pq_no_index"] == AEE_EBADPARM and "pure-PQ index" in r["pq_no_index_error"]
    assert r["sq_bad_cap"] == AEE_EBADPARM
    assert r["sq_unknown_fd"] == AEE_EFAILED


# ---------------------------------------------------------------------------------------------------------------
# child side

def _child(name: str) -> dict:
    import ctypes as C
    import threading
    import time

    import numpy as np

    sys.path.insert(0, str(ROOT))
    from rover_b200.calculator import Calculator

    calc = Calculator()
    L, h = calc.lib, calc.handle
    L.rpcmem_alloc.restype = C.c_void_p
    L.rpcmem_alloc.argtypes = [C.c_int, C.c_uint32, C.c_int]
    L.rpcmem_to_fd.argtypes = [C.c_void_p]
    L.rpcmem_free.argtypes = [C.c_void_p]
    L.calculator_retrieval_expand_sqmd_run.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32]
    L.calculator_retrieval_pure_pq_sqmd_run.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    err = lambda: calc.last_error()  # noqa: E731

    n, dim, k = 64, 16, 4
    rng = np.random.default_rng(5)
    graph = rng.integers(0, n, size=(n, k)).astype(np.int32)
    codes = rng.integers(0, 256, size=(n, dim)).astype(np.uint8)
    assert calc.retrieval_load(graph, codes, n, dim, k, 0, 0.05, -1.0) == AEE_SUCCESS, err()

    base = L.rpcmem_alloc(25, 1, SQ_CONTROL_BYTES)
    assert base
    C.memset(base, 0, SQ_CONTROL_BYTES)
    fd = L.rpcmem_to_fd(base)

    def i32(off):
        return C.cast(C.c_void_p(base + off), C.POINTER(C.c_int32))

    def f32(off):
        return C.cast(C.c_void_p(base + off), C.POINTER(C.c_float))

    def start(lanes=2, cap=32):
        out = {}

        def run():
            t0 = time.monotonic()
            out["rc"] = L.calculator_retrieval_expand_sqmd_run(h, fd, lanes, cap)
            out["seconds"] = time.monotonic() - t0
            out["error"] = err()   # the library's last error is per thread

        t = threading.Thread(target=run)
        t.start()
        limit = time.monotonic() + 20
        while i32(SQ_SESSION_STATE)[0] != SESS_RUNNING and t.is_alive() and time.monotonic() < limit:
            time.sleep(0.001)
        return t, out

    rep: dict = {}
    if name == "idle":
        t, out = start()
        time.sleep(0.1)
        rep["unload_while_live"] = L.calculator_retrieval_unload(h)
        rep["busy_error"] = err()
        t.join(60)
        assert not t.is_alive()
        rep.update(out)
        rep["session_state"] = i32(SQ_SESSION_STATE)[0]
        rep["unload_after"] = L.calculator_retrieval_unload(h)
    elif name == "shutdown":
        for state, key in ((SESS_SHUTDOWN, "shutdown"), (SESS_ABORT, "abort")):
            t, out = start()
            i32(SQ_SESSION_STATE)[0] = state
            t.join(60)
            assert not t.is_alive()
            rep[key + "_rc"], rep[key + "_seconds"] = out["rc"], out["seconds"]
    elif name == "bad_buffers":
        t, out = start(cap=32)
        slot = SQ_QUERY_SLOT
        q = rng.normal(0, 1, dim).astype(np.float32)
        for j in range(dim):
            f32(slot + SQ_QUERY_FLOATS + 4 * j)[0] = float(q[j])
        i32(slot + 4)[0] = dim      # query_dim
        i32(slot + 8)[0] = 0        # legacy contract
        i32(slot)[0] = 1            # query generation

        def submit(lane, b, ids, count=None):
            buf = SQ_LANES + lane * SQ_LANE_BYTES + b * SQ_BUF_BYTES
            for j, v in enumerate(ids):
                i32(buf + SQ_WORK + 8 * j)[0] = int(v)
                i32(buf + SQ_WORK + 8 * j + 4)[0] = 0
            i32(buf + 8)[0] = len(ids) if count is None else count
            i32(buf)[0] = BUF_CPU_READY
            limit = time.monotonic() + 20
            while i32(buf)[0] == BUF_CPU_READY and time.monotonic() < limit:
                time.sleep(0.001)
            return buf

        buf = submit(0, 0, [5, 9, 2])
        rep["good_state"], rep["good_count"] = i32(buf)[0], i32(buf + 12)[0]
        rep["good_ids"] = [i32(buf + SQ_RESULT + 12 * j)[0] for j in range(3)]
        rep["good_dists"] = [f32(buf + SQ_RESULT + 12 * j + 8)[0] for j in range(3)]
        buf = submit(1, 0, list(range(33)))
        rep["too_much"] = [i32(buf)[0], i32(buf + 12)[0]]
        i32(SQ_SESSION_STATE)[0] = SESS_SHUTDOWN
        t.join(60)
        # a fresh session for the out-of-range id (the failed one stopped serving)
        t, out = start(cap=32)
        i32(slot)[0] = 2
        buf = submit(0, 1, [3, n + 7])
        rep["bad_id"] = [i32(buf)[0], i32(buf + 12)[0]]
        i32(SQ_SESSION_STATE)[0] = SESS_SHUTDOWN
        t.join(60)
        assert not t.is_alive()
    elif name == "args":
        rep["pq_no_lanes"] = L.calculator_retrieval_pure_pq_sqmd_run(h, fd, fd, 0, 32)
        rep["pq_no_index"] = L.calculator_retrieval_pure_pq_sqmd_run(h, fd, fd, 2, 32)
        rep["pq_no_index_error"] = err()
        rep["sq_bad_cap"] = L.calculator_retrieval_expand_sqmd_run(h, fd, 2, 33)
        rep["sq_unknown_fd"] = L.calculator_retrieval_expand_sqmd_run(h, fd + 1000, 2, 32)
    L.rpcmem_free(base)
    return rep


if __name__ == "__main__":
    print(json.dumps(_child(sys.argv[1])))
