"""Reference-compatible calls (ansEncode / ansDecode, no workspace argument)
made from several host threads on one shared stream. The library keeps one
workspace per (device, stream); each call's launches must stay adjacent in
stream order, and a workspace that grows for one thread's larger input must
stay alive for the calls of other threads that still use it. Every stream
must equal the oracle's and every decoded buffer its input."""
import threading

import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def test_compat_calls_from_threads_on_one_stream(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    stream = torch.cuda.Stream()
    threads, rounds = 4, 6
    # thread t: sizes grow with the round, so calls resize the shared workspace
    # while other threads' calls are queued on it
    work = []
    for t in range(threads):
        jobs = []
        for r in range(rounds):
            n = (150_000 << (r + t % 2)) + 7919 * t  # 150 KB to 9.6 MB; starts at 1 MiB
            x = W.random_bytes(n, 100 * t + r, "skewed")
            d_in = to_dev(x)
            cap = mb.getMaxCompressedSize(n)
            jobs.append({"x": x, "n": n, "d_in": d_in,
                         "out": torch.empty(cap, dtype=torch.uint8, device="cuda"),
                         "size": torch.zeros(1, dtype=torch.int32, device="cuda"),
                         "dec": torch.empty(n, dtype=torch.uint8, device="cuda")})
        work.append(jobs)
    torch.cuda.synchronize()
    errors = []
    start = threading.Barrier(threads)

    def run(jobs):
        try:
            start.wait()
            for j in jobs:
                mb.ansEncode(10, j["d_in"], j["n"], j["out"], j["size"], stream=stream)
                mb.ansDecode(10, j["out"], j["dec"], stream=stream)
        except Exception as e:  # reported below
            errors.append(e)

    ts = [threading.Thread(target=run, args=(jobs,)) for jobs in work]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=120)
    assert not errors, errors
    assert not any(t.is_alive() for t in ts)
    stream.synchronize()
    st, detail = mb.ans_last_status(stream)
    assert st == 0, (st, detail)
    for jobs in work:
        for j in jobs:
            nbytes = int(j["size"].item())
            s = to_host(j["out"][:nbytes])
            np.testing.assert_array_equal(s, oracle.ans_encode(j["x"], 10), err_msg=f"n={j['n']}")
            np.testing.assert_array_equal(to_host(j["dec"]), j["x"], err_msg=f"n={j['n']}")
