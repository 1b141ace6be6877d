"""Batched and served jobs through the C ABI (cuda_replace_jobs, cuda_replace_server_*):
many independent jobs, each an input with its own sequence of pairs, run as segmented
launches. Every result must equal the chained bytes.replace of its job, alone or in a mix."""
import random
import threading
import time

import pytest

from cuda_replace_b200 import cuda_replace_wrapper as Wr
from cuda_replace_b200 import workloads as WL

pytestmark = pytest.mark.gpu


def chain(src, pairs):
    for p, r in pairs:
        src = src.replace(p, r)
    return src


def small_c5_jobs(count, seed=5, max_size=256 << 10):
    jobs = []
    for i in range(count):
        j = WL.c5_job(i, min_size=4096, max_size=max_size, seed=seed)
        jobs.append((j.data, j.pairs))
    return jobs


def test_replace_jobs_matches_chained(cr_lib):
    jobs = small_c5_jobs(160)
    outs = Wr.replace_jobs(cr_lib, jobs)
    for i, ((data, pairs), out) in enumerate(zip(jobs, outs)):
        assert out == chain(data, pairs), i


def test_replace_jobs_edge_cases(cr_lib):
    rng = random.Random(3)
    big_pat = bytes(rng.randrange(256) for _ in range(40))
    jobs = [
        (b"", [(b"a", b"b")]),                              # empty input
        (b"hello", []),                                     # no pair
        (b"abcabc" * 1000, [(b"", b"-")]),                  # empty pattern: Session path
        (b"ab" * 50000, [(b"ab" * 20, b"Z")]),              # bordered, L = 40: Session path
        (b"xyz" * 1000, [(b"y", b"Q" * 100)]),              # R > 64: Session path
        (b"a" * 100000, [(b"a", b"Q" * 64)]),               # 64x expansion: overflow, rerun
        (b"a" * 70001, [(b"aa", b"b"), (b"bb", b"c"), (b"cc", b"aaa")] * 6),  # 18 pairs: Session path
        (b"q" + big_pat * 3 + b"q", [(big_pat, b"")]),
        (bytes(range(256)) * 300, [(b"\x00\x01", b""), (b"\xff", b"\x00" * 33), (b"\x00\x00", b"N")]),
        (b"aaaa" * 5000 + b"b", [(b"aaa", b"X"), (b"XX", b"aa"), (b"aX", b"")]),
    ]
    outs = Wr.replace_jobs(cr_lib, jobs)
    for i, ((data, pairs), out) in enumerate(zip(jobs, outs)):
        assert out == chain(data, pairs), i


def test_jobs_across_tile_boundaries(cr_lib):
    """Periodic inputs whose every position is a candidate, cut at many sizes around the 16 KiB
    sub-tile and 128 KiB super-tile boundaries, mixed in one batch."""
    jobs = []
    for n in (1, 15, 16, 17, 16383, 16384, 16385, 131071, 131072, 131073, 400_001):
        for pat, rep in ((b"aa", b"X"), (b"aaa", b""), (b"a", b"bc"), (b"abab", b"Y"), (b"aab", b"QQQQQ")):
            base = b"a" if pat in (b"aa", b"aaa", b"a") else (b"ab" if pat == b"abab" else b"aab")
            src = (base * (n // len(base) + 1))[:n]
            jobs.append((src, [(pat, rep)]))
    outs = Wr.replace_jobs(cr_lib, jobs)
    for i, ((data, pairs), out) in enumerate(zip(jobs, outs)):
        assert out == chain(data, pairs), (i, len(data), pairs)


def test_server_results_alone_and_in_the_mix(cr_lib):
    """Continuous batching: requests submitted from several threads while earlier batches run
    give, per job, the same result as that job run alone, and as bytes.replace."""
    jobs = small_c5_jobs(120, seed=11, max_size=1 << 20)
    alone = []
    with Wr.Server(cr_lib, hbm_budget=256 << 20) as srv:
        for data, pairs in jobs[:12]:
            alone.append(srv.wait(srv.submit(data, pairs)))
    results = {}
    lock = threading.Lock()

    def client(idx):
        rng = random.Random(idx)
        for i in idx_lists[idx]:
            time.sleep(rng.random() * 0.002)
            t = srv.submit(*jobs[i])
            with lock:
                results[i] = t

    idx_lists = [list(range(k, len(jobs), 4)) for k in range(4)]
    with Wr.Server(cr_lib, hbm_budget=256 << 20, max_jobs_per_batch=16) as srv:
        threads = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        outs = {i: srv.wait(t) for i, t in results.items()}
        st = srv.stats()
    assert st["jobs_done"] == len(jobs) and st["batches"] >= 2
    assert st["p99_us"] >= st["p50_us"] > 0
    for i, (data, pairs) in enumerate(jobs):
        assert outs[i] == chain(data, pairs), i
    for i in range(12):
        assert outs[i] == alone[i], i


def test_server_budget_admission(cr_lib):
    """A small HBM budget: jobs are admitted batch by batch as memory frees up; a job larger
    than the whole arena runs through a Session; results stay exact."""
    rng = random.Random(8)
    jobs = []
    for i in range(30):
        n = rng.choice([100_000, 1_000_000, 3_000_000])
        src = bytes(rng.choice(b"abcd") for _ in range(2000)) * (n // 2000)
        jobs.append((src, [(b"ab", b"X"), (b"cd", b""), (b"dX", b"YYYY")]))
    jobs.append((b"abcd" * 6_000_000, [(b"bc", b"Q")]))  # 24 MB input: footprint above the arena
    with Wr.Server(cr_lib, hbm_budget=48 << 20) as srv:
        tickets = [srv.submit(d, p) for d, p in jobs]
        outs = [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["batches"] >= 3 and st["jobs_via_session"] >= 1
    assert st["arena_peak_bytes"] <= st["arena_bytes"]
    for i, ((data, pairs), out) in enumerate(zip(jobs, outs)):
        assert out == chain(data, pairs), i


def test_server_wait_timeout_and_unknown_ticket(cr_lib):
    with Wr.Server(cr_lib, hbm_budget=64 << 20) as srv:
        t = srv.submit(b"abc" * 1000, [(b"b", b"")])
        out = None
        for _ in range(2000):
            out = srv.wait(t, timeout_ms=10)
            if out is not None:
                break
        assert out == b"ac" * 1000
        with pytest.raises(RuntimeError, match="rc=-1"):
            srv.wait(t, timeout_ms=0)  # retired


def test_server_overflow_reruns_segmented(cr_lib):
    """Outputs far above the planned buffers (64x expansion) are flagged by the kernel without
    writing out of range; the job runs again in a later batch with buffers grown past the
    length that overflowed, not through a Session."""
    jobs = [(b"a" * 100_000, [(b"a", b"Q" * 64)]),
            (b"ab" * 300_000, [(b"b", b"R" * 60), (b"aR", b"S" * 64)]),
            (b"xyz" * 1000, [(b"y", b"")])]
    with Wr.Server(cr_lib, hbm_budget=512 << 20) as srv:
        outs = [srv.wait(srv.submit(d, p)) for d, p in jobs]
        st = srv.stats()
    assert st["jobs_via_session"] == 0
    for i, ((data, pairs), out) in enumerate(zip(jobs, outs)):
        assert out == chain(data, pairs), i


def test_server_cancel_queued_jobs(cr_lib):
    """Jobs cancelled while still queued give no result (their wait raises CancelledJob); jobs
    already on the device complete normally; every completed result is exact."""
    jobs = [WL.c5_job(i, min_size=1 << 20, max_size=4 << 20) for i in range(64)]
    with Wr.Server(cr_lib, max_jobs_per_batch=2) as srv:
        tickets = [srv.submit(j.data, j.pairs) for j in jobs]
        cancelled = {t for t in tickets[16:] if srv.cancel(t)}
        assert cancelled, "no queued job could be cancelled"
        for j, t in zip(jobs, tickets):
            if t in cancelled:
                with pytest.raises(Wr.CancelledJob):
                    srv.wait(t)
            else:
                assert srv.wait(t) == chain(j.data, j.pairs)
        assert srv.stats()["cancelled"] == len(cancelled)
        with pytest.raises(KeyError):
            srv.cancel(tickets[0])  # retired by its wait


def test_server_tenant_budgets(cr_lib):
    """A tenant's jobs never hold more device memory than its budget at once, they do not hold
    back another tenant's jobs, and a job larger than its tenant's whole budget is refused."""
    jobs = [WL.c5_job(i, min_size=256 << 10, max_size=2 << 20) for i in range(48)]
    with Wr.Server(cr_lib) as srv:
        budget = 24 << 20
        srv.set_tenant_budget(1, budget)
        tickets = [(j, srv.submit(j.data, j.pairs, tenant=1 + (i % 2))) for i, j in enumerate(jobs)]
        for j, t in tickets:
            assert srv.wait(t) == chain(j.data, j.pairs)
        cur, peak = srv.tenant_usage(1)
        assert cur == 0 and 0 < peak <= budget
        _, peak2 = srv.tenant_usage(2)
        assert peak2 > 0  # tenant 2 has no budget: it only shares the arena
        with pytest.raises(MemoryError):
            srv.submit(b"a" * (32 << 20), [(b"a", b"b")], tenant=1)


def test_replace_jobs_shared_server_reused(cr_lib):
    """cuda_replace_jobs keeps one server between calls (opened by the first, grown when a call
    needs more memory) and releases it on request; results stay exact across the calls."""
    small = small_c5_jobs(40)
    for _ in range(3):
        outs = Wr.replace_jobs(cr_lib, small)
        assert all(o == chain(d, p) for (d, p), o in zip(small, outs))
    large = [(WL.c5_job(i, min_size=8 << 20, max_size=24 << 20).data, [(b"\x01", b"xy")]) for i in range(6)]
    outs = Wr.replace_jobs(cr_lib, large)
    assert all(o == chain(d, p) for (d, p), o in zip(large, outs))
    cr_lib.lib.cuda_replace_jobs_release()
    outs = Wr.replace_jobs(cr_lib, small[:5])
    assert all(o == chain(d, p) for (d, p), o in zip(small[:5], outs))
