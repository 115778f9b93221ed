"""Served mode, host logic (no GPU): admission against the HBM budget,
first-in first-out order, job states, cancellation, release, the completion
queue, argument validation, and the seeded request stream.  The
scheduler-only server runs the same bookkeeping as the device server with
every step completing when it is issued."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from beamform_project_b200 import native, serve


def _grid(n_spectra=640, S=320, B=8, A=64, ns=1, offset=0):
    return serve.JobSpec(serve.GRID, A, ns, B, n_spectra, S, serve.array_positions(A),
                         serve.band_frequencies(ns * 336),
                         directions=np.tile(np.array([[0, 0, 1]], np.float32), (B, 1)), pool_offset=offset)


def _tracker(n_spectra=640, S=10, n_src=3, A=32, ns=2):
    tr = np.zeros((n_src, 4), np.float32)
    tr[:, 0] = np.linspace(-0.2, 0.2, n_src)
    tr[:, 2] = 1e-6
    return serve.JobSpec(serve.TRACKER, A, ns, n_src, n_spectra, S, serve.array_positions(A),
                         serve.band_frequencies(ns * 336), trajectories=tr)


def test_job_bytes_follow_the_layout():
    with serve.Server(10**9, host_only=True) as s:
        g = _grid(n_spectra=640, S=320, B=8, A=64, ns=2)
        al = lambda n: -(-n // 256) * 256  # noqa: E731
        W = 2
        split = 2 * 336 * 2 * 128 * 32 * 2          # padded to 16 beams: N = 32
        exp = (al(64 * 12) + al(split) + al(2 * W * 336 * 8 * 4) + al(2 * W * 336 * 8)
               + al(2 * W * 21 * 1 * 8) + al(2 * 336 * 4) + al(8 * 12))
        assert s.job_bytes(g) == exp
        t = _tracker(n_spectra=640, S=10, n_src=3, A=32, ns=2)
        W = 64
        exp = al(32 * 12) + al(672 * 8) + al(3 * 16) + al(W * 672 * 3 * 4)
        assert s.job_bytes(t) == exp


def test_admission_is_fifo_against_the_budget():
    g = _grid(n_spectra=960)  # three windows
    with serve.Server(10**9, host_only=True) as probe:
        need = probe.job_bytes(g)
    with serve.Server(int(2.5 * need), max_jobs=8, host_only=True) as s:
        ids = [s.submit(_grid(n_spectra=960)) for _ in range(4)]
        assert s.step() == 2
        assert [s.poll(i) for i in ids] == [serve.LIVE, serve.LIVE, serve.QUEUED, serve.QUEUED]
        assert s.step() == 2 and s.step() == 2
        assert [s.poll(i) for i in ids[:2]] == [serve.DONE, serve.DONE]
        # the queue waits until finished jobs give their memory back
        assert s.step() == 0
        assert s.take_done() == ids[:2]
        for i in ids[:2]:
            s.release(i)
        assert s.step() == 2
        st = s.stats()
        assert st["jobs_admitted"] == 4 and st["steps"] == 4 and st["job_windows"] == 8
        assert st["arena_bytes_peak"] <= int(2.5 * need)
        assert st["beam_samples"] == 8 * 320 * 336 * 8


def test_live_slots_bound_admission():
    with serve.Server(10**10, max_jobs=3, host_only=True) as s:
        for _ in range(5):
            s.submit(_tracker())
        assert s.step() == 3
        assert s.stats()["queued_jobs"] == 2


def test_oversize_and_invalid_jobs_are_rejected():
    with serve.Server(10**6, host_only=True) as s:
        with pytest.raises(native.ResourceError):
            s.submit(_grid(n_spectra=320 * 400, B=128))
        assert s.stats()["jobs_rejected"] == 1
    with serve.Server(10**9, host_only=True) as s:
        with pytest.raises(native.InvalidArgument, match="multiple of window_spectra"):
            s.submit(_grid(n_spectra=500))
        with pytest.raises(native.InvalidArgument, match="pool_offset"):
            s.submit(_grid(offset=100))
        with pytest.raises(native.InvalidArgument, match="divide window_spectra"):
            s.submit(_grid(S=30))
        with pytest.raises(native.Unsupported, match="multiple of 32"):
            s.submit(_grid(S=80))
        bad = _tracker()
        bad.trajectories = bad.trajectories.copy()
        bad.trajectories[0] = (0.9, 0.5, 0.0, 0.0)
        with pytest.raises(native.InvalidArgument, match="unit disk"):
            s.submit(bad)
        tilt = _grid()
        tilt.directions = tilt.directions * 1.1
        with pytest.raises(native.InvalidArgument, match="unit vectors"):
            s.submit(tilt)
        with pytest.raises(native.Unsupported):
            s.submit(_grid(A=128))
        assert s.stats()["jobs_submitted"] == 0


def test_cancel_and_release():
    with serve.Server(10**10, host_only=True) as s:
        a = s.submit(_grid(n_spectra=320 * 5))
        b = s.submit(_grid(n_spectra=320 * 5))
        s.step()
        q = s.submit(_grid())
        s.cancel(q)                     # queued: removed before admission
        assert s.poll(q) == serve.CANCELLED
        s.cancel(a)                     # live: leaves at the next step
        assert s.poll(a) == serve.CANCELLED
        assert s.step() == 1
        with pytest.raises(native.LogicError):
            s.release(b)                # still live
        with pytest.raises(native.LogicError):
            s.cancel(a)                 # already cancelled
        s.release(a)
        s.release(q)
        assert s.poll(a) == serve.UNKNOWN
        with pytest.raises(native.OutOfRange):
            s.release(a)
        for _ in range(3):
            s.step()
        assert s.poll(b) == serve.DONE and s.take_done() == [b]
        s.release(b)
        st = s.stats()
        assert st["jobs_cancelled"] == 2 and st["arena_bytes_in_use"] == 0


def test_results_of_unfinished_jobs_are_refused():
    with serve.Server(10**10, host_only=True) as s:
        a = s.submit(_grid(n_spectra=640))
        with pytest.raises(native.LogicError, match="not complete"):
            s.result_pointers(a)
        s.step()
        s.step()
        assert s.poll(a) == serve.DONE
        ip, cp, pp, W = s.result_pointers(a)
        assert W == 2 and cp != 0 and pp != 0


def test_poisson_mix_is_seeded_and_in_range():
    a = serve.poisson_mix(seed=1, duration_s=1.0)
    b = serve.poisson_mix(seed=1, duration_s=1.0)
    assert len(a) == len(b) and 150 <= len(a) <= 250
    for x, y in zip(a, b):
        assert (x.kind, x.n_ant, x.n_shards, x.n_beams, x.n_spectra, x.pool_offset) == \
               (y.kind, y.n_ant, y.n_shards, y.n_beams, y.n_spectra, y.pool_offset)
    for j in a:
        assert j.n_ant in (32, 64) and 1 <= j.n_shards <= 4 and j.integration_spectra in (10, 320)
        assert j.n_spectra % 320 == 0 and 0.1 <= j.n_spectra * serve.SPECTRUM_S <= 2.0 + 320 * serve.SPECTRUM_S
        if j.kind == serve.GRID:
            assert j.n_beams in (1, 8, 32, 128)
            assert np.allclose(np.linalg.norm(j.directions, axis=1), 1, atol=1e-6)
        else:
            assert 1 <= j.n_beams <= 16


def test_request_loop_drains_the_stream():
    jobs = serve.poisson_mix(seed=3, duration_s=0.2)
    with serve.Server(40 * 10**9, max_jobs=64, host_only=True) as s:
        done = []
        r = serve.run_stream(s, jobs, on_done=done.append)
        st = s.stats()
        assert r["submitted"] == len(jobs) == len(done) == st["jobs_done"]
        assert st["live_jobs"] == 0 and st["queued_jobs"] == 0 and st["arena_bytes_in_use"] == 0
        assert st["job_windows"] == sum(j.n_spectra // 320 for j in jobs)
        assert st["beam_samples"] == sum(j.beam_samples() for j in jobs)
        assert st["arena_bytes_peak"] <= 40 * 10**9


def test_window_time_bound_limits_admission():
    """With a window-time bound, admission stops while the cost model's
    prediction for the next window would exceed it; a job that alone exceeds
    it still runs when nothing else is live."""
    jobs = serve.poisson_mix(seed=2, duration_s=0.3)
    with serve.Server(120 * 10**9, max_jobs=512, window_budget_us=300.0, host_only=True) as s:
        worst = 0.0
        orig = s.step

        def step():
            nonlocal worst
            n = orig()
            st = s.stats()
            if n > 1:
                worst = max(worst, st["predicted_ms_last"])
            return n
        s.step = step
        serve.run_stream(s, jobs)
        assert s.stats()["jobs_done"] == len(jobs)
        assert 0.0 < worst <= 0.300 + 1e-9
    heavy = _tracker(n_spectra=640, S=10, n_src=16, A=64, ns=4)
    with serve.Server(10**10, window_budget_us=10.0, host_only=True) as s:
        a = s.submit(heavy)
        b = s.submit(_tracker())
        assert s.step() == 1          # alone over the bound: admitted anyway
        assert s.stats()["predicted_ms_last"] > 0.010
        s.step()
        assert s.step() == 1 and s.poll(b) == serve.LIVE and s.poll(a) in (serve.DONE, serve.RUNNING)


def test_released_jobs_leave_the_completion_queue():
    with serve.Server(10**10, host_only=True) as s:
        a = s.submit(_grid(n_spectra=320))
        b = s.submit(_grid(n_spectra=320))
        s.step()
        assert s.poll(a) == serve.DONE and s.poll(b) == serve.DONE
        s.release(a)                    # released before it was taken
        assert s.take_done() == [b]
        assert s.take_done() == []


def test_zero_lengths_are_rejected_not_divided_by():
    with serve.Server(10**9, host_only=True) as s:
        with pytest.raises(native.InvalidArgument, match="divide window_spectra"):
            s.submit(_grid(S=0))
        cfg = native.ServeConfig()          # all zero: an invalid configuration
        job = _grid().to_c()
        assert native.lib().bf_serve_job_bytes(C.byref(cfg), C.byref(job)) == 0
    with pytest.raises(native.InvalidArgument):
        serve.Server(10**9, window_spectra=0, host_only=True)


def test_checkpoint_restore_resumes_where_it_stopped():
    """A live job's checkpoint, restored into a second server, runs only its
    remaining windows; a queued job's checkpoint carries its description."""
    with serve.Server(10**9, host_only=True) as a, serve.Server(10**9, host_only=True) as b:
        g = _grid(n_spectra=320 * 5, S=10, B=40, ns=2, offset=640)
        t = _tracker(n_spectra=320 * 4, S=10, n_src=5)
        jg, jt = a.submit(g), a.submit(t)
        a.step()
        a.step()
        img_g, img_t = a.checkpoint(jg), a.checkpoint(jt)
        spec = serve.spec_of_checkpoint(img_g)
        assert (spec.kind, spec.n_ant, spec.n_shards, spec.n_beams, spec.n_spectra, spec.integration_spectra,
                spec.pool_offset, spec.quantize) == (serve.GRID, 64, 2, 40, 1600, 10, 640, True)
        assert np.array_equal(spec.positions, g.positions) and np.array_equal(spec.directions, g.directions)
        assert np.array_equal(serve.spec_of_checkpoint(img_t).trajectories, t.trajectories)
        rg, rt = b.restore(img_g), b.restore(img_t)
        assert b.poll(rg) == serve.QUEUED
        steps = 0
        while b.poll(rg) != serve.DONE or b.poll(rt) != serve.DONE:
            b.step()
            steps += 1
        assert steps == 3        # 5 - 2 windows of the grid job (the tracker had 2 left)
        # a queued job round-trips through a checkpoint unchanged
        q = b.submit(_grid(n_spectra=640))
        again = b.restore(b.checkpoint(q))
        assert b.checkpoint(again)[:-8] == b.checkpoint(q)[:-8]


def test_checkpoint_errors():
    with serve.Server(10**9, host_only=True) as a:
        j = a.submit(_grid())
        img = bytearray(a.checkpoint(j))
        img[100] ^= 0x40
        with pytest.raises(native.InvalidArgument, match="checksum"):
            a.restore(bytes(img))
        with pytest.raises(native.InvalidArgument):
            a.restore(b"not an image at all")
        a.cancel(j)
        with pytest.raises(native.LogicError):
            a.checkpoint(j)
        good = a.checkpoint(a.submit(_grid()))
    with serve.Server(10**9, host_only=True, pool_spectra=10240) as other:
        with pytest.raises(native.InvalidArgument, match="pool settings"):
            other.restore(good)


def test_pool_hook_checks_arguments():
    """bf_serve_pool: antenna count and host-only servers are checked before
    any pointer is handed out."""
    import ctypes as C
    from beamform_project_b200 import native
    with serve.Server(10**9, max_jobs=4, host_only=True) as srv:
        ptr = C.c_void_p()
        assert native.lib().bf_serve_pool(srv._h, 48, C.byref(ptr), None, None) == 1
        assert "32 or 64" in native.last_error()
        assert native.lib().bf_serve_pool(srv._h, 64, C.byref(ptr), None, None) == 2
        assert "host-only" in native.last_error()
        assert native.lib().bf_serve_pool(None, 64, C.byref(ptr), None, None) == 1
        with pytest.raises(native.LogicError, match="host-only"):
            srv.pool(64)


def test_windows_per_step_serve_several_windows_and_stop_at_the_pool_end():
    """windows_per_step k: a job's windows go k at a time, the last step takes
    what is left, and a span stops at the end of the voltage pool."""
    with serve.Server(10**10, host_only=True, pool_spectra=320 * 8, windows_per_step=4) as s:
        a = s.submit(_grid(n_spectra=320 * 10, offset=0))          # 4 + 4 + 2 windows
        b = s.submit(_grid(n_spectra=320 * 6, offset=320 * 6))     # pool end after 2: 2 + 4
        steps = 0
        while s.step():
            steps += 1
        assert steps == 3
        ia, ib = s.job_info(a), s.job_info(b)
        assert ia["windows_launched"] == 10 and ia["admit_step"] == 0 and ia["last_step"] == 2
        assert ib["windows_launched"] == 6 and ib["last_step"] == 1
        st = s.stats()
        assert st["job_windows"] == 16
        assert sorted(s.take_done()) == sorted([a, b])


def test_windows_per_step_is_validated():
    with pytest.raises(native.InvalidArgument):
        serve.Server(10**9, host_only=True, windows_per_step=257)


def test_job_info_reports_steps():
    with serve.Server(10**10, host_only=True) as s:
        s.submit(_grid(n_spectra=640))
        s.step()
        j = s.submit(_tracker(n_spectra=960))
        assert s.job_info(j)["admit_step"] is None and s.job_info(j)["submit_step"] == 1
        while s.step():
            pass
        info = s.job_info(j)
        assert info["admit_step"] == 1 and info["last_step"] == 3 and info["windows_launched"] == 3
        with pytest.raises(native.OutOfRange):
            s.job_info(999)
