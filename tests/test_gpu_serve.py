"""Served mode on the GPU: every job's result is the same alone and in a
mix (bit for bit), matches the plain entry points on the same voltage (the
tensor grid within the split-precision bar, the tracker and the int8 codes
exactly), and the device weight generator matches the reference's
generate_weights."""
from __future__ import annotations

import numpy as np
import pytest

from beamform_project_b200 import api, native, serve

pytestmark = pytest.mark.gpu
F = 336
POOL = 320 * 16
SEED, SIGMA = 5, 2.0


def _server(budget=4 * 10**9, max_jobs=32):
    return serve.Server(budget, max_jobs=max_jobs, pool_spectra=POOL, pool_seed=SEED, pool_sigma=SIGMA)


def _pool_rows(torch, A, row0, n_rows, ns):
    """The server's pool rows [row0, row0 + n_rows) (mod POOL) for channels
    of ns shards, from the same seeded generator: [shard][T][336][A]."""
    pool_ch = 4 * F
    out = []
    for r in range(row0, row0 + n_rows, 320):
        rr = r % POOL
        buf = torch.empty(320 * pool_ch * A, dtype=torch.uint8, device="cuda")
        api.generate_voltage(None, SEED + A, rr * pool_ch * A, SIGMA, None, 1, buf,
                             api.Dimensions(320, pool_ch, A, 1))
        out.append(buf.view(320, pool_ch, A))
    v = torch.cat(out, 0)[:, :ns * F, :].reshape(n_rows, ns, F, A).permute(1, 0, 2, 3).contiguous()
    return v


def _grid_job(A=64, ns=2, B=40, S=320, n_spectra=960, offset=320 * 15, seed=0):
    rng = np.random.default_rng(seed)
    lm = rng.uniform(-0.3, 0.3, size=(B, 2)).astype(np.float32)
    n = np.sqrt(np.float32(1) - (lm[:, 0] * lm[:, 0] + lm[:, 1] * lm[:, 1])).astype(np.float32)
    dirs = np.concatenate([lm, n[:, None]], 1).astype(np.float32)
    return serve.JobSpec(serve.GRID, A, ns, B, n_spectra, S, serve.array_positions(A),
                         serve.band_frequencies(ns * F), directions=dirs, pool_offset=offset, quantize=True)


def _tracker_job(A=64, ns=2, n_src=3, S=320, n_spectra=960, offset=640):
    tr = np.zeros((n_src, 4), np.float32)
    tr[:, 0] = np.linspace(-0.25, 0.25, n_src)
    tr[:, 1] = 0.05
    tr[:, 2] = np.float32(0.02 / n_spectra)
    tr[:, 3] = np.float32(-0.01 / n_spectra)
    return serve.JobSpec(serve.TRACKER, A, ns, n_src, n_spectra, S, serve.array_positions(A),
                         serve.band_frequencies(ns * F), trajectories=tr, pool_offset=offset)


def _run(server, specs):
    ids = [server.submit(s) for s in specs]
    for _ in range(10_000):
        if server.step() == 0:
            break
    server.sync()
    assert native.take_device_error() == 0
    out = [server.result(i) for i in ids]
    return out


def test_generate_weights_matches_reference(cuda, orc):
    torch = cuda
    A, B, ns = 64, 16, 2
    pos = serve.array_positions(A)
    freq = serve.band_frequencies(ns * F)
    job = _grid_job(A=A, ns=ns, B=B)
    w = torch.empty(ns * B * F * A * 2, dtype=torch.float32, device="cuda")
    api.generate_weights(None, torch.from_numpy(pos).cuda(), torch.from_numpy(freq).cuda(),
                         torch.from_numpy(job.directions).cuda(), w, api.Dimensions(1, F, A, B), ns)
    torch.cuda.synchronize()
    got = w.cpu().numpy().reshape(ns, B, F, A, 2)
    for s in range(ns):
        exp = orc.generate_weights(pos, freq[s * F:(s + 1) * F], job.directions).reshape(B, F, A, 2)
        ulp = np.abs(got[s].view(np.int32).astype(np.int64) - exp.view(np.int32).astype(np.int64))
        print(f"shard {s}: weights differing by 1 ulp: {int((ulp == 1).sum())} of {ulp.size}")
        assert ulp.max() <= 1


@pytest.mark.parametrize("S", [320, 10])
def test_served_grid_matches_plain_and_oracle(cuda, orc, S):
    torch = cuda
    job = _grid_job(S=S)
    with _server() as srv:
        (integ, codes, params), = _run(srv, [job])
    A, ns, B, T = job.n_ant, job.n_shards, job.n_beams, job.n_spectra
    v = _pool_rows(torch, A, job.pool_offset, T, ns)
    # plain tensor path on the same voltage and weights
    d = api.Dimensions(T, F, A, B)
    w = torch.empty(ns * B * F * A * 2, dtype=torch.float32, device="cuda")
    api.generate_weights(None, torch.from_numpy(job.positions).cuda(), torch.from_numpy(job.frequencies).cuda(),
                         torch.from_numpy(job.directions).cuda(), w, d, ns)
    split = torch.empty(api.split_weight_bytes(d, ns), dtype=torch.uint8, device="cuda")
    api.prepare_split_weights(None, w, split, d, ns)
    W = T // S
    pi = torch.empty(ns * W * F * B, dtype=torch.float32, device="cuda")
    api.grid_tensor_integrated(None, v, split, pi, None, None, d, S, ns)
    torch.cuda.synchronize()
    plain = pi.cpu().numpy().reshape(ns, W, F, B)
    assert integ.shape == plain.shape
    bar = 1e-3 + 1e-5 * np.abs(plain.astype(np.float64))
    assert np.all(np.abs(integ.astype(np.float64) - plain) <= bar)
    print(f"S={S}: served == plain bit for bit in {int((integ == plain).sum())} of {integ.size}")
    # against the FP64 oracle (shard 1, where the padding of 40 beams differs)
    wh = w.cpu().numpy().reshape(ns, B, F, A, 2)
    vh = v.cpu().numpy()
    ref64 = orc.beamform_integrated(vh[1], wh[1], T, F, A, B, S, f64=True)
    err = np.abs(integ[1].astype(np.float64) - ref64)
    assert np.all(err <= 1e-3 + 1e-5 * np.abs(ref64))
    # the served quantizer equals the reference quantizer on the served values
    for s in range(ns):
        qc, qp = orc.quantize(integ[s], W, F, B)
        assert np.array_equal(codes[s], qc)


@pytest.mark.parametrize("A,S,n_src", [(64, 320, 3), (64, 10, 9), (64, 16, 5), (32, 10, 16), (32, 20, 8),
                                       (32, 320, 1)])
def test_served_tracker_equals_plain_tracker(cuda, A, S, n_src):
    """Both tracker forms (windows of at most 16 spectra, and longer) give
    the plain tracker's results bit for bit."""
    torch = cuda
    job = _tracker_job(A=A, S=S, n_src=n_src)
    with _server() as srv:
        (integ, _, _), = _run(srv, [job])
    A, ns, T = job.n_ant, job.n_shards, job.n_spectra
    v = _pool_rows(torch, A, job.pool_offset, T, ns)
    W = T // S
    assert integ.shape == (W, ns * F, n_src)
    for s in range(ns):
        k = torch.from_numpy(api.wave_numbers(job.frequencies[s * F:(s + 1) * F])).cuda()
        for src in range(n_src):
            l0, m0, dl, dm = (float(x) for x in job.trajectories[src])
            dirs = api.tracker_window_directions(l0, m0, dl, dm, T, S)
            out = torch.empty(W * F, dtype=torch.float32, device="cuda")
            api.tracker(None, 1, v[s].contiguous(), torch.from_numpy(job.positions).cuda(), k,
                        torch.from_numpy(dirs).cuda(), None, out, api.Dimensions(T, F, A, 1), S)
            torch.cuda.synchronize()
            plain = out.cpu().numpy().reshape(W, F)
            assert np.array_equal(integ[:, s * F:(s + 1) * F, src], plain), (s, src)


def test_alone_equals_mix(cuda):
    """Each job's results are bit-identical served alone and in a mix that
    admits other jobs before, with and after it (other classes, other
    antenna counts, other window kinds), including admission while the job
    is live."""
    target_g = _grid_job(A=64, ns=2, B=40, S=320, n_spectra=1280, offset=320 * 3)
    target_t = _tracker_job(A=32, ns=3, n_src=5, S=10, n_spectra=960, offset=320 * 9)
    with _server() as srv:
        alone_g = _run(srv, [target_g])[0]
    with _server() as srv:
        alone_t = _run(srv, [target_t])[0]
    others = [_grid_job(A=32, ns=1, B=128, S=10, n_spectra=640, offset=320 * 5, seed=1),
              _grid_job(A=64, ns=4, B=8, S=320, n_spectra=960, offset=320 * 7, seed=2),
              _tracker_job(A=64, ns=1, n_src=16, S=320, n_spectra=640, offset=0)]
    with _server() as srv:
        first = [srv.submit(others[0])]
        ids = [srv.submit(target_g)]
        srv.step()
        ids.append(srv.submit(target_t))      # admitted while target_g is live
        srv.step()
        first += [srv.submit(o) for o in others[1:]]
        for _ in range(10_000):
            if srv.step() == 0:
                break
        srv.sync()
        assert native.take_device_error() == 0
        mix_g = srv.result(ids[0])
        mix_t = srv.result(ids[1])
        st = srv.stats()
        assert st["jobs_done"] == 5 and st["graph_captures"] >= 2
        assert st["step_ms_p50"] > 0.0
    for a, b in zip(alone_g, mix_g):
        assert np.array_equal(a, b)
    assert np.array_equal(alone_t[0], mix_t[0])


def test_admission_waits_for_memory_on_the_device(cuda):
    """A budget that holds one job at a time still serves a queue of three,
    each with the result it has alone."""
    jobs = [_grid_job(A=64, ns=1, B=8, S=320, n_spectra=640, offset=320 * i, seed=i) for i in range(3)]
    with serve.Server(10**9, pool_spectra=POOL, pool_seed=SEED, pool_sigma=SIGMA) as probe:
        need = probe.job_bytes(jobs[0])
    alone = []
    for j in jobs:
        with _server() as srv:
            alone.append(_run(srv, [j])[0][0])
    with serve.Server(int(1.5 * need), max_jobs=8, pool_spectra=POOL, pool_seed=SEED, pool_sigma=SIGMA) as srv:
        got = {}
        serve.run_stream(srv, jobs, on_done=lambda jid: got.__setitem__(jid, srv.result(jid)[0]))
        assert srv.stats()["jobs_done"] == 3
        assert srv.stats()["arena_bytes_peak"] <= int(1.5 * need)
    for k, jid in enumerate(sorted(got)):
        assert np.array_equal(got[jid], alone[k])


def test_checkpoint_restore_equals_uninterrupted(cuda):
    """Jobs checkpointed after two windows, their server destroyed, and
    restored into a new server finish with results bit-identical to an
    uninterrupted run (grid S = 10 and 320 with int8 codes, tracker S = 10);
    a job checkpointed before admission and one checkpointed when done
    restore too."""
    specs = [_grid_job(A=64, ns=2, B=40, S=10, n_spectra=320 * 5, offset=320 * 2, seed=3),
             _grid_job(A=32, ns=1, B=128, S=320, n_spectra=320 * 4, offset=320 * 6, seed=4),
             _tracker_job(A=64, ns=2, n_src=9, S=10, n_spectra=320 * 4, offset=320 * 11)]
    with _server() as srv:
        straight = _run(srv, specs)
    with _server() as a:
        ids = [a.submit(s) for s in specs]
        a.step()
        a.step()
        images = [a.checkpoint(i) for i in ids]
        queued = a.checkpoint(a.submit(specs[0]))        # not admitted yet: no windows served
        a.sync()
    with _server() as b:
        rids = [b.restore(img) for img in images]
        qid = b.restore(queued)
        for _ in range(10_000):
            if b.step() == 0:
                break
        b.sync()
        assert native.take_device_error() == 0
        resumed = [b.result(i) for i in rids]
        fresh = b.result(qid)
        done_image = b.checkpoint(rids[0])               # every window served
    with _server() as c:
        did = c.restore(done_image)
        c.step()
        c.sync()
        redone = c.result(did)
    for x, y in zip(straight, resumed):
        for u, v in zip(x, y):
            assert (u is None and v is None) or np.array_equal(u, v)
    for u, v in zip(straight[0], fresh):
        assert (u is None and v is None) or np.array_equal(u, v)
    for u, v in zip(straight[0], redone):
        assert (u is None and v is None) or np.array_equal(u, v)


def test_ingest_into_pool_is_what_jobs_read(cuda, orc):
    """The ingest hook: voltage written into the server's pool on its stream
    (a capture stage's job) is what a served grid job beamforms."""
    from conftest import random_voltage
    torch = cuda
    A, T, S, B, offset = 64, 640, 320, 24, 320 * 7
    v = random_voltage(T, F, A, seed=77)
    job = _grid_job(A=A, ns=1, B=B, S=S, n_spectra=T, offset=offset, seed=3)
    with _server() as srv:
        pool = srv.pool(A)
        assert tuple(pool.shape) == (POOL, 4 * F, A)
        src = torch.from_numpy(v).cuda()
        torch.cuda.synchronize()
        with torch.cuda.stream(torch.cuda.ExternalStream(srv.stream_handle())):
            pool[offset:offset + T, :F, :].copy_(src)
        (integ, _, _), = _run(srv, [job])
    d = api.Dimensions(T, F, A, B)
    w = torch.empty(B * F * A * 2, dtype=torch.float32, device="cuda")
    api.generate_weights(None, torch.from_numpy(job.positions).cuda(), torch.from_numpy(job.frequencies).cuda(),
                         torch.from_numpy(job.directions).cuda(), w, d, 1)
    torch.cuda.synchronize()
    ref64 = orc.beamform_integrated(v, w.cpu().numpy().reshape(B, F, A, 2), T, F, A, B, S, f64=True)
    err = np.abs(integ[0].astype(np.float64) - ref64)
    assert np.all(err <= 1e-3 + 1e-5 * np.abs(ref64))


def test_windows_per_step_products(cuda):
    """Serving k windows per step: the S = 10 grid, the trackers and the int8
    codes of S = 10 jobs equal one window per step bit for bit (their sums do
    not depend on where a step starts); the S = 320 grid stays within the
    split-precision bar of it (a window's tiles may start elsewhere); and a
    job alone equals the job in a mix at the same k."""
    specs = [_grid_job(A=64, ns=2, B=40, S=320, n_spectra=1280, offset=320 * 3),
             _grid_job(A=32, ns=1, B=128, S=10, n_spectra=960, offset=320 * 5, seed=1),
             _tracker_job(A=32, ns=3, n_src=5, S=10, n_spectra=960, offset=320 * 9),
             _tracker_job(A=64, ns=1, n_src=9, S=320, n_spectra=1280, offset=0)]
    with _server() as srv:
        one = _run(srv, specs)
    for k in (3, 4):
        with serve.Server(4 * 10**9, max_jobs=32, pool_spectra=POOL, pool_seed=SEED, pool_sigma=SIGMA,
                          windows_per_step=k) as srv:
            many = _run(srv, specs)
        with serve.Server(4 * 10**9, max_jobs=32, pool_spectra=POOL, pool_seed=SEED, pool_sigma=SIGMA,
                          windows_per_step=k) as srv:
            alone = _run(srv, [specs[0]])[0]
        for a, b in zip(alone, many[0]):
            assert np.array_equal(a, b)
        g320 = many[0][0].astype(np.float64)
        ref = one[0][0].astype(np.float64)
        assert np.all(np.abs(g320 - ref) <= 1e-3 + 2e-5 * np.abs(ref))
        for idx in (1, 2, 3):
            for a, b in zip(one[idx], many[idx]):
                if a is not None:
                    assert np.array_equal(a, b), (k, idx)
