"""Streaming server (continuous batching): every window's images are the same when its stream runs
alone and when it runs in a mix of streams of different sizes, rates, forms and propagation that
are admitted and closed while others are on the GPU -- bit for bit in the chosen form, within
1e-5 relative L2 in the plain form (its FP32 Gram partials are split by batch size); admission
follows free device memory."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu


def _streams():
    from holoflow_b200 import pipeline as pl
    specs = {
        # 256^2, T = 64 hop 16, Fresnel, top-4 clutter filter, chosen form
        "a": (pl.PipelineConfig(height=256, width=256, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                                clutter_rank=4, form=1, max_batch=4), 64 + 16 * 11),
        # 128^2, T = 128 hop 32, Fresnel, plain form
        "b": (pl.PipelineConfig(height=128, width=128, frames=128, hop=32, z_begin=8, z_end=40, fs=37e3, z=0.2,
                                clutter_rank=4, form=0, max_batch=2), 128 + 32 * 5),
        # 256 x 512, T = 64 hop 16, angular spectrum, no clutter filter
        "c": (pl.PipelineConfig(height=256, width=512, frames=64, hop=16, z_begin=6, z_end=16, fs=37e3, z=0.3,
                                propagation=2, form=1, max_batch=3), 64 + 16 * 8),
    }
    data = {}
    for k, (cfg, n) in specs.items():
        fr = S.Interferograms(S.config1(n, height=cfg.height, width=cfg.width)).frames(0, n)
        data[k] = O.pack12(fr.reshape(-1)).reshape(n, -1)
    return specs, data


def _host(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).pin_memory()


def test_server_results_same_alone_and_in_the_mix(cuda):
    import torch
    from holoflow_b200.server import Server
    specs, data = _streams()
    outs = {k: torch.empty((cfg.max_batch, 3, cfg.height, cfg.width), dtype=torch.float32, pin_memory=True)
            for k, (cfg, n) in specs.items()}

    def run_alone(k):
        cfg, n = specs[k]
        srv = Server(max_streams=4)
        sid = srv.open(cfg, cfg.frames + 4 * cfg.max_batch * cfg.hop)
        frames = _host(data[k])
        got, pos = [], 0
        while pos < n or srv.ready(sid) > 0:
            if pos < n:
                step = min(cfg.hop * cfg.max_batch, n - pos)
                srv.push(sid, frames[pos:], step)
                pos += step
            done = srv.step({sid: outs[k]})
            srv.sync()
            got += [outs[k][i].numpy().copy() for i in range(done.get(sid, 0))]
        srv.close_all()
        return got

    alone = {k: run_alone(k) for k in specs}
    assert [len(alone[k]) for k in "abc"] == [12, 6, 9]

    # the mix: a and b start, c is admitted later, b closes early.  No round waits for the device:
    # each stream has two pinned output buffers, a step goes into a free one, and poll() reports
    # which batches have reached the host (their buffers are then read and reused).
    srv = Server(max_streams=4)
    sids, pos, got = {}, {k: 0 for k in specs}, {k: [] for k in specs}
    frames = {k: _host(v) for k, v in data.items()}
    bufs = {k: [torch.empty((cfg.max_batch, 3, cfg.height, cfg.width), dtype=torch.float32, pin_memory=True)
                for _ in range(2)] for k, (cfg, n) in specs.items()}
    issued = {k: [] for k in specs}   # (buffer, windows, cumulative windows at its end), oldest first
    total = {k: 0 for k in specs}

    def drain():
        delivered = srv.poll()
        for k, sid in list(sids.items()):
            while issued[k] and delivered.get(sid, 0) >= issued[k][0][2]:
                b, nw, _ = issued[k].pop(0)
                got[k] += [bufs[k][b][i].numpy().copy() for i in range(nw)]

    for k in "ab":
        cfg, _ = specs[k]
        sids[k] = srv.open(cfg, cfg.frames + 4 * cfg.max_batch * cfg.hop)
    import time
    t_end = time.monotonic() + 60.0   # the loop never waits for the device; bound it in time
    rnd = -1
    while time.monotonic() < t_end:
        rnd += 1
        if rnd == 2:
            cfg, _ = specs["c"]
            sids["c"] = srv.open(cfg, cfg.frames + 4 * cfg.max_batch * cfg.hop)
        if rnd == 5 and "b" in sids:
            srv.sync()      # b's delivered batches are read before it closes
            drain()
            srv.close(sids.pop("b"))
        for k, sid in sids.items():
            cfg, n = specs[k]
            # push only what the ring can take beside the windows still to deliver
            if pos[k] < n and len(issued[k]) < 2:
                step = min(cfg.hop * (1 + rnd % cfg.max_batch), n - pos[k])
                srv.push(sid, frames[k][pos[k]:], step)
                pos[k] += step
        outs = {}
        for k, sid in sids.items():
            used = {b for b, _, _ in issued[k]}
            free = [b for b in (0, 1) if b not in used]
            if free:
                outs[sid] = bufs[k][free[0]]
        done = srv.step(outs)
        for k, sid in sids.items():
            if done.get(sid, 0):
                b = next(b for b in (0, 1) if outs.get(sid) is bufs[k][b])
                total[k] += done[sid]
                issued[k].append((b, done[sid], total[k]))
        drain()
        if all(pos[k] >= specs[k][1] and srv.ready(sid) == 0 and not issued[k] for k, sid in sids.items()):
            break
        if not done:
            time.sleep(50e-6)  # nothing issued this round: the device is busy with earlier batches
    srv.sync()
    drain()
    lat = srv.latencies()
    assert len(lat) == sum(len(v) for v in got.values()) and min(lat) > 0
    srv.close_all()
    assert len(got["a"]) == 12 and len(got["c"]) == 9 and 1 <= len(got["b"]) < 6
    # bit for bit, except the plain form's FP32 Gram partials, whose split follows the batch size
    for k in specs:
        for w, img in enumerate(got[k]):
            if specs[k][0].form == 1:
                assert np.array_equal(img, alone[k][w]), (k, w)
            else:
                assert O.rel_l2(img, alone[k][w]) < 1e-5, (k, w)


def test_server_admission_by_free_device_memory(cuda):
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200.server import Server
    cfg = pl.PipelineConfig(height=128, width=128, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4, form=1, max_batch=2)
    free, _ = torch.cuda.mem_get_info()
    srv = Server(max_streams=2, hbm_reserve_bytes=free + (1 << 30))  # more than the device has free
    assert srv.open(cfg, 128) is None and srv.open_count() == 0
    srv.close_all()
    srv = Server(max_streams=2, hbm_reserve_bytes=1 << 20)
    a, b = srv.open(cfg, 128), srv.open(cfg, 128)
    assert a is not None and b is not None and srv.open(cfg, 128) is None  # no free slot
    srv.close(a)
    assert srv.open(cfg, 128) is not None  # the freed slot and memory admit the next stream
    big = pl.PipelineConfig(height=1024, width=1024, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4, form=1, max_batch=8)
    free, _ = torch.cuda.mem_get_info()
    srv2 = Server(max_streams=2, hbm_reserve_bytes=max(free - (512 << 20), 0))  # room for < 512 MB
    assert srv2.open(big, 256) is None                                        # needs ~2.6 GB
    assert srv2.open(cfg, 128) is not None                                    # needs ~30 MB
    srv2.close_all()
    srv.close_all()


def test_server_opens_a_stream_while_another_batch_is_on_the_device(cuda):
    """Admission does not wait for the device: while stream A's batches are still executing (their
    completion events not yet fired), stream B opens, is pushed and steps; A's images are the same
    as when A runs alone."""
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200.server import Server
    ca = pl.PipelineConfig(height=1024, width=1024, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                           clutter_rank=4, form=0, max_batch=8)
    cb = pl.PipelineConfig(height=128, width=128, frames=32, hop=8, z_begin=6, z_end=16, fs=37e3, z=0.2,
                           clutter_rank=2, form=1, max_batch=2)
    na, nb = 64 + 16 * 15, 32 + 8 * 3
    fa = S.Interferograms(S.config1(64, height=1024, width=1024)).frames(0, 64)
    pa = O.pack12(fa.reshape(-1)).reshape(64, -1)
    ha = _host(np.concatenate([pa] * ((na + 63) // 64))[:na])
    fb = S.Interferograms(S.config1(nb, height=128, width=128)).frames(0, nb)
    hb = _host(O.pack12(fb.reshape(-1)).reshape(nb, -1))

    def out(cfg):
        return torch.empty((cfg.max_batch, 3, cfg.height, cfg.width), dtype=torch.float32, pin_memory=True)

    # A alone: two batches of 8 windows
    srv = Server(max_streams=4)
    a = srv.open(ca, na)
    srv.push(a, ha, na)
    alone = []
    for _ in range(2):
        o = out(ca)
        assert srv.step({a: o})[a] == 8
        srv.sync()
        alone.append(o.clone())
    srv.close_all()

    srv = Server(max_streams=4)
    srv.reserve(1 << 30)  # later streams come from the pool
    a = srv.open(ca, na)
    srv.push(a, ha, na)
    oa = [out(ca), out(ca)]
    assert srv.step({a: oa[0]})[a] == 8
    assert srv.step({a: oa[1]})[a] == 8            # two plain 1024^2 batches queued on the device
    assert srv.inflight(a) >= 1
    b = srv.open(cb, nb)                            # admitted while A's batches run
    assert b is not None
    assert srv.inflight(a) >= 1, "opening a stream waited for the device"
    srv.push(b, hb, nb)
    ob = out(cb)
    assert srv.step({b: ob})[b] == 2
    srv.sync()
    assert srv.poll()[a] == 16 and srv.inflight(a) == 0
    for k in range(2):
        assert O.rel_l2(oa[k].numpy(), alone[k].numpy()) < 1e-5   # plain form: FP32 Gram partials
    ref = pl.Pipeline(cb).run(torch.from_numpy(O.pack12(fb.reshape(-1))).to(cuda), nb, 0, 2).cpu()
    assert torch.equal(ob, ref)
    srv.close_all()
