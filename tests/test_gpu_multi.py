"""Uneven acquisitions in one graph launch: every acquisition's images equal those of its own
hf_pipeline_exec, for the initial schedule, for fused segment band passes (one persistent launch
per window length over several acquisitions) with several tile parameters, and for the schedule the
autotuner picks."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu


def test_multi_graph_matches_per_acquisition_exec(cuda):
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200.multi import Multi
    cfgs = [
        pl.PipelineConfig(height=256, width=256, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                          clutter_rank=4, form=1, max_batch=3),
        pl.PipelineConfig(height=128, width=256, frames=32, hop=8, z_begin=6, z_end=16, fs=37e3, z=0.18,
                          clutter_rank=2, form=0, max_batch=2),
        pl.PipelineConfig(height=256, width=128, frames=128, hop=32, z_begin=8, z_end=40, fs=37e3, z=0.35,
                          clutter_rank=4, form=1, max_batch=2),
        pl.PipelineConfig(height=128, width=128, frames=32, hop=8, z_begin=6, z_end=16, fs=37e3, z=0.3,
                          propagation=2, form=0, max_batch=4),
        pl.PipelineConfig(height=512, width=256, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.22,
                          clutter_rank=4, form=1, max_batch=2),
    ]
    rings, nframes, outs, expect = [], [], [], []
    for i, c in enumerate(cfgs):
        n = c.frames + (c.max_batch - 1) * c.hop
        fr = S.Interferograms(S.config1(n, height=c.height, width=c.width, acquisition=i)).frames(0, n)
        ring = torch.from_numpy(O.pack12(fr.reshape(-1))).to(cuda)
        rings.append(ring)
        nframes.append(n)
        p = pl.Pipeline(c)
        expect.append(p.run(ring, n, 0, c.max_batch).cpu().numpy())
        p.close()
        outs.append(torch.full((c.max_batch, 3, c.height, c.width), float("nan"), device=cuda))
    m = Multi(cfgs)
    first = [0] * len(cfgs)
    m.exec(rings, nframes, first, outs)
    torch.cuda.synchronize()
    for i in range(len(cfgs)):
        assert np.array_equal(outs[i].cpu().numpy(), expect[i]), i
    streams, ms = m.tune(rings, nframes, first, outs, reps=2)
    assert streams != 0 and ms > 0
    for o in outs:
        o.fill_(float("nan"))
    m.exec(rings, nframes, first, outs)
    m.exec(rings, nframes, first, outs)  # the graph is reused
    torch.cuda.synchronize()
    for i in range(len(cfgs)):
        assert np.array_equal(outs[i].cpu().numpy(), expect[i]), i
    m.close()


def _inputs(cfgs, cuda):
    import torch
    from holoflow_b200 import pipeline as pl
    rings, nframes, outs, expect = [], [], [], []
    for i, c in enumerate(cfgs):
        n = c.frames + (c.max_batch - 1) * c.hop
        fr = S.Interferograms(S.config1(n, height=c.height, width=c.width, acquisition=20 + i)).frames(0, n)
        ring = torch.from_numpy(O.pack12(fr.reshape(-1))).to(cuda)
        rings.append(ring)
        nframes.append(n)
        p = pl.Pipeline(c)
        expect.append(p.run(ring, n, 0, c.max_batch).cpu().numpy())
        p.close()
        outs.append(torch.full((c.max_batch, 3, c.height, c.width), float("nan"), device=cuda))
    return rings, nframes, outs, expect


def test_fused_segment_passes_match_per_acquisition_exec(cuda):
    import holoflow_b200 as hf
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200.multi import Multi
    cfgs = [  # two T = 32 and two T = 128 acquisitions on the segment pass, one plain, one fused-row
        pl.PipelineConfig(height=128, width=256, frames=32, hop=8, z_begin=6, z_end=16, fs=37e3, z=0.2,
                          clutter_rank=2, form=1, max_batch=3),
        pl.PipelineConfig(height=256, width=128, frames=32, hop=8, z_begin=4, z_end=12, fs=67e3, z=0.3,
                          clutter_rank=4, form=1, max_batch=2),
        pl.PipelineConfig(height=256, width=128, frames=128, hop=32, z_begin=8, z_end=40, fs=37e3, z=0.35,
                          clutter_rank=4, form=1, max_batch=2),
        pl.PipelineConfig(height=128, width=256, frames=128, hop=32, z_begin=10, z_end=50, fs=67e3, z=0.25,
                          clutter_rank=4, form=1, max_batch=2),
        pl.PipelineConfig(height=128, width=128, frames=32, hop=8, z_begin=6, z_end=16, fs=37e3, z=0.3,
                          clutter_rank=2, form=0, max_batch=2),
        pl.PipelineConfig(height=256, width=256, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.22,
                          clutter_rank=4, form=1, max_batch=2),
    ]
    for i, c in enumerate(cfgs):
        p = pl.Pipeline(c)
        kind = p.band_pass()
        p.close()
        assert kind == (hf.HF_BAND_TC_SEGMENTS if i < 4 else hf.HF_BAND_FP32 if i == 4 else hf.HF_BAND_TC_ROWS), i
    rings, nframes, outs, expect = _inputs(cfgs, cuda)
    first = [0] * len(cfgs)
    m = Multi(cfgs)
    for sch in [dict(branches=2, largest_first=1, fused=1),
                dict(branches=1, largest_first=1, fused=1, seg_tiles=1, band_ctas=40),
                dict(branches=3, largest_first=0, fused=1, seg_tiles=2)]:
        m.set_schedule(**sch)
        assert m.schedule() == {"branches": 1, "largest_first": 1, "fused": 0, "seg_tiles": 0, "band_ctas": 0,
                                **sch}
        for o in outs:
            o.fill_(float("nan"))
        m.exec(rings, nframes, first, outs)
        torch.cuda.synchronize()
        for i in range(len(cfgs)):
            assert np.array_equal(outs[i].cpu().numpy(), expect[i]), (sch, i)
    streams, ms = m.tune(rings, nframes, first, outs, reps=2)
    sch = m.schedule()
    assert abs(streams) == sch["branches"] and (streams > 0) == bool(sch["largest_first"]) and ms > 0
    for o in outs:
        o.fill_(float("nan"))
    m.exec(rings, nframes, first, outs)
    torch.cuda.synchronize()
    for i in range(len(cfgs)):
        assert np.array_equal(outs[i].cpu().numpy(), expect[i]), (sch, i)
    for bad in [dict(branches=0), dict(branches=7), dict(fused=2), dict(seg_tiles=-1), dict(band_ctas=-3)]:
        with pytest.raises(hf.HfError):
            m.set_schedule(**bad)
    m.close()
