"""Uneven acquisitions in one graph launch: every acquisition's images equal those of its own
hf_pipeline_exec, for the initial schedule and for the one the autotuner picks."""
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
