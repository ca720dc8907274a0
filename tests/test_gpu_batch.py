"""Batched rendering (rx_batch_*): every job's accumulators after a batch
equal rendering that job alone with rx_render, bit for bit, whatever the
batch mixes (scenes, sizes, spp, depth, light modes, estimators), however
the frames split into waves, and whatever extend block shape runs."""
import numpy as np
import pytest

import golden_scenes as gs
import roxy_native as nat
import workloads
from rendering.batch import BatchConfig, BatchRenderer, Job
from test_host_logic import _ns

pytestmark = pytest.mark.gpu

BUFS = (nat.RX_ACC_RADIANCE, nat.RX_ACC_NORMAL, nat.RX_ACC_ALBEDO, nat.RX_ACC_DEPTH, nat.RX_ACC_DISPLAY)


def _jobs():
    ns = _ns()
    return [
        Job(workloads.cornell_box(40, 40), 40, 40, 6, 8, direct_light_max_depth=8, seed=1),
        Job(gs.build_trace_scene(ns), 33, 47, 3, 6, direct_light_mode=1, direct_light_max_depth=3, seed=2),
        Job(gs.build_texture_scene(ns, indexed=True), 24, 24, 5, 5, direct_light_max_depth=2, seed=3,
            reference_compat=True),
        Job(workloads.instanced_box_scene(3000, 11, 50, 30), 50, 30, 2, 12, direct_light_max_depth=4, seed=4),
        Job(workloads.cornell_box(16, 16), 16, 16, 1, 4, seed=5, sample_clamp=0.0),
    ]


def _solo(job):
    acc = nat.Accumulator(job.width, job.height)
    acc.render(job.scene.native, job.params, job.spp)
    return acc


def _same(a, b):
    for w in BUFS:
        x, y = a.read(w), b.read(w)
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), w
    assert a.info()["rays"] == b.info()["rays"]
    assert a.info()["frames"] == b.info()["frames"]


@pytest.mark.parametrize("wave_paths,block", [(1 << 25, 128), (3000, 64), (9000, 256)])
def test_batch_equals_solo_renders(wave_paths, block):
    br = BatchRenderer(_jobs(), BatchConfig(wave_paths=wave_paths, extend_block=block))
    solo = [_solo(j) for j in br.jobs]
    br.render()
    st = br.batch.last_stats()
    assert st["waves"] >= (1 if wave_paths > 1e6 else 3)
    for j, s in zip(br.jobs, solo):
        _same(j.acc, s)


@pytest.mark.parametrize("tail", [0, 1 << 30, 400])
def test_batch_tail_equals_solo_renders_without_tail(tail):
    """k_tail in a batch (a wave's remaining bounces run path by path for
    every scene of the wave, each path's rays counted for its job) leaves
    every job's accumulators, frames and ray count equal to a solo render
    with one launch pair per bounce, whether it is off, takes over at bounce
    1 or takes over part way."""
    br = BatchRenderer(_jobs(), BatchConfig(wave_paths=9000, extend_block=128))
    br.batch.set_tail(tail)
    solo = []
    for j in br.jobs:
        acc = nat.Accumulator(j.width, j.height)
        acc.set_tail(0)
        acc.render(j.scene.native, j.params, j.spp)
        solo.append(acc)
    br.render()
    for j, s in zip(br.jobs, solo):
        _same(j.acc, s)


def test_batch_graph_replay_continues_accumulation():
    br = BatchRenderer(_jobs()[:3], BatchConfig(wave_paths=5000, extend_block=128))
    br.render()
    br.render()  # same batch: the captured graph replays
    for j in br.jobs:
        acc = nat.Accumulator(j.width, j.height)
        acc.render(j.scene.native, j.params, 2 * j.spp)
        _same(j.acc, acc)


def test_batch_argument_errors():
    jobs = _jobs()[:2]
    for j in jobs:
        j.prepare()
    b = nat.Batch()
    b.add(jobs[0].scene.native, jobs[0].acc, jobs[0].params, 1)
    with pytest.raises(ValueError, match="share one accumulator"):
        b.add(jobs[1].scene.native, jobs[0].acc, jobs[0].params, 1)
    with pytest.raises(ValueError, match="does not match the accumulator"):
        b.add(jobs[1].scene.native, nat.Accumulator(8, 8), jobs[1].params, 1)
    with pytest.raises(ValueError, match="extend block"):
        b.set_config(1 << 20, 96)


def test_autotuner_picks_a_measured_config():
    br = BatchRenderer(_jobs()[:3])
    cfg = br.autotune(waves=(1 << 12, 1 << 20), blocks=(64, 128), leaves=(2, 4), use_cache=False)
    t = br.tuning
    assert len(t["timings"]) == 8 and all(x["ms"] > 0 for x in t["timings"])
    best = min(t["timings"], key=lambda x: x["ms"])
    assert (cfg.leaf_size, cfg.wave_paths, cfg.extend_block) == (best["leaf"], best["wave_paths"],
                                                                 best["extend_block"])
    # the tuned batch still renders each job exactly as alone
    solo = [_solo(j) for j in br.jobs]
    br.render()
    for j, s in zip(br.jobs, solo):
        _same(j.acc, s)
