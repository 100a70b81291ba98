"""Batched events with deposits resident on the GPU: CUDA-graph replay and
every launch shape reproduce the host-buffer call bit for bit, and the
autotuner picks one of its candidates."""
import numpy as np
import pytest

from cases import BOX_CSI, GRID, OP_CSI_TEFLON, TB80

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def deposits():
    from crysplight_b200.events import GammaMaterial, gamma_stage
    mat = GammaMaterial.from_csv("CsI", 4.51, "xcom_CSI.csv")
    g = gamma_stage(mat, BOX_CSI, n_events=1500, seed=21, yield_per_mev=5400.0)
    return g


def _device_events(engine, g):
    import torch
    from crysplight_b200.batching import DeviceEvents
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return DeviceEvents(engine, BOX_CSI, OP_CSI_TEFLON, GRID, TB80, xyz=T(g.dep_xyz), t0=T(g.dep_t),
                        photons=T(g.dep_photons), segment=T(g.dep_event), n_segments=1500, seed=8,
                        tau_ns=1000.0)


def _same(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    assert np.array_equal(a[2], b[2])
    assert a[3] == b[3]


def test_graph_replay_equals_the_host_call(engine, deposits):
    g = deposits
    ref = engine.run_segments(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, sources=g.dep_xyz, photons_per_source=g.dep_photons,
                              segment_of_source=g.dep_event, n_segments=1500, seed=8, t0s=g.dep_t,
                              tau_ns=1000.0)
    ev = _device_events(engine, g)
    ev.step()
    ev.sync()
    direct = ev.result()
    assert np.array_equal(direct[0], ref.maps)
    assert np.array_equal(direct[1].view(np.uint32), ref.tmin.view(np.uint32))
    assert np.array_equal(direct[2], ref.npe) and direct[3] == ref.counters
    ev.capture()
    for _ in range(2):
        ev.maps.zero_()
        ev.replay()
        ev.sync()
        _same(ev.result(), direct)


def test_launch_shape_does_not_change_results(engine, deposits):
    from crysplight_b200.batching import LaunchShape
    ev = _device_events(engine, deposits)
    out = []
    for s in (LaunchShape(), LaunchShape(2, 128, 32), LaunchShape(3, 256, 128), LaunchShape(1, 64, 32)):
        engine.set_launch(s.ctas_per_sm, s.threads_per_cta, s.warp_chunk)
        ev.step()
        ev.sync()
        out.append(ev.result())
    engine.set_launch(0, 0, 0)
    for o in out[1:]:
        _same(o, out[0])


def test_autotune_picks_a_candidate(engine, deposits):
    from crysplight_b200.batching import LaunchShape, autotune
    ev = _device_events(engine, deposits)
    cands = (LaunchShape(0, 256, 64), LaunchShape(0, 128, 32), LaunchShape(3, 256, 256))
    best, times = autotune(engine, ev.step, candidates=cands, repeats=2)
    assert best in cands and set(times) == set(cands) and all(t > 0 for t in times.values())
    ev.step()
    ev.sync()
    tuned = ev.result()
    engine.set_launch(0, 0, 0)
    ev.step()
    ev.sync()
    _same(tuned, ev.result())
