"""CUDA-graph replay, launch shapes and ensembles of the acoustic substep.

A captured AcousticDynamics call replays to the same bits as an eager call,
the thread-block shape chosen by the autotuner changes no result, and an
ensemble step recorded in one graph advances every member exactly as the
members' own eager calls do."""
import numpy as np
import pytest

import cases


def _host(st):
    from fv3core_b200.storage import to_host

    return {k: to_host(getattr(st, k)) for k in cases.ACOUSTIC_STATE}


def _same(a, b):
    for k in a:
        np.testing.assert_array_equal(np.nan_to_num(a[k], nan=7.0), np.nan_to_num(b[k], nan=7.0), err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_graph_replay_matches_eager(precision):
    import torch

    import gpu_runs

    case = cases.acoustics_case(12, 8, 21, n_split=2)
    gd_a, ad_a, st_a = gpu_runs.make_acoustics(case, 12, 8, precision)
    ad_a(st_a)
    ad_a(st_a)
    torch.cuda.synchronize()
    eager = _host(st_a)
    gd_b, ad_b, st_b = gpu_runs.make_acoustics(case, 12, 8, precision)
    ad_b(st_b)  # the eager first call uploads the per-level factors
    graph = ad_b.capture(st_b)  # capturing runs nothing
    graph.replay()
    torch.cuda.synchronize()
    _same(eager, _host(st_b))
    del graph
    gd_a.close()
    gd_b.close()


@pytest.mark.gpu
def test_launch_shape_changes_no_result():
    import torch

    import gpu_runs
    from fv3core_b200 import _lib

    case = cases.acoustics_case(12, 8, 22, n_split=2)
    default = _lib.get_launch_shape()
    results = []
    try:
        for shape in [(32, 4, 128), (64, 2, 64), (128, 1, 256)]:
            _lib.set_launch_shape(*shape)
            gd, ad, st = gpu_runs.make_acoustics(case, 12, 8)
            ad(st)
            torch.cuda.synchronize()
            results.append(_host(st))
            gd.close()
    finally:
        _lib.set_launch_shape(*default)
    _same(results[0], results[1])
    _same(results[0], results[2])


@pytest.mark.gpu
def test_autotune_keeps_the_fastest_shape():
    import gpu_runs
    from fv3core_b200 import _lib, autotune

    case = cases.acoustics_case(12, 8, 23, n_split=1)
    gd, ad, st = gpu_runs.make_acoustics(case, 12, 8)
    default = _lib.get_launch_shape()
    try:
        cands = [(32, 4, 128), (64, 2, 128)]
        best, timings = autotune.tune(lambda: ad(st), candidates=cands, repeats=1)
        assert set(timings) == set(cands) and all(t > 0 for t in timings.values())
        assert best == min(timings, key=timings.get)
        assert _lib.get_launch_shape() == best
    finally:
        _lib.set_launch_shape(*default)
        gd.close()


@pytest.mark.gpu
def test_ensemble_graph_matches_members_eager():
    import torch

    from fv3core_b200.ensemble import Ensemble

    spec = [(12, 8, 1), (16, 6, 2)]
    a = Ensemble(spec, n_split=2)
    a.step()
    a.step()
    torch.cuda.synchronize()
    b = Ensemble(spec, n_split=2)
    b.step()
    graph = b.capture()
    graph.replay()
    torch.cuda.synchronize()
    for ma, mb in zip(a.members, b.members):
        for name in ("delp", "pt", "u", "v", "w", "delz"):
            x, y = getattr(ma.state, name).cpu().numpy(), getattr(mb.state, name).cpu().numpy()
            np.testing.assert_array_equal(np.nan_to_num(x, nan=7.0), np.nan_to_num(y, nan=7.0), err_msg=name)
    del graph
    a.close()
    b.close()


@pytest.mark.gpu
def test_streamed_round_trips_match_sequential_calls():
    """StreamedAcoustics overlaps the copies of one state with the call on
    another; each host state must come back exactly as from a plain
    copy-in / call / copy-out.  Both runs start from a fresh context and make
    the same calls in the same order: like the reference's, the driver's
    heat_source temporary accumulates over calls, so a call's pt depends on
    every call before it."""
    import types

    import torch

    import gpu_runs
    from fv3core_b200 import _lib
    from fv3core_b200.pipeline import StreamedAcoustics

    fields = cases.ACOUSTIC_STATE
    cases_in = [cases.acoustics_case(12, 8, seed, n_split=2) for seed in (31, 32, 33)]
    gd_a, ad_a, st_a = gpu_runs.make_acoustics(cases_in[0], 12, 8)
    batches, expected = [], []
    for case in cases_in:
        host_in = {}
        for k in fields:
            a = case[k]
            t = torch.from_numpy(np.ascontiguousarray(a.transpose(0, 3, 2, 1) if a.ndim == 4 else a.transpose(0, 2, 1)))
            host_in[k] = t.to(getattr(st_a, k).dtype).pin_memory()
        host_out = {k: torch.empty_like(host_in[k]).pin_memory() for k in fields}
        batches.append((host_in, host_out))
        for k in fields:  # sequential: copy in, call, read back
            getattr(st_a, k).copy_(host_in[k])
        ad_a(st_a)
        torch.cuda.synchronize()
        expected.append({k: getattr(st_a, k).cpu().clone() for k in fields})
    gd_a.close()
    gd_b, ad_b, st_b = gpu_runs.make_acoustics(cases_in[0], 12, 8)
    st_b2 = types.SimpleNamespace(**vars(st_b))
    for k in _lib.DYCORE_FIELDS:
        setattr(st_b2, k, getattr(st_b, k).clone())
    streamed = StreamedAcoustics(ad_b, [st_b, st_b2], fields, fields)
    streamed.run(batches)
    streamed.synchronize()
    for (host_in, host_out), exp in zip(batches, expected):
        for k in fields:
            np.testing.assert_array_equal(np.nan_to_num(host_out[k].numpy(), nan=7.0),
                                          np.nan_to_num(exp[k].numpy(), nan=7.0), err_msg=k)
    gd_b.close()
