"""Batched ensembles: members of one resolution kept in one batched context
(fv3b_ctx_create_batched, 6 x members tile slots), so that every kernel of a
stage advances all of them in one launch.  A batched member must come out
exactly as the same member run alone in its own context; halo updates must
stay within a member."""
import numpy as np
import pytest

from fv3core_b200 import _lib

FIELDS = ("delp", "pt", "u", "v", "w", "delz", "pe", "pk", "peln", "q_con", "pkz", "omga", "uc", "vc")


def _nan7(a):
    return np.nan_to_num(a, nan=7.0)


def test_batched_halo_neighbours_stay_in_the_member(tmp_path):
    """The CUDA halo map's tile connectivity (csrc/halo.cuh, compiled for the
    host) for 24 tile slots, four batched cubes: every neighbour of slot t
    is a tile of t's own cube, and the map of member m is member 0's
    shifted by 6m."""
    import os
    import shutil
    import subprocess

    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "dump")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-o", exe, os.path.join(root, "tests", "native",
                                                                                  "halo_dump.cpp")])
    rows = {}
    for line in subprocess.check_output([exe, "12", "edges"], text=True).split("\n"):
        if line:
            _, t, edge, t2, e2, rev = line.split()
            rows[(int(t), int(edge))] = (int(t2), int(e2), int(rev))
    assert len(rows) == 96
    for (t, edge), (t2, e2, rev) in rows.items():
        base = t - t % 6
        t20, e20, rev0 = rows[(t % 6, edge)]
        assert (t2, e2, rev) == (base + t20, e20, rev0), (t, edge)
        assert base <= t2 < base + 6


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_batched_members_match_runs_alone(precision):
    """Three C12 L16 members (seeds 1, 2, 3) in one batched context against
    each member in its own context: two AcousticDynamics calls, every field
    bit for bit on the full storage (the mixed build too: the same kernels
    on the same numbers)."""
    import torch

    from fv3core_b200.ensemble import Member, MemberGroup

    seeds = (1, 2, 3)
    group = MemberGroup(12, 16, seeds, precision=precision, n_split=2)
    alone = [Member(12, 16, s, precision=precision, n_split=2) for s in seeds]
    try:
        for _ in range(2):
            group.step()
            for m in alone:
                m.step()
        torch.cuda.synchronize()
        for q, m in enumerate(alone):
            for name in FIELDS:
                x = group.member_field(name, q).cpu().numpy()
                y = getattr(m.state, name).cpu().numpy()
                np.testing.assert_array_equal(_nan7(x), _nan7(y), err_msg=f"member {q} {name}")
    finally:
        group.close()
        for m in alone:
            m.close()


@pytest.mark.gpu
def test_mixed_resolution_ensemble_batched_matches_unbatched():
    """An ensemble at two resolutions (three C12 L8 members and two C16 L6
    members): the batched form (one context and one launch per kernel per
    resolution) against one context per member, one graph-captured step
    each, bit for bit; the batched step issues fewer launches."""
    import torch

    from fv3core_b200.ensemble import Ensemble

    spec = [(12, 8, 1), (16, 6, 2), (12, 8, 3), (12, 8, 4), (16, 6, 5)]
    a = Ensemble(spec, n_split=2, batched=True)
    b = Ensemble(spec, n_split=2, batched=False)
    try:
        l0 = _lib.launch_count()
        a.step()
        la = _lib.launch_count() - l0
        l0 = _lib.launch_count()
        b.step()
        lb = _lib.launch_count() - l0
        torch.cuda.synchronize()
        assert len(a.members) == 2 and len(b.members) == 5
        assert la * 2 < lb, (la, lb)
        groups = {(g.n, g.npz): g for g in a.members}
        counters = {}
        for mb in b.members:
            g = groups[(mb.n, mb.npz)]
            q = counters.get((mb.n, mb.npz), 0)
            counters[(mb.n, mb.npz)] = q + 1
            assert g.seeds[q] == mb.seed
            for name in FIELDS:
                x = g.member_field(name, q).cpu().numpy()
                y = getattr(mb.state, name).cpu().numpy()
                np.testing.assert_array_equal(_nan7(x), _nan7(y), err_msg=f"{mb.n} seed {mb.seed} {name}")
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_batched_dynamical_core_step_matches_runs_alone():
    """The whole step_dynamics on a batched context of two C12 L12 members
    against each member alone (tracer advection, remapping with the
    saturation adjustment, the step's epilogue): every field bit for bit on
    the compute domain."""
    import sys
    import os

    import torch

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import cases
    from fv3core_b200.config import DynamicalCoreConfig
    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.fv_dynamics import DynamicalCore
    from fv3core_b200.storage import to_device

    n, nz = 12, 12
    cs = [cases.step_case(n, nz, seed, 2, sat_adj=True) for seed in (201, 202)]
    names = [k for k in tuple(cases.ACOUSTIC_STATE) + cases.STEP_TRACERS + ("ps",) if k != "phis"]
    config = DynamicalCoreConfig(**cases.dycore_namelist(n, nz, 2, True))

    def run(members_cases):
        gd = GridData(cases.grid_for(n), nz, members=len(members_cases))
        try:
            sf = StencilFactory(StencilConfig(), gd.grid_indexing)
            cat = {k: np.concatenate([c[k] for c in members_cases], axis=0) for k in names + ["phis"]}
            phis = to_device(cat["phis"])
            core = DynamicalCore(None, gd, sf, gd, config, cs[0]["ak"], cs[0]["bk"], phis)
            state = {k: to_device(cat[k]) for k in names}
            state["phis"] = phis
            core.step_dynamics(state, False, False, 225.0, cs[0]["ptop"], 2, cs[0]["ks"])
            torch.cuda.synchronize()
            return {k: v.cpu().numpy() for k, v in state.items()}
        finally:
            gd.close()

    both = run(cs)
    h = 3
    for q, c in enumerate(cs):
        alone = run([c])
        for k in ("u", "v", "w", "delp", "pt", "delz", "qvapor", "qliquid", "qcld", "pe", "omga", "ua"):
            x = both[k][6 * q:6 * q + 6][:, :nz, h:h + n, h:h + n]
            y = alone[k][:, :nz, h:h + n, h:h + n]
            np.testing.assert_array_equal(_nan7(x), _nan7(y), err_msg=f"member {q} {k}")
