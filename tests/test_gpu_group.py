"""Serving groups (dfdm_group_*): one grouped launch per kernel family for several cases.

A member's result does not depend on the other members: the same case steps bit-identically in a group of one and
in any mix, on any stream.  Against the member's own per-context steps it agrees to FP32 rounding (the grouped kernels
are a separate compilation of the per-case kernels' source, whose scalar multiply-add contractions may differ), and
against the oracle at the FP32 parity bar."""
import os
import sys

import numpy as np
import pytest

from dfdm import cases, serve
from dfdm.native import DfdmError, Group, Solver

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (kind, N, Re, seed): Taylor-Green (periodic y: column transforms in y) and channels (walls: y solve, constant flux)
MIX = [("tgv", 32, 800.0, 3), ("chan", 48, 0.0, 5), ("tgv", 64, 1600.0, 7), ("chan", 32, 0.0, 11),
       ("tgv", 48, 2400.0, 13), ("chan", 64, 0.0, 17), ("tgv", 32, 1200.0, 19)]

GROUP_MAX = 24   # jobs per grouped launch (kernels_group.cuh)
BRANCH_CELLS = 512 * 1024   # default cells per graph branch (dfdm_group_set_branch_cells)


def _first_step(case, stream=None):
    s = Solver(case, "fp32", stream=stream)
    s.set_state(*cases.initial_condition(case))
    s.compute_time_step_RK3(1)
    return s


def _expected_launches(solvers):
    """Kernels of one group step.  The members fall into shape classes (stage-kernel form, Nx, Nz, periodic Ny), split
    into branches of consecutive members of at most BRANCH_CELLS cells; per branch and RK stage: the stage kernel, the
    forward and the inverse x transform, the forward and the inverse z transform, the y solve (walls) or the
    periodic-y transform; per branch the stage-3 correction and, for its constant-flux cases, the bulk sum, its
    reduction and the shift.  Each takes one launch per GROUP_MAX jobs."""
    from collections import defaultdict
    up = lambda n: -(-n // GROUP_MAX)
    classes = defaultdict(list)
    for s in solvers:
        per = s.case.ny if s.case.y_bc_type == 0 else -1
        classes[(1 if s.stage_variant()[0] else 0, s.case.nx, s.case.nz, per)].append(s)
    branches = []
    for members in classes.values():
        cur, cells = [], 0
        for s in members:
            if cur and cells + s.case.n_cells > BRANCH_CELLS:
                branches.append(cur)
                cur, cells = [], 0
            cur.append(s)
            cells += s.case.n_cells
        branches.append(cur)
    total = 0
    for members in branches:
        n = len(members)
        flux = sum(s.case.flow_forcing_mode == 1 for s in members)
        total += 3 * 6 * up(n) + up(n) + 3 * up(flux)
    return total


def _grouped(cs, k):
    """States of the cases after a first step each and k group steps; the group's launch count and its expected
    value."""
    ss = [_first_step(c) for c in cs]
    with Group(ss) as g:
        g.step(k)
        launched = g.launch_count()
    out = [s.get_state() for s in ss]
    expected = k * _expected_launches(ss)
    for s in ss:
        s.close()
    return out, launched, expected


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.parametrize("k", [1, 4])
def test_group_steps_match_steps_alone(k):
    """Seven cases of three sizes: the grouped launch count, and each member against its own per-context steps
    (relative L2 at FP32 rounding)."""
    cs = [serve.serve_case(kind, N, Re, seed) for kind, N, Re, seed in MIX]
    alone, per_case, t_alone = [], [], []
    for c in cs:
        s = _first_step(c)
        before = s.launch_count()
        s.compute_time_step_RK3(k)
        per_case.append(s.launch_count() - before)
        alone.append(s.get_state())
        t_alone.append(s.t)
        s.close()
    ss = [_first_step(c) for c in cs]
    with Group(ss) as g:
        g.step(k)
        launched = g.launch_count()
    assert launched == k * _expected_launches(ss)
    assert launched < sum(per_case)   # 6 shape classes: 123 launches a step against 142 alone
    for c, a, s, ta in zip(cs, alone, ss, t_alone):
        for name, x, y in zip("UVWP", a, s.get_state()):
            # P = phi / (dt c3) carries the rounding of the Poisson solve amplified by 1/dt
            assert _rel(y, x) <= (1e-5 if name == "P" else 2e-6), (c.name, name, _rel(y, x))
        assert s.t == ta
        s.close()


def test_results_do_not_depend_on_the_group():
    """Each case in a group of one, and in the group of seven in reverse order: bit-identical states."""
    cs = [serve.serve_case(kind, N, Re, seed) for kind, N, Re, seed in MIX]
    mixed, launched, expected = _grouped(cs[::-1], 3)
    assert launched == expected
    mixed = mixed[::-1]
    for c, m in zip(cs, mixed):
        one, _, _ = _grouped([c], 3)
        for x, y in zip(one[0], m):
            assert np.array_equal(x, y), c.name


def test_group_on_its_own_stream_orders_with_the_members_streams():
    """Members on their own streams, the group on a third: the members' transfers before and after the group's steps
    need no host synchronisation, and a member's own steps continue from the group's state."""
    import torch
    streams = [torch.cuda.Stream() for _ in range(3)]
    cs = [serve.serve_case("tgv", 48, 1000.0, 23), serve.serve_case("chan", 64, 0.0, 29)]
    ref, _, _ = _grouped(cs, 3)
    ss = [_first_step(c, st.cuda_stream) for c, st in zip(cs, streams)]
    g = Group(ss, stream=streams[2].cuda_stream)
    g.step_async(3)
    for s, r in zip(ss, ref):
        for x, y in zip(s.get_state(), r):
            assert np.array_equal(x, y)
    # per-context step, group step, per-context step: against reference contexts taking the same sequence
    refs = [_first_step(c) for c in cs]
    with Group(refs) as gr:
        gr.step(3)
        for s in refs:
            s.compute_time_step_RK3(1)
        gr.step(1)
        for s in refs:
            s.compute_time_step_RK3(1)
    for s in ss:
        s.compute_time_step_RK3_async(1)
    g.step_async(1)
    for s in ss:
        s.compute_time_step_RK3_async(1)
    for s, r in zip(ss, refs):
        for x, y in zip(s.get_state(), r.get_state()):
            assert np.array_equal(x, y)
    g.close()
    for s in ss + refs:
        s.close()


def test_more_members_than_one_job_table():
    """Thirty members, one job table each, in two shape classes of 15; each is bit-identical to its group of one."""
    cs = [serve.serve_case("tgv" if q % 2 else "chan", 32, 900.0 + 50 * q, 100 + q) for q in range(30)]
    big, launched, expected = _grouped(cs, 2)
    assert launched == expected and launched <= 2 * 2 * (19 * 1 + 3)   # two branches of 15 (491,520 cells each)
    for c, b in zip(cs, big):
        one, _, _ = _grouped([c], 2)
        for x, y in zip(one[0], b):
            assert np.array_equal(x, y)


def test_grouped_channel_matches_the_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    c = serve.serve_case("chan", 32, 0.0, 31)
    t = serve.serve_case("tgv", 32, 1600.0, 37)
    o = oracle.Oracle(c)
    o.set_state(*cases.initial_condition(c))
    o.step(5)
    members = [_first_step(c), _first_step(t)]
    with Group(members) as g:
        g.step(4)
    got = members[0].get_state()
    for a, b in zip(got, o.get_state()):
        assert _rel(a, b) <= 1e-5, _rel(a, b)
    for s in members:
        s.close()


def test_ineligible_members_are_refused():
    c = serve.serve_case("tgv", 32, 800.0, 41)
    s64 = Solver(c, "fp64")
    s64.set_state(*cases.initial_condition(c))
    s64.compute_time_step_RK3(1)
    with pytest.raises(DfdmError) as e:
        Group([s64])
    assert e.value.code != 0
    fresh = Solver(c, "fp32")
    fresh.set_state(*cases.initial_condition(c))
    with pytest.raises(DfdmError):
        Group([fresh])   # no first step yet
    les = Solver(cases.chan_les_amd_small(), "fp32")
    les.set_state(*cases.initial_condition(cases.chan_les_amd_small()))
    les.compute_time_step_RK3(1)
    with pytest.raises(DfdmError):
        Group([les])
    fresh.compute_time_step_RK3(1)
    with pytest.raises(DfdmError):
        Group([fresh, fresh])
    for s in (s64, fresh, les):
        s.close()


def test_branch_splitting_leaves_results_unchanged():
    """A class of eight 64^3 cases stepped as one branch, as branches of at most 2^19 cells (two cases) and as one
    branch per case: bit-identical states, and the launch counts of the branch model."""
    cs = [serve.serve_case("tgv", 64, 1000.0 + 100 * q, 200 + q) for q in range(8)]
    ref = None
    for cells, nbranch in [(0, 1), (1 << 19, 4), (1, 8)]:
        ss = [_first_step(c) for c in cs]
        with Group(ss) as g:
            g.set_branch_cells(cells)
            before = g.launch_count()
            g.step(2)
            assert g.launch_count() - before == 2 * nbranch * (3 * 6 + 1)
        st = [s.get_state() for s in ss]
        for s in ss:
            s.close()
        if ref is None:
            ref = st
        for a, b in zip(st, ref):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


def test_stage_tile_shapes_leave_results_unchanged():
    """The grouped stage launches with each member's own z-chunk, with 4 planes per block, with one chunk per column,
    each with one block per tile and with resident blocks walking the tiles (more tiles than resident blocks at 4
    planes), and with the group's timed choice: bit-identical states."""
    cs = [serve.serve_case("tgv" if q % 2 else "chan", 48, 1000.0 + 10 * q, 300 + q) for q in range(6)]
    ref = None
    for kc, walk in [(-1, False), (0, False), (4, False), (4, True), (0, True), (1000, True)]:
        ss = [_first_step(c) for c in cs]
        with Group(ss) as g:
            g.set_stage_tiles(kc, walk)
            g.step(3)
        st = [s.get_state() for s in ss]
        for s in ss:
            s.close()
        if ref is None:
            ref = st
        for a, b in zip(st, ref):
            for x, y in zip(a, b):
                assert np.array_equal(x, y), (kc, walk)
