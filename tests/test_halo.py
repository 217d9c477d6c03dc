"""The domain-and-halo form of the hydro pass (gizmo_b200/halo.py) on two and
three ``gloo`` ranks on the CPU, each rank computing its share with the oracle in
place of its GPU: the outputs of every particle equal those of a one-domain
pass, bit for bit, except the MFV dMass, whose sum collects the j-side terms
of other ranks in another order (within 1e-14 of its largest value). One run
starts from converged kernel lengths, the other from seeds so small that the
first halo is too thin and the pass is redone deeper; with three ranks a cell
is imported by both others and its dMass collects j-side terms from both."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT_FIELDS = ("h", "num_ngb", "drkern", "divvel", "rho", "pressure", "nvt", "cond", "fce", "pvel", "grad_rho",
              "grad_p", "grad_v", "accel", "dudt", "vsig", "dtmass", "dmass", "gravwork", "iters")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload(h=None):
    from gizmo_b200 import ics
    from gizmo_b200.abi import METHOD_MFV
    wl = ics.sedov(36, seed=3)
    wl.params.method = METHOD_MFV
    wl.params.des_num_ngb = 16.0
    wl.h = wl.h * (16.0 / 32.0) ** (1.0 / 3.0) if h is None else h.copy()
    return wl


def _oracle_engine(params, local, dens, grad, force):
    from oracle import oracle as O
    st = O.new_state(len(local["mass"]), local)
    orc = O.Oracle(params, "port", n_threads=1)
    assert orc.density(st, dens) == 0
    h_iter_max = orc.density_h_iter_max()
    assert orc.gradients(st, grad) == 0
    assert orc.force(st, force) == 0
    out = {k: st[k] for k in OUT_FIELDS}
    out["h_iter_max"] = h_iter_max
    return out


class _FirstIterationTooLong:
    """The oracle engine, except that its first call reports a density iteration
    that took sums at ten times the largest seed: beyond twice any halo depth
    the pass could have used, so that attempt must be thrown away."""

    def __init__(self):
        self.calls = 0

    def __call__(self, params, local, dens, grad, force):
        out = _oracle_engine(params, local, dens, grad, force)
        if self.calls == 0:
            out["h_iter_max"] = 10.0 * float(np.max(local["h"]))
        self.calls += 1
        return out


def _rank(rank, world, port, h, q, engine_kind="oracle"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    from gizmo_b200 import halo
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        wl = _workload(h)
        inputs = wl.inputs()
        owner = halo.domain_owner(inputs["pos"], wl.params.box_size, world)
        gid = np.nonzero(owner == rank)[0]
        mine = {k: np.asarray(v)[gid] for k, v in inputs.items()}
        if engine_kind == "gpu":
            engine = halo.hydro_pass_engine(0)
        else:
            engine = _oracle_engine if engine_kind == "oracle" else _FirstIterationTooLong()
        hp = halo.HaloPass(wl.params, halo.Exchange(rank, world), engine)
        out = hp(gid, mine)
        q.put((rank, gid, out, hp.last_radius, hp.last_imported, hp.last_h_iter_max))
    finally:
        dist.destroy_process_group()


def _run_ranks(h, world=2, engine_kind="oracle"):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, h, q, engine_kind)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    return got


@pytest.mark.parametrize("seed_scale,world", [(None, 2), (0.6, 2), (None, 3)],
                         ids=["converged-seeds", "thin-first-halo", "three-domains"])
def test_domains_equal_one_domain(seed_scale, world):
    from oracle import oracle as O
    wl = _workload()
    st = O.new_state(wl.n, wl.inputs())
    assert O.Oracle(wl.params, "port").density(st) == 0
    # converged lengths (as a step after the first starts from), or seeds so small
    # that the halo built from them is too thin and the pass is redone deeper
    wl.h = st["h"].copy() if seed_scale is None else st["h"] * seed_scale
    ref = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(ref) == 0 and orc.gradients(ref) == 0 and orc.force(ref) == 0
    got = _run_ranks(wl.h, world)
    covered = np.zeros(wl.n, dtype=int)
    for rank, gid, out, radius, imported, h_iter_max in got:
        covered[gid] += 1
        assert imported < wl.n - len(gid)  # the halo left part of the other domains out
        assert h_iter_max <= radius / 2  # no density sum was taken beyond 2H
        if seed_scale is not None:  # the first halo (4 x 1.1 x the largest seed) was redone deeper
            assert radius > 4.0 * 1.1 * wl.h.max() * 1.2
        for f in OUT_FIELDS:
            a, b = np.asarray(out[f]), np.asarray(ref[f])[gid]
            if f == "dmass":
                np.testing.assert_allclose(a, b, rtol=0, atol=1e-14 * np.abs(ref[f]).max())
            else:
                assert np.array_equal(a, b), (rank, f)
    assert (covered == 1).all()


def test_long_intermediate_kernel_length_redoes_the_pass():
    """A density iteration that took sums beyond twice the halo depth H (here
    reported by the engine's first call) is thrown away and the pass redone with
    a deeper halo, although every converged kernel length stayed below H."""
    from oracle import oracle as O
    wl = _workload()
    st = O.new_state(wl.n, wl.inputs())
    assert O.Oracle(wl.params, "port").density(st) == 0
    wl.h = st["h"].copy()
    ref = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(ref) == 0 and orc.gradients(ref) == 0 and orc.force(ref) == 0
    got = _run_ranks(wl.h, 2, engine_kind="first-too-long")
    for rank, gid, out, radius, imported, h_iter_max in got:
        assert radius > 4.0 * 1.1 * wl.h.max() * 1.2  # redone deeper
        for f in OUT_FIELDS:
            a, b = np.asarray(out[f]), np.asarray(ref[f])[gid]
            if f == "dmass":
                np.testing.assert_allclose(a, b, rtol=0, atol=1e-14 * np.abs(ref[f]).max())
            else:
                assert np.array_equal(a, b), (rank, f)


@pytest.mark.gpu
def test_domains_on_the_gpu_engine_equal_one_domain():
    """The GPU engine (hydro_pass_engine: a HydroPass per rank over the C ABI,
    density / gradients / force on the rank's active lists) in two gloo ranks
    that share one GPU: the ranks exchange on the host, so no kernel of one
    waits on the other's. Against one GPU pass over the whole set, FP64 form:
    the parity tolerances of tests/test_gpu_parity.py (the active lists change
    the lanes per row, so the sums run in another order)."""
    from gizmo_b200.hydro import HydroPass
    from tests._util import DENSITY_FIELDS, FORCE_FIELDS, GRADIENT_FIELDS, field_err
    wl = _workload()
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.density()
        wl.h = hp.download(["h"])["h"].copy()  # converged lengths, as a step after the first starts from
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        ref = hp.download()
    got = _run_ranks(wl.h, 2, engine_kind="gpu")
    covered = np.zeros(wl.n, dtype=int)
    for rank, gid, out, radius, imported, h_iter_max in got:
        covered[gid] += 1
        assert imported < wl.n - len(gid)
        assert h_iter_max <= radius / 2
        h_rel = np.abs(np.asarray(out["h"]) - ref["h"][gid]) / ref["h"][gid]
        same = (np.asarray(out["iters"]) == ref["iters"][gid]) & (h_rel <= 1e-10)
        assert same.mean() >= 0.999 and h_rel.max() <= 3e-3, (same.mean(), h_rel.max())
        keep = np.flatnonzero(same)
        for f in DENSITY_FIELDS + GRADIENT_FIELDS:
            assert field_err(f, np.asarray(out[f])[keep], ref[f][gid][keep], 1e-6) < 1e-10, (rank, f)
        if same.all():
            for f in FORCE_FIELDS:
                if f == "dmass":
                    continue
                assert field_err(f, np.asarray(out[f]), ref[f][gid], 1e-3) < 1e-10, (rank, f)
            np.testing.assert_allclose(np.asarray(out["dmass"]), ref["dmass"][gid], rtol=0,
                                       atol=1e-12 * np.abs(ref["dmass"]).max())
    assert (covered == 1).all()
