"""One particle set on several GPUs: spatial domains and one halo exchange per
hydro pass, with the reverse writeback of the MFV j-side mass fluxes.

This mirrors what the reference's ghost import and writeback do around its
neighbour loops: each rank owns the particles of one domain, imports copies of
the other ranks' particles near it, computes, and sends back what its
computation wrote into those copies. Here the exchange happens once per pass,
before density, instead of once per loop:

  * domains are contiguous ranges of Morton keys with equal particle counts,
    so a domain is spatially compact; it is described by the boxes of its
    particles in each occupied top-level Morton cell (4 x 4 x 4), which stay
    tight for any number of ranks;
  * a rank imports every particle within 4H of its own domain boxes (periodic),
    where H bounds every kernel length the pass produces. That is deep enough
    to compute, redundantly, everything its own particles read: density runs on
    own particles and on imports within 2H of the box, gradients on own
    particles and imports within H, force on own particles only. A force
    neighbour lies within H of an own particle, its gradient neighbours within
    2H, and their density neighbours within 3H. The last H leaves room for the
    kernel-length iteration: a density-active particle sees every particle
    within 2H of it, so an intermediate kernel length may reach twice the
    converged bound. The iteration can grow h by up to exp(1.631) per step
    from a seed far too small (density_loop.h:864-947), so the engine reports
    the largest kernel length at which the density iteration took sums, and a
    pass in which it exceeded 2H is redone deeper (below): no sum is ever taken
    over a halo that was too thin;
  * after the pass, the j-side dMass that own force targets wrote into
    imported copies (the MFV mass flux, hydro_functions.h:513-544) goes back to
    the owners, who add it to their own;
  * if a converged kernel length came out above H, or an intermediate one of
    the density iteration above 2H, the pass is redone with a larger H (the
    same on every rank), so the result never depends on a halo that was too
    thin.

Each rank keeps its own and imported particles in global-index order, so every
neighbour row, and with it every sum, has the order of a one-domain run.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

INPUT_FIELDS = (("pos", 3), ("vel", 3), ("mass", 1), ("u", 1), ("dt", 1), ("h", 1), ("cond", 1))
N_INPUT = sum(k for _, k in INPUT_FIELDS)


def morton_keys(pos: np.ndarray, box: float, bits: int = 21) -> np.ndarray:
    """63-bit Morton keys of positions in [0, box)^3, x in the highest bit of each triple."""
    q = np.clip((pos / box * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1).astype(np.uint64)
    key = np.zeros(len(pos), dtype=np.uint64)
    for b in range(bits - 1, -1, -1):
        for a in range(3):
            key = (key << np.uint64(1)) | ((q[:, a] >> np.uint64(b)) & np.uint64(1))
    return key


def domain_owner(pos: np.ndarray, box: float, world: int) -> np.ndarray:
    """Rank owning each particle: equal-count contiguous ranges of Morton keys
    (ties by particle index)."""
    order = np.lexsort((np.arange(len(pos)), morton_keys(pos, box)))
    owner = np.empty(len(pos), dtype=np.int64)
    owner[order] = (np.arange(len(pos)) * world) // max(len(pos), 1)
    return owner


def box_distance(x: np.ndarray, lo: np.ndarray, hi: np.ndarray, box: float) -> np.ndarray:
    """Distance of each point to the axis-aligned box [lo, hi] in a periodic cube of side `box`."""
    d2 = np.zeros(len(x))
    for a in range(3):
        best = None
        for shift in (-box, 0.0, box):
            xa = x[:, a] + shift
            d = np.maximum(np.maximum(lo[a] - xa, xa - hi[a]), 0.0)
            best = d if best is None else np.minimum(best, d)
        d2 += best * best
    return np.sqrt(d2)


N_DOMAIN_BOXES = 64  # top two Morton levels: a domain is described by up to 64 boxes


def domain_boxes(pos: np.ndarray, box: float) -> np.ndarray:
    """[N_DOMAIN_BOXES, 6] boxes (lo, hi) of the particles in each occupied top-level Morton
    cell (4 x 4 x 4); unused rows are empty (lo = +inf, hi = -inf). Their union holds
    every particle, so a distance to it never exceeds the distance to the nearest particle."""
    out = np.empty((N_DOMAIN_BOXES, 6))
    out[:, :3], out[:, 3:] = np.inf, -np.inf
    if not len(pos):
        return out
    cell = (morton_keys(pos, box) >> np.uint64(63 - 6)).astype(np.int64)
    for c in np.unique(cell):
        sel = pos[cell == c]
        out[c, :3], out[c, 3:] = sel.min(0), sel.max(0)
    return out


def boxes_distance(x: np.ndarray, boxes: np.ndarray, box: float) -> np.ndarray:
    """Distance of each point to the union of boxes (rows lo, hi) in a periodic cube."""
    d = np.full(len(x), np.inf)
    for b in boxes:
        if np.isfinite(b[0]):
            d = np.minimum(d, box_distance(x, b[:3], b[3:], box))
    return d


def pack(inputs: dict, idx: np.ndarray) -> np.ndarray:
    """Rows idx of the input fields as one [m, N_INPUT] float64 array."""
    cols = [np.asarray(inputs[name], dtype=np.float64).reshape(len(inputs["mass"]), k)[idx] for name, k in INPUT_FIELDS]
    return np.concatenate(cols, axis=1) if len(idx) else np.zeros((0, N_INPUT))


def unpack(rows: np.ndarray) -> dict:
    out, c = {}, 0
    for name, k in INPUT_FIELDS:
        v = rows[:, c:c + k]
        out[name] = v.copy() if k == 3 else v[:, 0].copy()
        c += k
    return out


@dataclass
class Exchange:
    """Point-to-point transfers between the ranks of a process group
    (torch.distributed: NCCL on GPUs, gloo on the CPU)."""
    rank: int
    world: int
    device: str = "cpu"

    def _dist(self):
        import torch.distributed as dist
        return dist

    def all_max(self, x: float) -> float:
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self._dist().all_reduce(t, op=self._dist().ReduceOp.MAX)
        return float(t.item())

    def all_gather_rows(self, row: np.ndarray) -> np.ndarray:
        import torch
        t = torch.as_tensor(np.ascontiguousarray(row, dtype=np.float64), device=self.device)
        out = [torch.empty_like(t) for _ in range(self.world)]
        self._dist().all_gather(out, t)
        return np.stack([o.cpu().numpy() for o in out])

    def swap(self, send: list) -> list:
        """send[r]: a float64 array [m_r, k] for rank r (k the same everywhere); returns what every rank sent here."""
        import torch
        dist = self._dist()
        k = next((a.shape[1] for a in send if a.ndim == 2), 1)
        counts = torch.tensor([len(a) for a in send], dtype=torch.int64, device=self.device)
        got = [torch.zeros(self.world, dtype=torch.int64, device=self.device) for _ in range(self.world)]
        dist.all_gather(got, counts)
        incoming = [int(got[r][self.rank]) for r in range(self.world)]
        reqs, recv = [], [None] * self.world
        for r in range(self.world):
            if r == self.rank:
                continue
            recv[r] = torch.empty((incoming[r], k), dtype=torch.float64, device=self.device)
            if incoming[r]:
                reqs.append(dist.irecv(recv[r], src=r))
            if len(send[r]):
                reqs.append(dist.isend(torch.as_tensor(np.ascontiguousarray(send[r], dtype=np.float64).reshape(-1, k),
                                                       device=self.device), dst=r))
        for q in reqs:
            q.wait()
        return [np.zeros((0, k)) if r == self.rank else recv[r].cpu().numpy() for r in range(self.world)]


class HaloPass:
    """One hydro pass over a particle set split into domains across ranks.

    ``engine(params, local_inputs, density_active, gradient_active, force_active)``
    computes the pass on one rank's own and imported particles and returns the
    output fields (``HydroPass`` names) for all of them, plus ``h_iter_max``:
    the largest kernel length at which its density iteration took sums;
    ``hydro_pass_engine`` below is the one that runs on the GPU. ``__call__`` takes this rank's own
    particles (their global indices and input fields) and returns the outputs of
    those particles, equal to what a one-domain pass gives them.
    """

    def __init__(self, params, exchange: Exchange, engine, h_margin: float = 1.1, h_growth: float = 1.26,
                 max_tries: int = 6):
        self.params = params
        self.ex = exchange
        self.engine = engine
        self.h_margin = h_margin
        self.h_growth = h_growth
        self.max_tries = max_tries
        self.last_radius = None
        self.last_imported = None
        self.last_h_iter_max = None

    def __call__(self, gid: np.ndarray, inputs: dict) -> dict:
        box = float(self.params.box_size)
        pos = np.asarray(inputs["pos"], dtype=np.float64).reshape(-1, 3)
        n_own = len(gid)
        mine = domain_boxes(pos, box)
        boxes = self.ex.all_gather_rows(mine.ravel()).reshape(self.ex.world, N_DOMAIN_BOXES, 6)
        H = self.ex.all_max(float(np.max(inputs["h"])) if n_own else 0.0) * self.h_margin
        for _ in range(self.max_tries):
            out, h_max, h_iter_max = self._attempt(gid, inputs, pos, mine, boxes, H, box)
            # every rank takes both reductions, in the same order
            h_max, h_iter_max = self.ex.all_max(h_max), self.ex.all_max(h_iter_max)
            self.last_h_iter_max = h_iter_max
            if h_max <= H and h_iter_max <= 2.0 * H:
                return out
            H *= self.h_growth
        raise RuntimeError(f"halo pass: kernel lengths still above the halo depth after {self.max_tries} tries")

    def _attempt(self, gid, inputs, pos, mine, boxes, H, box):
        ex = self.ex
        # own particles each other rank needs: within 4H of its domain box
        send = []
        for r in range(ex.world):
            if r == ex.rank or not len(gid):
                send.append(np.zeros((0, N_INPUT + 1)))
                continue
            near = np.nonzero(boxes_distance(pos, boxes[r], box) < 4.0 * H)[0]
            send.append(np.concatenate([gid[near, None].astype(np.float64), pack(inputs, near)], axis=1))
        got = ex.swap(send)
        imported = np.concatenate([g for g in got], axis=0) if any(len(g) for g in got) else np.zeros((0, N_INPUT + 1))
        src = np.concatenate([np.full(len(g), r) for r, g in enumerate(got)]) if len(imported) else np.zeros(0, int)
        # local set in global-index order
        all_gid = np.concatenate([gid.astype(np.int64), imported[:, 0].astype(np.int64)])
        order = np.argsort(all_gid, kind="stable")
        rows = np.concatenate([pack(inputs, np.arange(len(gid))), imported[:, 1:]], axis=0)[order]
        local = unpack(rows)
        is_own = (order < len(gid))
        owner = np.where(is_own, ex.rank, np.concatenate([np.full(len(gid), ex.rank), src])[order])
        d = boxes_distance(local["pos"], mine, box)
        d = np.where(is_own, 0.0, d)
        dens = np.nonzero(d < 2.0 * H)[0].astype(np.int32)
        grad = np.nonzero(d < H)[0].astype(np.int32)
        force = np.nonzero(is_own)[0].astype(np.int32)
        out = dict(self.engine(self.params, local, dens, grad, force))
        h_iter_max = float(out.pop("h_iter_max"))
        h_max = float(np.max(out["h"][dens])) if len(dens) else 0.0
        # reverse writeback: the j-side dMass own targets wrote into imported copies
        back = []
        gid_local = all_gid[order]
        for r in range(ex.world):
            sel = np.nonzero((owner == r) & ~is_own)[0] if r != ex.rank else np.zeros(0, int)
            back.append(np.stack([gid_local[sel].astype(np.float64), out["dmass"][sel]], axis=1)
                        if len(sel) else np.zeros((0, 2)))
        returned = ex.swap(back)
        own_local = np.nonzero(is_own)[0]  # own particles in global-index order
        own_rank = np.argsort(order[own_local], kind="stable")
        own_rows = own_local[own_rank]  # local row of each own particle, in the caller's order
        result = {k: np.asarray(v)[own_rows].copy() for k, v in out.items()}
        back_rows = np.concatenate(returned, axis=0) if any(len(r) for r in returned) else np.zeros((0, 2))
        if len(back_rows):
            by_gid = np.argsort(gid, kind="stable")
            at = by_gid[np.searchsorted(gid[by_gid], back_rows[:, 0].astype(np.int64))]
            np.add.at(result["dmass"], at, back_rows[:, 1])
        self.last_radius = 4.0 * H
        self.last_imported = len(imported)
        return result, h_max, h_iter_max


def hydro_pass_engine(device: int = 0):
    """The engine that runs a rank's share on its GPU through the C ABI."""
    from .hydro import HydroPass

    def run(params, local, dens, grad, force):
        with HydroPass(params, device=device) as hp:
            hp.upload(local["pos"], local["vel"], local["mass"], local["u"], local["dt"], local["h"], local["cond"])
            hp.density(dens)
            h_iter_max = hp.status()["h_iter_max"]
            hp.hydro_gradient_calc(grad)
            hp.hydro_force(force)
            out = hp.download()
            out["h_iter_max"] = h_iter_max
            return out
    return run
