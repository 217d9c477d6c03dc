"""Seeded synthetic particle sets for the hydro pass.

The reference's own problem ICs are downloaded at test time and are not part
of its tree, so these generators stand in for them with the shapes, sizes and
value distributions of the named workloads (all in a unit periodic box, equal
particle masses, numpy ``default_rng`` with the listed seeds):

  sedov         lattice n^3 + U(-0.1, 0.1) spacing jitter, rho = 1, u = 1e-5,
                E = 1 put on the 32 particles nearest the centre with cubic
                spline weights; MFM, gamma 5/3, cubic kernel, 32 neighbours.
  lognormal     positions ~ exp(delta), delta a Gaussian random field with
                P(k) ~ k^-3 scaled to sigma_lnrho; solenoidal Gaussian velocity
                field P(k) ~ k^-4 at rms Mach 2; isothermal u = 1 (gamma 1.0001);
                MFM, Wendland C2, 64 neighbours.
  shock_tube    lattice + U(-0.1, 0.1) spacing jitter; a plane through the box
                centre with a random unit normal splits left and right states,
                rho_L, rho_R ~ U[0.125, 1] (set through the particle masses),
                P_L, P_R ~ U[0.1, 1], at rest; MFM, gamma 5/3, cubic, 32
                neighbours. In the periodic box the plane's image is a second
                discontinuity.
  boxes         a batch of independent boxes of log-uniform sizes, each a
                shock tube or a Sedov blast (E ~ U[0.1, 10]) with equal odds.
  plummer_mix   90% of particles in 1000 Plummer spheres (scale radius
                log-uniform in [0.002, 0.02], truncated at 20a, velocity
                dispersion sqrt(M/sqrt(r^2+a^2)) per axis), 10% uniform
                background at rest; u = 1e-2; MFV, gamma 5/3, cubic, 32 neighbours.

Timesteps are power-of-two bins dt = 2^-k (exact in FP64), assigned from a
Courant-like estimate 0.2 h / c_s of the seed kernel length.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .abi import GzParams, KERNEL_CUBIC, KERNEL_WENDLAND_C2, METHOD_MFM, METHOD_MFV, PRECISION_FP64

VOLNORM = 4.188790204786  # 4 pi / 3, constants.h:445


@dataclass
class Workload:
    name: str
    params: GzParams
    pos: np.ndarray
    vel: np.ndarray
    mass: np.ndarray
    u: np.ndarray
    dt: np.ndarray
    h: np.ndarray
    cond: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def inputs(self) -> dict:
        return dict(pos=self.pos, vel=self.vel, mass=self.mass, u=self.u, dt=self.dt, h=self.h, cond=self.cond)


def make_params(kernel: int, method: int, gamma: float, des_num_ngb: float, max_num_ngb_dev: float,
                precision: int = PRECISION_FP64, box: float = 1.0, first_step: int = 0,
                selfgravity_off: int = 1, min_kernel_radius: float = 0.0,
                max_kernel_radius: float = 0.25) -> GzParams:
    p = GzParams()
    p.kernel = kernel
    p.method = method
    p.precision = precision
    p.first_step = first_step
    p.selfgravity_off = selfgravity_off
    p.box_size = box
    p.gamma = gamma
    p.des_num_ngb = des_num_ngb
    p.max_num_ngb_dev = max_num_ngb_dev
    p.min_kernel_radius = min_kernel_radius
    p.max_kernel_radius = max_kernel_radius
    return p


def _cubic_w(q: np.ndarray) -> np.ndarray:
    w = np.where(q < 0.5, 1 + 6 * (q - 1) * q * q, 2 * (1 - q) ** 3)
    return np.where(q < 1, w, 0.0)


def _morton21(pos: np.ndarray, box: float) -> np.ndarray:
    """63-bit Morton keys of positions in [0, box) (21 bits per axis)."""
    G = 1 << 21
    c = np.minimum((pos / box * G).astype(np.int64), G - 1).astype(np.uint64)
    key = np.zeros(pos.shape[0], dtype=np.uint64)
    for b in range(21):
        for k in range(3):
            key |= ((c[:, k] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + k)
    return key


def octree_density_h(pos: np.ndarray, des_num_ngb: float, box: float = 1.0) -> np.ndarray:
    """Cold kernel-length seed (3 N_ngb / (4 pi n_local))^(1/3), with n_local the
    particle count over the volume of the smallest octree cell (Morton-key
    prefix) that still holds N_ngb / 4 particles: a dense clump smaller than
    any fixed grid cell still gets a seed of its own size (on the Plummer
    mixture the seed is within [0.46, 3] x the converged h for 98% of
    particles)."""
    n = pos.shape[0]
    key = _morton21(pos, box)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    need = 0.25 * des_num_ngb
    count = np.full(n, float(n))
    level = np.zeros(n, dtype=np.int64)
    for L in range(1, 21):
        pref = ks >> np.uint64(3 * (21 - L))
        starts = np.flatnonzero(np.r_[True, pref[1:] != pref[:-1]])
        lens = np.diff(np.r_[starts, n])
        cnt = np.repeat(lens, lens).astype(np.float64)
        ok = cnt >= need
        if not ok.any():
            break
        count[ok] = cnt[ok]
        level[ok] = L
    nloc = count * (8.0 ** level) / box ** 3
    h = np.empty(n)
    h[order] = (des_num_ngb / (VOLNORM * nloc)) ** (1.0 / 3.0)
    return h


def timestep_bins(h: np.ndarray, cs: np.ndarray, kmin: int = 4, kmax: int = 30) -> np.ndarray:
    est = 0.2 * h / np.maximum(cs, 1e-30)
    k = np.clip(np.ceil(-np.log2(est)), kmin, kmax)
    return np.ldexp(1.0, -k.astype(np.int64))


def sedov(n1: int = 32, seed: int = 1, precision: int = PRECISION_FP64, energy: float = 1.0) -> Workload:
    rng = np.random.default_rng(seed)
    N = n1 ** 3
    s = 1.0 / n1
    g = (np.arange(n1) + 0.5) * s
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pos += rng.uniform(-0.1, 0.1, size=pos.shape) * s
    pos %= 1.0
    mass = np.full(N, 1.0 / N)
    u = np.full(N, 1e-5)
    d = pos - 0.5
    r = np.sqrt((d * d).sum(1))
    order = np.argsort(r, kind="stable")
    near = order[:32]
    h_inj = r[order[32]]
    w = _cubic_w(r[near] / h_inj)
    u[near] += energy * w / (mass[near] * w).sum()
    vel = np.zeros((N, 3))
    params = make_params(KERNEL_CUBIC, METHOD_MFM, 5.0 / 3.0, 32.0, 0.1, precision)
    h = np.full(N, (32.0 / (VOLNORM * N)) ** (1.0 / 3.0)) * (1.0 + rng.uniform(-0.05, 0.05, N))
    cs = np.sqrt(params.gamma * (params.gamma - 1) * u)
    dt = timestep_bins(h, cs)
    return Workload("sedov", params, pos, vel, mass, u, dt, h, np.zeros(N), dict(n1=n1, seed=seed))


def _jittered_lattice(n1: int, rng: np.random.Generator) -> np.ndarray:
    s = 1.0 / n1
    g = (np.arange(n1) + 0.5) * s
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pos += rng.uniform(-0.1, 0.1, size=pos.shape) * s
    return pos % 1.0


def shock_tube(n1: int = 16, seed: int = 5, precision: int = PRECISION_FP64) -> Workload:
    rng = np.random.default_rng(seed)
    N = n1 ** 3
    pos = _jittered_lattice(n1, rng)
    normal = rng.standard_normal(3)
    normal /= np.linalg.norm(normal)
    rho_l, rho_r = rng.uniform(0.125, 1.0, 2)
    p_l, p_r = rng.uniform(0.1, 1.0, 2)
    left = (pos - 0.5) @ normal < 0
    rho = np.where(left, rho_l, rho_r)
    mass = rho / N  # equal volumes per lattice particle: the density follows the mass
    params = make_params(KERNEL_CUBIC, METHOD_MFM, 5.0 / 3.0, 32.0, 0.1, precision)
    u = np.where(left, p_l, p_r) / ((params.gamma - 1.0) * rho)
    vel = np.zeros((N, 3))
    h = np.full(N, (32.0 / (VOLNORM * N)) ** (1.0 / 3.0)) * (1.0 + rng.uniform(-0.05, 0.05, N))
    cs = np.sqrt(params.gamma * (params.gamma - 1) * u)
    dt = timestep_bins(h, cs)
    return Workload("shock_tube", params, pos, vel, mass, u, dt, h, np.zeros(N),
                    dict(n1=n1, seed=seed, normal=normal.tolist(), rho=(rho_l, rho_r), p=(p_l, p_r)))


def boxes(n_boxes: int, seed: int = 5, n_min: int = 1024, n_max: int = 65536,
          precision: int = PRECISION_FP64) -> list:
    """A batch of independent boxes: sizes log-uniform in [n_min, n_max] (rounded
    to a lattice n1^3), each a shock tube or a Sedov blast with equal odds."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_boxes):
        n = np.exp(rng.uniform(np.log(n_min), np.log(n_max)))
        n1 = max(4, int(round(n ** (1.0 / 3.0))))
        sub = int(rng.integers(1 << 30))
        if rng.uniform() < 0.5:
            out.append(shock_tube(n1, seed=sub, precision=precision))
        else:
            out.append(sedov(n1, seed=sub, precision=precision, energy=float(rng.uniform(0.1, 10.0))))
    return out


def _grf(ng: int, slope: float, rng: np.random.Generator) -> np.ndarray:
    kx = np.fft.fftfreq(ng) * ng
    kz = np.fft.rfftfreq(ng) * ng
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    amp = k2 ** (slope / 4.0)  # sqrt(P(k)), P ~ k^slope
    amp[0, 0, 0] = 0.0
    f = (rng.standard_normal(k2.shape) + 1j * rng.standard_normal(k2.shape)) * amp
    field = np.fft.irfftn(f, s=(ng, ng, ng), axes=(0, 1, 2))
    return field / field.std()


def _solenoidal_velocity(ng: int, slope: float, rng: np.random.Generator) -> np.ndarray:
    kx = np.fft.fftfreq(ng) * ng
    kz = np.fft.rfftfreq(ng) * ng
    K = np.stack(np.broadcast_arrays(kx[:, None, None], kx[None, :, None], kz[None, None, :]), axis=0)
    k2 = (K ** 2).sum(0)
    k2[0, 0, 0] = 1.0
    amp = k2 ** (slope / 4.0)
    amp[0, 0, 0] = 0.0
    v = (rng.standard_normal((3,) + k2.shape) + 1j * rng.standard_normal((3,) + k2.shape)) * amp
    kv = (K * v).sum(0) / k2
    v -= K * kv
    out = np.stack([np.fft.irfftn(v[c], s=(ng, ng, ng), axes=(0, 1, 2)) for c in range(3)], axis=-1)
    return out


def lognormal(n1: int = 128, sigma_lnrho: float = 1.5, seed_density: int = 2, seed_velocity: int = 3,
              grid: int | None = None, precision: int = PRECISION_FP64, n_particles: int | None = None) -> Workload:
    """n1^3 particles, or n_particles when given (the density grid follows n1)."""
    N = n1 ** 3 if n_particles is None else int(n_particles)
    ng = grid or min(2 * n1, 256)
    rng = np.random.default_rng(seed_density)
    delta = _grf(ng, -3.0, rng) * sigma_lnrho
    rho = np.exp(delta - delta.max())
    p = rho.ravel() / rho.sum()
    cells = rng.choice(p.size, size=N, p=p)
    cz = cells % ng
    cy = (cells // ng) % ng
    cx = cells // (ng * ng)
    pos = (np.stack([cx, cy, cz], axis=1) + rng.uniform(0, 1, size=(N, 3))) / ng
    pos %= 1.0
    rngv = np.random.default_rng(seed_velocity)
    vg = min(ng, 128)
    vf = _solenoidal_velocity(vg, -4.0, rngv)
    ci = np.minimum((pos * vg).astype(np.int64), vg - 1)
    vel = vf[ci[:, 0], ci[:, 1], ci[:, 2]]
    gamma = 1.0001
    cs = np.sqrt(gamma * (gamma - 1.0) * 1.0)
    # isothermal u = 1 with P = (gamma - 1) rho u; the sound speed of the Riemann
    # states is sqrt(gamma P / rho); rms Mach 2 against that speed
    vel *= 2.0 * cs / np.sqrt((vel ** 2).sum(1).mean())
    mass = np.full(N, 1.0 / N)
    u = np.ones(N)
    params = make_params(KERNEL_WENDLAND_C2, METHOD_MFM, gamma, 64.0, 0.1, precision)
    h = octree_density_h(pos, 64.0)
    dt = timestep_bins(h, np.full(N, cs) + np.sqrt((vel ** 2).sum(1)))
    return Workload("lognormal", params, pos, vel, mass, u, dt, h, np.zeros(N),
                    dict(n1=n1, sigma_lnrho=sigma_lnrho, seeds=(seed_density, seed_velocity)))


def plummer_mix(n1: int = 256, seed: int = 4, n_spheres: int = 1000, precision: int = PRECISION_FP64,
                u0: float = 1e-2) -> Workload:
    rng = np.random.default_rng(seed)
    N = n1 ** 3
    n_bg = N // 10
    n_cl = N - n_bg
    per = np.full(n_spheres, n_cl // n_spheres)
    per[: n_cl - per.sum()] += 1
    centres = rng.uniform(0, 1, size=(n_spheres, 3))
    a = np.exp(rng.uniform(np.log(0.002), np.log(0.02), size=n_spheres))
    sid = np.repeat(np.arange(n_spheres), per)
    aa = a[sid]
    r = np.empty(n_cl)
    todo = np.arange(n_cl)
    while todo.size:
        U = rng.uniform(1e-12, 1.0, size=todo.size)
        rr = aa[todo] * (U ** (-2.0 / 3.0) - 1.0) ** -0.5
        ok = rr <= 20.0 * aa[todo]
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    dirs = rng.standard_normal((n_cl, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos_cl = centres[sid] + dirs * r[:, None]
    m = 1.0 / N
    m_sph = per[sid] * m
    sig = np.sqrt(m_sph / np.sqrt(r * r + aa * aa))
    vel_cl = rng.standard_normal((n_cl, 3)) * sig[:, None]
    pos_bg = rng.uniform(0, 1, size=(n_bg, 3))
    pos = np.concatenate([pos_cl, pos_bg]) % 1.0
    vel = np.concatenate([vel_cl, np.zeros((n_bg, 3))])
    perm = rng.permutation(N)
    pos = np.ascontiguousarray(pos[perm])
    vel = np.ascontiguousarray(vel[perm])
    mass = np.full(N, m)
    u = np.full(N, u0)
    params = make_params(KERNEL_CUBIC, METHOD_MFV, 5.0 / 3.0, 32.0, 0.1, precision)
    h = octree_density_h(pos, 32.0)
    cs = np.sqrt(params.gamma * (params.gamma - 1) * u) + np.sqrt((vel ** 2).sum(1))
    dt = timestep_bins(h, cs)
    return Workload("plummer_mix", params, pos, vel, mass, u, dt, h, np.zeros(N),
                    dict(n1=n1, seed=seed, n_spheres=n_spheres, u0=u0))


def steady_state_seed(h_converged: np.ndarray, seed: int) -> np.ndarray:
    """h0 = converged h x (1 + U(-0.05, 0.05)), the timed-pass seed."""
    rng = np.random.default_rng(seed + 100)
    return h_converged * (1.0 + rng.uniform(-0.05, 0.05, h_converged.shape[0]))
