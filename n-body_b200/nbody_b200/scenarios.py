"""Seeded synthetic scenarios (host-side input data, not part of the force path).

The reference measures on AGORA/MUGS snapshots that are not available here; these generators
produce inputs with the configured shapes instead. All return float32 arrays of shape (n, 4):
bodies as (x, y, z, m) and velocities as (vx, vy, vz, 0). G = 1 throughout.

  uniform_ball   positions uniform in the unit ball (rejection from [-1, 1]^3), masses uniform
                 in [0.5, 1.5] / n, zero velocities
  plummer        Plummer sphere (scale radius a, total mass M): radii from the inverse cumulative
                 mass r = a (X^(-2/3) - 1)^(-1/2), truncated at r_max; isotropic speeds from the
                 distribution function by von Neumann rejection (Aarseth, Henon & Wielen 1974)
  hernquist      Hernquist sphere: r = a sqrt(X) / (1 - sqrt(X)), truncated at r_max; isotropic
                 speeds by rejection from the Hernquist (1990) ergodic distribution function
  colliding_hernquist  two Hernquist spheres on a collision course (the dual-tree scene)
  batched_plummer      many Plummer spheres of log-uniform sizes and uniform theta (the batch)
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.MT19937(seed))


def _isotropic(rng: np.random.Generator, n: int) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t], axis=1)


def _pack(pos: np.ndarray, mass: np.ndarray, vel: np.ndarray):
    n = len(pos)
    bodies = np.zeros((n, 4), np.float32)
    bodies[:, :3] = pos
    bodies[:, 3] = mass
    velocities = np.zeros((n, 4), np.float32)
    velocities[:, :3] = vel
    return bodies, velocities


def uniform_ball(n: int, seed: int = 42):
    rng = _rng(seed)
    pts = np.zeros((0, 3))
    while len(pts) < n:
        c = rng.uniform(-1.0, 1.0, (max(2 * (n - len(pts)), 16), 3))
        pts = np.concatenate([pts, c[(c * c).sum(1) < 1.0]])
    mass = rng.uniform(0.5, 1.5, n) / n
    return _pack(pts[:n], mass, np.zeros((n, 3)))


def plummer(n: int, seed: int = 43, a: float = 1.0, M: float = 1.0, r_max: float = 100.0):
    rng = _rng(seed)
    r = np.zeros(0)
    while len(r) < n:
        X = rng.uniform(0.0, 1.0, n - len(r))
        X = X[(X > 0.0)]
        rr = a / np.sqrt(X ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[rr <= r_max * a]])
    r = r[:n]
    pos = r[:, None] * _isotropic(rng, n)
    # speed fraction q = v / v_esc with density g(q) = q^2 (1 - q^2)^(7/2) (max < 0.1)
    q = np.zeros(0)
    while len(q) < n:
        qq = rng.uniform(0.0, 1.0, 2 * (n - len(q)) + 16)
        yy = rng.uniform(0.0, 0.1, len(qq))
        q = np.concatenate([q, qq[yy < qq * qq * (1.0 - qq * qq) ** 3.5]])
    q = q[:n]
    v_esc = np.sqrt(2.0 * M / a) * (1.0 + (r / a) ** 2) ** -0.25
    vel = (q * v_esc)[:, None] * _isotropic(rng, n)
    pos -= pos.mean(0)
    vel -= vel.mean(0)
    return _pack(pos, np.full(n, M / n), vel)


def _hernquist_df(E: np.ndarray) -> np.ndarray:
    """Hernquist (1990) ergodic DF for G = M = a = 1, q = sqrt(-E) in (0, 1), up to a constant."""
    q = np.sqrt(np.clip(-E, 0.0, 1.0 - 1e-12))
    qq = q * q
    return (3.0 * np.arcsin(q) + q * np.sqrt(1.0 - qq) * (1.0 - 2.0 * qq) * (8.0 * qq * qq - 8.0 * qq - 3.0)) \
        / (1.0 - qq) ** 2.5


def hernquist(n: int, seed: int = 44, a: float = 1.0, M: float = 1.0, r_max: float = 100.0):
    rng = _rng(seed)
    r = np.zeros(0)
    while len(r) < n:
        X = rng.uniform(0.0, 1.0, n - len(r))
        s = np.sqrt(X)
        rr = a * s / np.maximum(1.0 - s, 1e-300)
        r = np.concatenate([r, rr[rr <= r_max * a]])
    r = r[:n]
    pos = r[:, None] * _isotropic(rng, n)
    # speeds by rejection from p(v) ~ v^2 f(psi - v^2/2), psi = 1 / (1 + r) in units G = M = a = 1
    psi = (M / a) / (1.0 + r / a)
    v_esc = np.sqrt(2.0 * psi)
    speed = np.zeros(n)
    todo = np.arange(n)
    while len(todo):
        u = rng.uniform(0.0, 1.0, len(todo))
        v = u * v_esc[todo]
        E = 0.5 * v * v - psi[todo]
        p = (u * u) * _hernquist_df(E / (M / a))
        # bound: the density in u peaks below u^2 f(-psi) at u = 0 .. 1; use f(-psi) as envelope
        env = _hernquist_df(-psi[todo] / (M / a))
        y = rng.uniform(0.0, 1.0, len(todo)) * env
        ok = y < p
        speed[todo[ok]] = v[ok]
        todo = todo[~ok]
    vel = speed[:, None] * _isotropic(rng, n)
    pos -= pos.mean(0)
    vel -= vel.mean(0)
    return _pack(pos, np.full(n, M / n), vel)


def colliding_hernquist(half: int, seed: int = 46, separation: float = 20.0, approach: float = 0.5):
    """Two Hernquist spheres of `half` bodies each (a = 1, total mass 1 each, truncated at 100 a),
    centred at x = -separation/2 and +separation/2 and approaching at `approach` along x (half of
    it each): the dual-tree precision-study scene."""
    a, va = hernquist(half, seed=seed)
    b, vb = hernquist(half, seed=seed + 1)
    a[:, 0] -= np.float32(separation / 2)
    b[:, 0] += np.float32(separation / 2)
    va[:, 0] += np.float32(approach / 2)
    vb[:, 0] -= np.float32(approach / 2)
    return np.concatenate([a, b]), np.concatenate([va, vb])


def batched_plummer(count: int, seed: int = 44, n_min: int = 1024, n_max: int = 200000,
                    theta_range=(0.4, 0.7)):
    """`count` independent Plummer spheres with N log-uniform in [n_min, n_max] (rounded) and theta
    uniform in theta_range: (sizes int64[count], thetas float32[count], bodies list, velocities list)."""
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(np.log(n_min), np.log(n_max), count))).astype(np.int64)
    thetas = rng.uniform(theta_range[0], theta_range[1], count).astype(np.float32)
    bodies, vels = [], []
    for k, n in enumerate(sizes):
        pm, vel = plummer(int(n), seed=seed * 1000 + k)
        bodies.append(pm)
        vels.append(vel)
    return sizes, thetas, bodies, vels


def softening_to_epsilon(softening_length: float) -> float:
    """A configured softening length e enters the reference's Gravity as epsilon = e^2, since
    Gravity adds epsilon to r^2 (Gravity.h:207)."""
    return float(np.float32(softening_length) * np.float32(softening_length))


def write_json(path: str, bodies, velocities=None, G: float | None = None, accelerations=None) -> None:
    """A scenario in the reference's JSON schema (NBody::to_json, Simulation.cpp:154-185):
    {"G": G (optional), "particles": [{"position", "velocity", "mass", "acceleration"}]}.
    Floats are written with 9 significant digits, which read back to the same float32."""
    import json

    pm = np.asarray(bodies, np.float32)
    vel = np.zeros_like(pm) if velocities is None else np.asarray(velocities, np.float32)
    acc = None if accelerations is None else np.asarray(accelerations, np.float32)

    def v3(a):
        return {"x": float(a[0]), "y": float(a[1]), "z": float(a[2])}

    parts = []
    for i in range(len(pm)):
        p = {"position": v3(pm[i]), "velocity": v3(vel[i]), "mass": float(pm[i, 3])}
        if acc is not None:
            p["acceleration"] = v3(acc[i])
        parts.append(p)
    root = {"particles": parts}
    if G is not None:
        root = {"G": float(np.float32(G)), **root}
    with open(path, "w") as f:
        json.dump(root, f)


def read_json(path: str):
    """(bodies, velocities, accelerations, G or None) of a JSON scenario (NBody::from_json,
    Simulation.cpp:187-228): missing vectors read as zero, a missing mass as 0."""
    import json

    with open(path) as f:
        root = json.load(f)
    parts = root["particles"]
    n = len(parts)
    pm = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 4), np.float32)
    acc = np.zeros((n, 4), np.float32)
    for i, p in enumerate(parts):
        for key, arr in (("position", pm), ("velocity", vel), ("acceleration", acc)):
            if key in p:
                arr[i, :3] = (p[key]["x"], p[key]["y"], p[key]["z"])
        pm[i, 3] = p.get("mass", 0.0)
    G = root.get("G")
    return pm, vel, acc, (None if G is None else float(G))
