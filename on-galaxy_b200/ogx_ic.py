"""Seeded synthetic initial conditions for the benchmark and parity configs.

All inputs are synthetic (no datasets).  Generators use numpy's PCG64 so the
same seed gives the same bodies on every machine.

* ``plummer``  -- equal-mass Plummer sphere (scale a), radii by inverse CDF of
  the enclosed mass like makePlummerSphere (src3d/InitialConditions3D.hpp:100-152),
  with an added truncation at ``rmax_a * a`` (sampled exactly by restricting the
  enclosed-mass fraction, not by rejection), Aarseth speeds by rejection from
  q^2 (1-q^2)^{7/2}, centre of mass and net momentum removed.
* ``disk_bulge`` -- 80% of the bodies in an exponential disk (scale length Rd,
  sech^2(z/z0) vertical profile, mass Md) and 20% in a Hernquist bulge (scale
  ab, mass Mb), equal masses inside each component.  The disk follows
  makeDisk's structure (src3d/gpu/GalaxyIC.hpp:43-72) with the profiles of the
  benchmark configuration; the disk is cut at 10 Rd and |z| <= 10 z0, the bulge
  at 50 ab (enclosed-mass fraction 0.961), to keep a bounded root box.
* ``set_circular_velocities`` -- v_c^2 = -a_R R from a measured FP64 force
  field plus an isotropic dispersion (setCircularVelocities,
  src3d/gpu/GalaxyIC.hpp:76-97; the dispersion here is 0.1 v_c by default).
* ``merger`` -- two disk+bulge galaxies at x = -/+ sep with bulk velocities
  +/- vrel/2 along x and the second disk tilted by ``tilt_deg`` about x
  (placeGalaxy, src3d/gpu/GalaxyIC.hpp:101-108; concat :111-125).
"""
from __future__ import annotations

import numpy as np


def _unit_vectors(rng, n):
    cz = 2.0 * rng.random(n) - 1.0
    sz = np.sqrt(np.maximum(0.0, 1.0 - cz * cz))
    ph = 2.0 * np.pi * rng.random(n)
    return np.stack([sz * np.cos(ph), sz * np.sin(ph), cz], axis=1)


def plummer(n, seed=1, a=1.0, total_mass=1.0, G=1.0, rmax_a=20.0):
    """Plummer sphere; returns pos (n,3), vel (n,3), mass (n,)."""
    if n <= 0:
        raise ValueError("Plummer N must be > 0")
    rng = np.random.Generator(np.random.PCG64(seed))
    rmax = rmax_a * a
    umax = rmax ** 3 / (rmax ** 2 + a ** 2) ** 1.5
    u = np.maximum(rng.random(n) * umax, 1e-12)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        qq = rng.random(todo.size)
        g = 0.1 * rng.random(todo.size)
        ok = g <= qq * qq * (1.0 - qq * qq) ** 3.5
        q[todo[ok]] = qq[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0 * G * total_mass) * (r * r + a * a) ** -0.25
    pos = r[:, None] * _unit_vectors(rng, n)
    vel = (q * vesc)[:, None] * _unit_vectors(rng, n)
    mass = np.full(n, total_mass / n)
    pos -= (mass[:, None] * pos).sum(0) / mass.sum()
    vel -= (mass[:, None] * vel).sum(0) / mass.sum()
    return pos, vel, mass


def disk_bulge(n, seed=1, Rd=1.0, z0=0.1, Md=1.0, ab=0.2, Mb=0.25, bulge_frac=0.2):
    """Exponential sech^2 disk + Hernquist bulge; returns pos (n,3), mass (n,), species (n,) 0=disk 1=bulge."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nb = int(round(bulge_frac * n))
    nd = n - nb
    # disk: surface density ~ exp(-R/Rd) -> R ~ Gamma(2, Rd), cut at 10 Rd
    R = np.empty(nd)
    todo = np.arange(nd)
    while todo.size:
        rr = rng.gamma(2.0, Rd, todo.size)
        ok = rr <= 10.0 * Rd
        R[todo[ok]] = rr[ok]
        todo = todo[~ok]
    ph = 2.0 * np.pi * rng.random(nd)
    # sech^2(z/z0): CDF (1 + tanh(z/z0))/2, cut at |z| <= 10 z0
    t = np.tanh(10.0)
    z = z0 * np.arctanh((2.0 * rng.random(nd) - 1.0) * t)
    disk = np.stack([R * np.cos(ph), R * np.sin(ph), z], axis=1)
    # Hernquist: M(<r)/Mb = r^2/(r+a)^2 -> r = a s/(1-s), s = sqrt(u); cut at 50 a
    umax = (50.0 / 51.0) ** 2
    s = np.sqrt(rng.random(nb) * umax)
    rb = ab * s / (1.0 - s)
    bulge = rb[:, None] * _unit_vectors(rng, nb)
    pos = np.concatenate([disk, bulge], axis=0)
    mass = np.concatenate([np.full(nd, Md / max(nd, 1)), np.full(nb, Mb / max(nb, 1))])
    species = np.concatenate([np.zeros(nd, np.int8), np.ones(nb, np.int8)])
    return pos, mass, species


def set_circular_velocities(pos, acc, seed=1, disp_frac=0.1):
    """Tangential circular speed from the measured field, v_c^2 = -a_R R, plus isotropic dispersion."""
    rng = np.random.Generator(np.random.PCG64(seed + 12345))
    x, y = pos[:, 0], pos[:, 1]
    R = np.sqrt(x * x + y * y)
    vel = np.zeros_like(pos)
    big = R > 1e-6
    a_rad = np.where(big, (acc[:, 0] * x + acc[:, 1] * y) / np.where(big, R, 1.0), 0.0)
    vc = np.sqrt(np.maximum(-a_rad * R, 0.0))
    tang = np.stack([-y, x, np.zeros_like(x)], axis=1) / np.where(big, R, 1.0)[:, None]
    vel[big] = (vc[:, None] * tang)[big]
    sig = disp_frac * vc
    vel += sig[:, None] * rng.standard_normal(pos.shape)
    return vel


def place(pos, vel, incl_rad, center, bulk):
    c, s = np.cos(incl_rad), np.sin(incl_rad)
    rot = np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    return pos @ rot.T + np.asarray(center), vel @ rot.T + np.asarray(bulk)


def merger(n_per, seed=1, accel_fn=None, sep=5.0, vrel=0.5, tilt_deg=30.0, disp_frac=0.1):
    """Two-galaxy merger.  ``accel_fn(pos, mass) -> acc`` supplies the FP64 field used for v_c
    (the caller passes the library's FP64 solver); returns pos, vel, mass, species."""
    out = []
    for g, (cx, vx, tilt, sd) in enumerate(((-sep, +0.5 * vrel, 0.0, seed), (+sep, -0.5 * vrel, tilt_deg, seed + 7))):
        p, m, sp = disk_bulge(n_per, seed=sd)
        if accel_fn is not None:
            acc = accel_fn(p, m)
            v = set_circular_velocities(p, acc, seed=sd, disp_frac=disp_frac)
        else:
            v = np.zeros_like(p)
        p, v = place(p, v, np.deg2rad(tilt), (cx, 0.0, 0.0), (vx, 0.0, 0.0))
        out.append((p, v, m, sp + 2 * g))
    pos = np.concatenate([o[0] for o in out])
    vel = np.concatenate([o[1] for o in out])
    mass = np.concatenate([o[2] for o in out])
    species = np.concatenate([o[3] for o in out])
    return pos, vel, mass, species


def uniform_cube(n, seed=1):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(-1.0, 1.0, (n, 3)), rng.uniform(0.5, 1.5, n)
