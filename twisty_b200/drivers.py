"""Receiver-grid drivers: the reference's experiment programs that loop RunExperiment over
receivers, rebuilt as one batched pass (twisty_run_batch) each.

* ``ring_experiments`` -- Experiments/RingBenchmark.cpp:168-201: a receiver at
  (ringRadius, 0, z) for z over [zMin, zMax], tangent pointing away from the emitter,
  arclength max(1.1 |x_e - x_s|, 3). The reference runs only the last z (its loop is a TODO);
  here every z of the sweep is one experiment of the batch.
* ``beam_spread_experiments`` -- Experiments/BeamSpreadExperiment.cpp:178-196: receivers on a
  sphere of radius sphereRadius around the source, the direction drawn as the reference draws
  it from std::mt19937(targetSeed) with std::uniform_real_distribution<float> (the same
  stream: the first receiver is the reference's). The reference hands RunExperiment boundary
  conditions without an arclength (:269); here arclength_scale times the minimum
  arclength (CalculateMinimumArclength, Twisty/PathGeneration.cpp:12-43) is used.
* ``image_plane_experiments`` -- the pixel loop of the image drivers
  (Experiments/NoisyCircleExperiment.cpp:259-361): a grid of receivers on a plane, one
  experiment per pixel.

Each returns a list of twisty_experiment structs; ``run`` passes them to a context's
run_batch and returns one result per experiment.
"""
from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np

from . import _abi, make_bc, make_experiment, min_arclength

F32 = np.float32


def ring_experiments(start_pos: Sequence[float], start_dir: Sequence[float], ring_radius: float, z_min: float,
                     z_max: float, num_z: int, num_segments: int, scatter: float, eps: float,
                     paths: int) -> List[_abi.Experiment]:
    """RingBenchmark's geometry for every z of its sweep (z_i = zMin + i (zMax - zMin)/(numZ - 1))."""
    sp = np.asarray(start_pos, F32)
    out = []
    dz = (z_max - z_min) / (num_z - 1) if num_z > 1 else 0.0
    for i in range(num_z):
        z = z_min + dz * i
        ep = np.array([ring_radius, 0.0, z], F32)
        d = (ep - sp).astype(F32)
        dist = F32(math.sqrt(float(F32(d @ d))))
        S = max(float(F32(dist * F32(1.1))), 3.0)
        bc = make_bc(sp, start_dir, ep, d, S)
        out.append(make_experiment(bc, num_segments, scatter, eps, paths))
    return out


def _mt19937_uniform_floats(seed: int, n: int) -> np.ndarray:
    """n draws of std::uniform_real_distribution<float>(0, 1) from std::mt19937(seed) (libstdc++:
    generate_canonical<float, 24> takes one 32-bit output x and returns float(x) / 2^32 in
    float, pulled below 1)."""
    bg = np.random.MT19937(0)
    bg._legacy_seeding(int(seed) & 0xFFFFFFFF)
    raw = np.array([bg.random_raw() for _ in range(n)], dtype=np.uint64)
    u = (raw.astype(F32) / F32(4294967296.0)).astype(F32)
    return np.where(u >= F32(1.0), np.nextafter(F32(1.0), F32(0.0)), u).astype(F32)


def beam_spread_experiments(start_pos: Sequence[float], start_dir: Sequence[float], sphere_radius: float,
                            num_receivers: int, target_seed: int, num_segments: int, scatter: float, eps: float,
                            paths: int, arclength_scale: float = 1.05) -> List[_abi.Experiment]:
    """BeamSpreadExperiment's receivers: direction (n1, cos(2 pi e1) sqrt(1 - n1^2),
    sin(2 pi e1) sqrt(1 - n1^2)) with n1 = 2u - 1, e1 = u' from the reference's stream, the
    receiver at start + R dir with tangent dir."""
    u = _mt19937_uniform_floats(target_seed, 2 * num_receivers)
    sp = np.asarray(start_pos, F32)
    pi = F32(3.141592653589793)
    out = []
    for i in range(num_receivers):
        n1 = F32(u[2 * i] * F32(2.0)) - F32(1.0)
        e1 = u[2 * i + 1]
        r = F32(math.sqrt(float(F32(1.0) - n1 * n1)))
        ang = float(F32(F32(2.0) * pi) * e1)
        d = np.array([n1, F32(math.cos(ang)) * r, F32(math.sin(ang)) * r], F32)
        ep = (sp + F32(sphere_radius) * d).astype(F32)
        bc = make_bc(sp, start_dir, ep, d, 1.0)
        bc.arclength = float(F32(arclength_scale) * F32(min_arclength(bc, num_segments)))
        out.append(make_experiment(bc, num_segments, scatter, eps, paths))
    return out


def image_plane_experiments(nx: int, ny: int, half_extent: float, plane_z: float, num_segments: int, scatter: float,
                            eps: float, paths: int, source_pos: Sequence[float] = (0.0, 0.0, 0.0),
                            source_dir: Sequence[float] = (0.0, 0.0, 1.0), receiver_dir: Sequence[float] = (0.0, 0.0, 1.0),
                            arclength_factor: float = 1.3) -> List[_abi.Experiment]:
    """A pixel grid: receivers at (x_i, y_j, plane_z) with x, y spanning [-half_extent,
    half_extent] (pixel centres), one tangent for all, S = arclength_factor x distance, raised
    to 1.01 x the minimum arclength where that is larger."""
    sp = np.asarray(source_pos, F32)
    out = []
    for j in range(ny):
        for i in range(nx):
            x = -half_extent + (i + 0.5) * (2.0 * half_extent / nx)
            y = -half_extent + (j + 0.5) * (2.0 * half_extent / ny)
            ep = np.array([x, y, plane_z], F32)
            d = (ep - sp).astype(F32)
            bc = make_bc(sp, source_dir, ep, receiver_dir, 1.0)
            S = float(arclength_factor) * math.sqrt(float(d @ d))
            S = max(S, 1.01 * float(min_arclength(bc, num_segments)))
            bc.arclength = float(S)
            out.append(make_experiment(bc, num_segments, scatter, eps, paths))
    return out


def run(ctx, experiments: Sequence[_abi.Experiment], iterations: int = 1):
    """One batched pass over the experiments (twisty_run_batch)."""
    return ctx.run_batch(list(experiments), iterations=iterations)
