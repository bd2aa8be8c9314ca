"""Shared helpers of the parity tests: run the same scenario through the CUDA
library and the CPU oracle and compare."""
import numpy as np

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED, Simulation


def make(lib, sc, precision=FP64, history_capacity=0):
    sim = Simulation(lib, precision, max_particles=max(sc.n, 1), n_systems=len(sc.domains),
                     history_capacity=history_capacity)
    S.apply(sim, sc)
    return sim


def pair_set(a):
    return set(map(tuple, np.asarray(a).reshape(-1, 2).tolist()))


def rel_err(a, b, floor):
    """max |a - b| / max(|b|, floor) over rows (vector norms)."""
    a, b = np.asarray(a), np.asarray(b)
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), floor)
    return float(np.max(num / den)) if len(num) else 0.0


def perturbed_cluster(n=200, seed=0, sigma=0.2, spacing=2.04):
    """A cluster of spheres with velocities large enough to collide in a few
    steps and with walls in reach."""
    return S.small_box(n, seed=seed, velocity_sigma=sigma, spacing=spacing)


def rel_err_quantile(a, b, floor, q):
    """q-quantile over rows of |a - b| / max(|b|, floor)."""
    a, b = np.asarray(a), np.asarray(b)
    num = np.linalg.norm(a - b, axis=-1)
    den = np.maximum(np.linalg.norm(b, axis=-1), floor)
    return float(np.quantile(num / den, q)) if len(num) else 0.0


def check_contact_forces(fg, fo, floor, precision):
    """Per-contact forces: FP64 at rounding level.  Mixed: 1e-5 for 99 % of the
    contacts and 1e-4 for all.  The FP32 law rounds each term to ~6e-8 of
    itself, but where the elastic and viscous normal terms nearly cancel (a
    contact about to open) the relative error of their sum grows by the
    cancellation ratio."""
    if precision == FP64:
        assert rel_err(fg, fo, floor) < 1e-12
    else:
        assert rel_err_quantile(fg, fo, floor, 0.99) < 1e-5
        assert rel_err(fg, fo, floor) < 1e-4
