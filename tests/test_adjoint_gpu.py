"""The adjoint of the DEM step (grains_gpu_adjoint_*) against the FP64
dual-number forward-mode oracle (oracle/tangent_oracle.cpp) and against central
finite differences of the same differentiable run.

Loss (the settling calibration of the adjoint workload): the squared error of
the final centre-of-mass height and of the mean kinetic energy,
    L = (z_com - z*)^2 + (KE - K*)^2,  KE = mean(m |v|^2 / 2 + I |w|^2 / 2).
Derivatives with respect to kn, en, muc, kt of the two laws of the scenario
and to the initial velocities along seeded directions.

512 spheres dropped with N(0, 0.2 m/s) velocities, 100 steps, a checkpoint
every 30 force evaluations (4 segments, the last one short).  The horizon
covers the first collisions; beyond it the granular dynamics is chaotic
(sensitivities grow about tenfold per 10-20 steps) and finite differences
leave their linear range.  Finite differences are accepted only when the runs
at +h and -h have equal contact signatures (same contacts in the same law
branches at every step): the law is not differentiable at contact onset (the
dashpot) nor at stick / slip changes."""
import numpy as np
import pytest

from pacific_b200 import scenarios as S
from pacific_b200.abi import FP64, MIXED, Adjoint

from helpers import make, tangent_run

pytestmark = pytest.mark.gpu

N, STEPS, CHECKPOINT = 512, 100, 30
M = 4                                              # max_materials: law slot (a, b) = a * M + b
SLOTS = [0, 1, M]                                  # (0, 0) particle pairs, (0, 1) and (1, 0) walls
PARAM_INDEX = {"kn": 0, "en": 1, "muc": 3, "kt": 4}  # in the HookeMemory parameter list


def scenario(param=None, delta=0.0, dv=None):
    sc = S.adjoint_4k(n=N)
    if param is not None:
        idx = PARAM_INDEX[param]
        sc.laws = [[(a, b, law, [p + delta if k == idx else p for k, p in enumerate(prm)])
                    for a, b, law, prm in sc.laws[0]]]
    if dv is not None:
        sc.particles = dict(sc.particles)
        sc.particles["velocity"] = sc.particles["velocity"] + dv
    return sc


def loss(sc, final, targets):
    """L and dL/d(final position, velocity, angular velocity)."""
    m = sc.particles["mass"]
    inertia = np.asarray(sc.particles["inertia"])[:, 0]
    x, v, w = final["position"], final["velocity"], final["omega"]
    n = len(m)
    zc = x[:, 2].mean()
    ke = np.mean(0.5 * m * (v * v).sum(1) + 0.5 * inertia * (w * w).sum(1))
    z0, k0 = targets
    gx = np.zeros_like(x)
    gx[:, 2] = 2.0 * (zc - z0) / n
    gv = 2.0 * (ke - k0) * (m[:, None] * v) / n
    gw = 2.0 * (ke - k0) * (inertia[:, None] * w) / n
    return (zc - z0) ** 2 + (ke - k0) ** 2, gx, gv, gw


def targets_of(sc, final):
    """Targets 0.1 mm below the run's final height and at 60 % of its energy."""
    m = sc.particles["mass"]
    inertia = np.asarray(sc.particles["inertia"])[:, 0]
    v, w = final["velocity"], final["omega"]
    ke = np.mean(0.5 * m * (v * v).sum(1) + 0.5 * inertia * (w * w).sum(1))
    return final["position"][:, 2].mean() - 1e-4, 0.6 * ke


def run(gpu_lib, sc, precision, targets=None, backward=False):
    sim = make(gpu_lib, sc, precision)
    adj = Adjoint(sim, CHECKPOINT)
    final = adj.forward(STEPS, sc.dt)
    sig = adj.signature()
    targets = targets or targets_of(sc, final)
    L, gx, gv, gw = loss(sc, final, targets)
    grads = adj.backward(gx, gv, gw) if backward else None
    adj.close()
    sim.close()
    return dict(L=L, grads=grads, sig=sig, targets=targets, final=final, dfinal=(gx, gv, gw))


def directions(seed=7, n_v=2):
    """Directions of (initial velocities, law parameters per slot): one per
    parameter (both laws together), then n_v random velocity directions."""
    rng = np.random.default_rng(seed)
    nd = 4 + n_v
    dv = np.zeros((nd, N, 3))
    dl = np.zeros((nd, M * M, 4))
    for t in range(4):
        dl[t, SLOTS, t] = 1.0
    for t in range(n_v):
        d = rng.normal(size=(N, 3))
        dv[4 + t] = d / np.linalg.norm(d)
    return dv, dl


def adjoint_directional(grads, dv, dl):
    return np.array([(grads["velocity"] * dv[d]).sum() + (grads["laws"] * dl[d]).sum() for d in range(len(dv))])


def test_forward_run_equals_the_oracle_run(gpu_lib):
    """The CUDA FP64 differentiable run and the oracle's FP64 run of the same
    map: same arithmetic, same results."""
    sc = scenario()
    r = run(gpu_lib, sc, FP64)
    fin, _ = tangent_run(sc, STEPS)
    assert np.max(np.abs(r["final"]["position"] - fin["position"])) < 1e-15
    assert np.max(np.abs(r["final"]["velocity"] - fin["velocity"])) < 1e-12
    assert np.max(np.abs(r["final"]["omega"] - fin["omega"])) < 1e-9
    assert r["sig"][1] > 100, "the run should meet contacts"


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_adjoint_matches_dual_number_gradient(gpu_lib, precision):
    """<dL/dtheta, direction> from the adjoint against the FP64 forward-mode
    derivative of the oracle.  FP64 adjoint: 1e-6 relative.  Mixed precision
    (FP32 velocities, law and adjoint): 2e-3, the drift of the FP32 run itself
    from the FP64 one over the collisions it differentiates."""
    sc = scenario()
    r = run(gpu_lib, sc, precision, backward=True)
    dv, dl = directions()
    fin, tan = tangent_run(sc, STEPS, dv, dl)
    _, gx, gv, gw = loss(sc, fin, r["targets"])
    dual = np.array([(gx * tan["position"][d]).sum() + (gv * tan["velocity"][d]).sum() +
                     (gw * tan["omega"][d]).sum() for d in range(len(dv))])
    adj = adjoint_directional(r["grads"], dv, dl)
    tol = 1e-6 if precision == FP64 else 2e-3
    rel = np.abs(adj - dual) / np.abs(dual)
    assert np.all(rel < tol), (rel, adj, dual)


def test_adjoint_matches_finite_differences(gpu_lib):
    """FP64 adjoint against central differences of the CUDA FP64 run: h = 1e-6
    relative on the law parameters, 1e-8 on unit velocity directions."""
    base = scenario()
    r = run(gpu_lib, base, FP64, backward=True)
    dv, dl = directions(n_v=2)
    adj = adjoint_directional(r["grads"], dv, dl)
    checked = 0
    for t, name in enumerate(["kn", "en", "muc", "kt"]):
        value = base.laws[0][0][3][PARAM_INDEX[name]]
        h = 1e-6 * value
        rp = run(gpu_lib, scenario(name, h), FP64, r["targets"])
        rm = run(gpu_lib, scenario(name, -h), FP64, r["targets"])
        if rp["sig"] != rm["sig"]:
            continue
        fd = (rp["L"] - rm["L"]) / (2 * h)
        assert abs(adj[t] - fd) <= 1e-5 * abs(fd), (name, adj[t], fd)
        checked += 1
    for t in range(4, len(dv)):
        h = 1e-8
        rp = run(gpu_lib, scenario(dv=h * dv[t]), FP64, r["targets"])
        rm = run(gpu_lib, scenario(dv=-h * dv[t]), FP64, r["targets"])
        if rp["sig"] != rm["sig"]:
            continue
        fd = (rp["L"] - rm["L"]) / (2 * h)
        assert abs(adj[t] - fd) <= 1e-4 * abs(fd), ("velocity", adj[t], fd)
        checked += 1
    assert checked >= 4


def test_forward_run_follows_the_step(gpu_lib):
    """The differentiable run is the leapfrog of grains_gpu_step: equal final
    state up to rounding (the angular velocity is integrated in the world frame
    instead of the body frame)."""
    sc = scenario()
    r = run(gpu_lib, sc, FP64)
    sim = make(gpu_lib, sc, FP64)
    sim.initialize_leapfrog(0.0, sc.dt)
    sim.step(STEPS, 0.0, sc.dt)
    d = sim.download()
    assert np.max(np.abs(d["position"] - r["final"]["position"])) < 1e-15
    assert np.max(np.abs(d["velocity"] - r["final"]["velocity"])) < 1e-12
    sim.close()


def test_adjoint_is_deterministic(gpu_lib):
    sc = scenario()
    g1 = run(gpu_lib, sc, MIXED, backward=True)["grads"]
    g2 = run(gpu_lib, sc, MIXED, backward=True)["grads"]
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k


def test_adjoint_rejects_unsupported_scenes(gpu_lib):
    """Non-spherical particles and the Hertz laws are outside the
    differentiable run's scope: the call fails with a message instead of
    returning wrong gradients."""
    sc = S.convex_box(27, seed=1)
    sim = make(gpu_lib, sc, MIXED)
    with pytest.raises(Exception, match="spheres"):
        Adjoint(sim, 10).forward(5, sc.dt)
    sim.close()
    sc = S.dense_cluster(27, seed=1)
    sc.laws = [[(a, b, S.HERTZ_MEMORY, [1.0e9, 0.8, 0.4, 0.3e9, 0.0, 0.0, 0.0]) for a, b, _, _ in sc.laws[0]]]
    sim = make(gpu_lib, sc, MIXED)
    with pytest.raises(Exception, match="Hooke"):
        Adjoint(sim, 10).forward(5, 2.0e-6)
    sim.close()


class GrainsRun:
    """torch.autograd.Function over the differentiable run (test harness only):
    inputs the initial velocities (n, 3) and theta = (kn, en, muc, kt) of both
    laws; outputs the final positions, velocities and angular velocities."""

    @staticmethod
    def make(gpu_lib, precision):
        import torch

        class Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, v0, theta):
                sc = S.adjoint_4k(n=N)
                kn, en, muc, kt = [float(x) for x in theta]
                sc.laws = [[(a, b, law, S.hooke_memory_params(kn, en, muc, kt)) for a, b, law, _ in sc.laws[0]]]
                sc.particles = dict(sc.particles)
                sc.particles["velocity"] = v0.detach().cpu().numpy().astype(np.float64)
                sim = make(gpu_lib, sc, precision)
                adj = Adjoint(sim, CHECKPOINT)
                fin = adj.forward(STEPS, sc.dt)
                ctx.keep = (sim, adj)
                as_t = lambda a: torch.tensor(a, dtype=torch.float64)  # noqa: E731
                return as_t(fin["position"]), as_t(fin["velocity"]), as_t(fin["omega"])

            @staticmethod
            def backward(ctx, gx, gv, gw):
                sim, adj = ctx.keep
                g = adj.backward(gx.numpy(), gv.numpy(), gw.numpy())
                laws = g["laws"][SLOTS].sum(0)
                adj.close()
                sim.close()
                return torch.tensor(g["velocity"]), torch.tensor(laws)

        return Fn


def test_autograd_function_wrapper(gpu_lib):
    """The adjoint through torch.autograd: L.backward() gives the gradients of
    the C ABI, equal to the dual-number oracle's derivatives."""
    import torch
    Fn = GrainsRun.make(gpu_lib, FP64)
    sc = scenario()
    prm = sc.laws[0][0][3]
    v0 = torch.tensor(sc.particles["velocity"], dtype=torch.float64, requires_grad=True)
    theta = torch.tensor([prm[0], prm[1], prm[3], prm[4]], dtype=torch.float64, requires_grad=True)
    x, v, w = Fn.apply(v0, theta)
    m = torch.tensor(sc.particles["mass"])
    inertia = torch.tensor(np.asarray(sc.particles["inertia"])[:, 0])
    zc = x[:, 2].mean()
    ke = (0.5 * m * (v * v).sum(1) + 0.5 * inertia * (w * w).sum(1)).mean()
    targets = (float(zc) - 1e-4, 0.6 * float(ke))
    L = (zc - targets[0]) ** 2 + (ke - targets[1]) ** 2
    L.backward()
    dv, dl = directions()
    fin, tan = tangent_run(sc, STEPS, dv, dl)
    _, gx, gv, gw = loss(sc, fin, targets)
    dual = np.array([(gx * tan["position"][d]).sum() + (gv * tan["velocity"][d]).sum() +
                     (gw * tan["omega"][d]).sum() for d in range(len(dv))])
    # theta's gradient is summed over the law slots; the directions move all slots together
    via_torch = np.array([(v0.grad.numpy() * dv[d]).sum() + (theta.grad.numpy() * dl[d][0]).sum()
                          for d in range(len(dv))])
    assert np.all(np.abs(via_torch - dual) <= 1e-6 * np.abs(dual)), (via_torch, dual)
