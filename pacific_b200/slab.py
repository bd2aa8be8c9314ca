"""One system over several processes: a slab decomposition of the domain with
a ghost layer, the partition of the reference's MPI build.

The reference's GrainsMPI::Simulation (Base/src/GrainsMPI.cpp:120-210) moves
its particles, sends the positions and velocities of the particles near a
subdomain face to the neighbouring process, where they live as clones
(GrainsMPIWrapper::UpdateOrCreateClones_SendRecvLocal_GeoLoc,
GrainsMPIWrapper.cpp:1337-1555), relinks, computes the forces of its own
particles with the clones present, and kicks.  The same step here, over any
implementation of the grains_gpu C ABI (one per process, each on its own
device):

* Each rank owns the particles of one slab of the domain along an axis (the
  longest by default).  The slab bounds are quantiles of the particle
  coordinates, so each rank owns about N / world particles; they are set again
  at every rebuild.
* Each rank also holds as ghosts the particles of other slabs within
  H = 2 r_max + 2 d of its slab, where r_max is the largest circumscribed
  radius and d the largest displacement allowed between two rebuilds.  An
  owned particle then meets every contact partner it can have before the next
  rebuild, so its force is the single-domain force: the contact forces of
  ghost pairs are computed here as well and thrown away (the reference's
  clones do the same).
* Every step: move all local particles; the owners send the moved state
  (position, quaternion, basis, velocity, angular velocity) of their particles
  that are ghosts elsewhere, and the receivers overwrite their ghosts with it;
  relink; compute forces; second half kick.  This is the one exchange of the
  step.
* Rebuild (every `rebuild_every` steps, or at once when some particle has
  moved more than d since the last rebuild): all ranks gather the states of
  the owned particles and the contact memory held by them, recompute the
  slabs, and every rank re-uploads its owned particles and ghosts with the
  memory of their pairs.  A pair's memory is exact on the rank that owns
  either particle (its partners were always present there), so particles that
  change owner keep their tangential history.

The exchange runs on torch.distributed: point-to-point tensors for the
per-step ghost states, gathered Python objects at rebuilds.  With the CPU
oracle and the gloo backend this runs and is tested as several processes on
one host; with the CUDA library each process drives its own GPU."""
import numpy as np
import torch
import torch.distributed as dist

from . import scenarios as S
from .abi import Simulation

# kinematic state exchanged per particle: position 3, quaternion 4, basis 9,
# velocity 3, angular velocity 3
KINEMATIC = [("position", 3), ("quaternion", 4), ("basis", 9), ("velocity", 3), ("omega", 3)]
WIDTH = sum(w for _, w in KINEMATIC)


def _pack(st, rows):
    return np.concatenate([st[k][rows].reshape(len(rows), w) for k, w in KINEMATIC], axis=1)


def _unpack(st, rows, data):
    c = 0
    for k, w in KINEMATIC:
        st[k][rows] = data[:, c:c + w].reshape(st[k][rows].shape)
        c += w


class SlabRun:
    """A single-system scenario `sc` stepped over the ranks of the default
    process group (or `group`), each rank with its own simulation of `lib`.

    drift: the largest displacement d of a particle between rebuilds (m;
      default half the largest circumscribed radius).  rebuild_every: steps
      between rebuilds (a rebuild also happens as soon as a particle has moved
      more than d).  axis: 0, 1 or 2 (default: the longest side of the
      domain).  memory: contact memory of the initial state (the layout of
      Simulation.contact_memory), or None."""

    def __init__(self, lib, sc, precision, drift=None, rebuild_every=50, axis=None, device=0, group=None,
                 memory=None):
        if len(sc.domains) != 1:
            raise ValueError("a slab run takes one system")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.sc = sc
        dom = sc.domains[0]
        self.axis = int(np.argmax(dom["size"])) if axis is None else int(axis)
        self.lo = float(dom["origin"][self.axis])
        self.hi = self.lo + float(dom["size"][self.axis])
        p = sc.particles
        self.n = len(p["id"])
        rmax = float(np.max(p["radius"]))
        self.drift = 0.5 * rmax if drift is None else float(drift)
        self.halo = 2.0 * rmax + 2.0 * self.drift
        self.rebuild_every = int(rebuild_every)
        self.sim = Simulation(lib, precision, max_particles=self.n, device=device)
        ids = S.setup(self.sim, sc)
        self.static = {k: np.asarray(p[k]) for k in ["id", "material", "radius", "crust", "mass", "inertia"]}
        self.static["shape"] = np.asarray(ids, np.int32)[np.asarray(p["shape"])]
        self.order = np.argsort(self.static["id"], kind="stable")  # particle index by increasing id
        full = {k: np.array(p[k], dtype=np.float64, copy=True) for k, _ in KINEMATIC if k != "basis"}
        full["basis"] = (np.array(p["basis"], dtype=np.float64, copy=True) if p.get("basis") is not None
                         else S.quaternion_basis(np.asarray(p["quaternion"])).reshape(self.n, 9))
        self.has_basis = p.get("basis") is not None
        self.since = 0
        self.rebuilds = 0
        self._build(full, memory)

    # ---- partition -------------------------------------------------------
    def _slabs(self, x):
        """Slab bounds: quantiles of the coordinates, so that each rank owns
        about the same number of particles."""
        q = np.quantile(x, np.arange(1, self.world) / self.world) if self.world > 1 else np.zeros(0)
        return np.concatenate([[-np.inf], q, [np.inf]])

    def _sets(self, x, bounds):
        """Owned and ghost particle indices (increasing id) of every rank."""
        owner = np.searchsorted(bounds, x, side="right") - 1
        owner = np.clip(owner, 0, self.world - 1)
        owned, ghosts = [], []
        for r in range(self.world):
            a, b = bounds[r], bounds[r + 1]
            near = (x >= a - self.halo) & (x < b + self.halo) & (owner != r)
            owned.append(self.order[np.isin(self.order, np.nonzero(owner == r)[0])])
            ghosts.append(self.order[np.isin(self.order, np.nonzero(near)[0])])
        return owned, ghosts

    def _build(self, full, memory):
        """(Re)distributes the particles from the full kinematic state and the
        full contact memory (entries of owned holders, or None at the start)."""
        x = full["position"][:, self.axis]
        self.bounds = self._slabs(x)
        self.owned, self.ghosts = self._sets(x, self.bounds)
        r = self.rank
        self.local = np.concatenate([self.owned[r], self.ghosts[r]])
        self.n_owned = len(self.owned[r])
        pos_of = {int(i): k for k, i in enumerate(self.local)}
        # ghost exchange plan: rows of my local array to send to each rank, in
        # that rank's ghost order; rows of my ghosts received from each rank
        self.send_rows, self.recv_rows = {}, {}
        mine = set(self.owned[r].tolist())
        for s in range(self.world):
            if s == r:
                continue
            out = [i for i in self.ghosts[s].tolist() if i in mine]
            if out:
                self.send_rows[s] = np.array([pos_of[i] for i in out], np.int64)
            theirs = set(self.owned[s].tolist())
            inn = [i for i in self.ghosts[r].tolist() if i in theirs]
            if inn:
                self.recv_rows[s] = np.array([pos_of[i] for i in inn], np.int64)
        loc = {k: v[self.local] for k, v in self.static.items()}
        loc["system"] = None
        for k, _ in KINEMATIC:
            loc[k] = full[k][self.local]
        if not self.has_basis:
            loc["basis"] = None
        self.x0 = full["position"][self.local].copy()
        self.sim.upload(loc)
        if memory is not None and len(memory["owner"]):
            ids = set(self.static["id"][self.local].tolist())
            keep = np.array([(int(o) in ids) and (int(t) < 0 or int(t) in ids)
                             for o, t in zip(memory["owner"], memory["other"])], bool)
            if keep.any():
                self.sim.upload_contact_memory({k: v[keep] for k, v in memory.items()})
        self.since = 0
        self.rebuilds += 1

    # ---- exchanges -------------------------------------------------------
    def _exchange_ghosts(self, st):
        reqs, bufs = [], {}
        for s, rows in self.send_rows.items():
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(_pack(st, rows))), s, group=self.group))
        for s, rows in self.recv_rows.items():
            bufs[s] = torch.empty((len(rows), WIDTH), dtype=torch.float64)
            reqs.append(dist.irecv(bufs[s], s, group=self.group))
        for q in reqs:
            q.wait()
        for s, rows in self.recv_rows.items():
            _unpack(st, rows, bufs[s].numpy())

    def _write_ghosts(self, st):
        """The received ghost states into the simulation: only the ghost rows
        where the library can (grains_gpu_update_particle_rows), else the
        whole state written back."""
        fields = ["position", "quaternion", "velocity", "omega"] + (["basis"] if self.has_basis else [])
        if "update_particle_rows" in self.sim.lib.fn:
            rows = np.concatenate(list(self.recv_rows.values())) if self.recv_rows else np.zeros(0, np.int64)
            if len(rows):
                self.sim.update_rows(rows, {k: st[k][rows] for k in fields})
        else:
            self.sim.update({k: st[k] for k in fields})

    def _gather_full(self, st):
        """The kinematic state of every particle (index order) from the owners."""
        mine = (self.owned[self.rank], _pack(st, np.arange(self.n_owned)))
        parts = [None] * self.world
        dist.all_gather_object(parts, mine, group=self.group)
        full = {k: np.zeros((self.n, w)) for k, w in KINEMATIC}
        for idx, data in parts:
            rows = {k: np.zeros((len(idx), w)) for k, w in KINEMATIC}
            _unpack(rows, np.arange(len(idx)), data)
            for k, _ in KINEMATIC:
                full[k][idx] = rows[k]
        full["quaternion"] = full["quaternion"].reshape(self.n, 4)
        return full

    def _gather_memory(self):
        m = self.sim.contact_memory()
        owned_ids = set(self.static["id"][self.owned[self.rank]].tolist())
        keep = np.array([int(o) in owned_ids for o in m["owner"]], bool)
        mine = {k: v[keep] for k, v in m.items()}
        parts = [None] * self.world
        dist.all_gather_object(parts, mine, group=self.group)
        return {k: np.concatenate([q[k] for q in parts]) for k in mine}

    def _moved_too_far(self, st):
        d = np.max(np.abs(st["position"][:self.n_owned] - self.x0[:self.n_owned]), initial=0.0)
        flag = torch.tensor([1 if d > self.drift else 0], dtype=torch.int32)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=self.group)
        return bool(flag.item())

    # ---- the run ---------------------------------------------------------
    def initialize_leapfrog(self, time, dt):
        self.sim.initialize_leapfrog(time, dt)

    def step(self, n_steps, time, dt):
        """n_steps kick-drift-kick steps of Grains::Simulation (Grains.cpp:
        344-364) on every rank, with the ghost exchange after the move."""
        for _ in range(n_steps):
            time += dt
            self.sim.move(time, 0.5 * dt, dt)
            st = self.sim.download()
            self.since += 1
            if self.since >= self.rebuild_every or self._moved_too_far(st):
                full = self._gather_full(st)
                memory = self._gather_memory()
                self._build(full, memory)
            else:
                self._exchange_ghosts(st)
                self._write_ghosts(st)
            self.sim.link_update(time, dt)
            self.sim.compute_forces(time, dt)
            self.sim.advance_velocity(time, 0.5 * dt)
        return time

    def gather(self):
        """The state of every particle in the scenario's order (on every rank):
        position, quaternion, basis, velocity, omega, force, torque and
        coordination, each from the particle's owner."""
        st = self.sim.download()
        cols = [("force", 3), ("torque", 3)]
        extra = np.concatenate([st[k][:self.n_owned] for k, _ in cols] +
                               [st["coordination"][:self.n_owned, None].astype(np.float64)], axis=1)
        mine = (self.owned[self.rank], _pack(st, np.arange(self.n_owned)), extra)
        parts = [None] * self.world
        dist.all_gather_object(parts, mine, group=self.group)
        out = {k: np.zeros((self.n, w)) for k, w in KINEMATIC + cols}
        out["coordination"] = np.zeros(self.n, np.int32)
        for idx, data, ex in parts:
            rows = {k: np.zeros((len(idx), w)) for k, w in KINEMATIC}
            _unpack(rows, np.arange(len(idx)), data)
            for k, _ in KINEMATIC:
                out[k][idx] = rows[k]
            out["force"][idx] = ex[:, 0:3]
            out["torque"][idx] = ex[:, 3:6]
            out["coordination"][idx] = ex[:, 6].astype(np.int32)
        return out

    def close(self):
        self.sim.close()
