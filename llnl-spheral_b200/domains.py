"""Slab domain decomposition of one problem over ranks (one GPU each).

The reference splits a problem into domains with DistributedBoundary
(src/Distributed/DistributedBoundary.cc; setGhostNodes at :1183 builds the
domain ghost nodes, the remote nodes a domain's internal nodes interact
with, and applyGhostBoundaries exchanges their Field values at every stage
of the integrator) and NestedGridDistributedBoundary
(src/Distributed/NestedGridDistributedBoundary.cc), which picks the domain
ghosts from each domain's occupied grid cells.

Here a rank owns the nodes of one slab of the periodic box along x and
keeps their state and derivatives.  Once per RK2 step it receives the
halo: every remote node within `depth` kernel reaches (kernel extent x the
largest h of the problem) of its slab, with that node's state and
derivatives.  The halo is deep enough that the whole CheapSynchronousRK2
step runs on the rank's own nodes plus the halo without another exchange:
a node k reaches from the slab has complete rows, and so correct mid-point
state, evaluation and end state, while k + 1 <= depth; the rank's nodes need
their neighbors' mid-point derivatives (compatible energy) and end state
(sum density), which needs two reaches, three with grad-h (the neighbors'
omega), four with CRKSPH (the corrections of the neighbors' neighbors, and
the sum volume before the sum density).  Halo rows are computed and
discarded.  So a step costs one halo exchange and one allreduce(MIN) for
the time step instead of the reference's exchange per stage, in exchange for
the redundant work on the halo.  The time step is the minimum of the
domains' votes (Integrator::selectDt over all domains); each domain then
takes the step with that dt imposed through the dt bounds.

Neighbor sets are the single-domain ones (the same exact predicate on the
same positions and H; compared as global node and periodic image), and the
states stay within 1e-12 of a single-domain run: only the order of the
pair sums differs (a domain numbers its nodes owned first, then halo).

Ownership is fixed (no node redistribution): the slab a rank reports is its
nominal slab widened by the farthest of its nodes outside it.
"""
import numpy as np

from . import abi
from .hydro import SPHHydro

# StateDerivatives a step reads before it recomputes them (the time-step vote
# and the mid-point advance): all of them, by the keys of distinct fields.
DERIV_KEYS = [("delta position", 3), ("delta velocity hydro", 3), ("delta mass density", 1),
              ("delta specific thermal energy", 1), ("delta H", 6), ("new H", 6), ("velocity gradient", 9),
              ("M SPH gradient correction", 9), ("new mass density", 1), ("normalization", 1),
              ("weighted neighbor sum", 1), ("mass second moment", 6), ("XSPH weight sum", 1),
              ("XSPH delta vi", 3), ("max viscous pressure", 1), ("effective viscous pressure", 1),
              ("viscous work rate", 1)]
STATE_KEYS = [("position", 3), ("velocity", 3), ("mass", 1), ("mass density", 1),
              ("specific thermal energy", 1), ("H", 6)]
# one exchanged node: global id, state, derivatives, CRKSPH node volume
ROW = 1 + sum(c for _, c in STATE_KEYS) + sum(c for _, c in DERIV_KEYS) + 1
KERNEL_EXTENT = 2.0          # the B-spline and Wendland C4 TableKernels


def halo_depth(cfg):
    """Kernel reaches of halo a whole RK2 step needs."""
    if cfg.hydro == abi.HYDRO_CRKSPH:
        return 4
    return 3 if cfg.gradhCorrection else 2


def slab_of(x, world, lo, hi):
    """Owner rank of each x: equal slabs of [lo, hi) along x."""
    k = np.floor((np.asarray(x) - lo) / (hi - lo) * world).astype(np.int64)
    return np.clip(k, 0, world - 1)


def periodic_gap(x, a, b, length):
    """Distance along a periodic axis of length `length` from x to the
    interval [a, b) (0 inside)."""
    x = np.asarray(x, dtype=np.float64)
    below = np.mod(a - x, length)
    above = np.mod(x - b, length)
    inside = (np.mod(x - a, length) < (b - a))
    return np.where(inside, 0.0, np.minimum(below, above))


def max_h(H):
    """Largest smoothing scale 1/min eig(H) of SymTensor rows (xx xy xz yy yz zz)."""
    H = np.asarray(H, dtype=np.float64).reshape(-1, 6)
    if H.shape[0] == 0:
        return 0.0
    M = np.empty((H.shape[0], 3, 3))
    M[:, 0, 0], M[:, 0, 1], M[:, 0, 2] = H[:, 0], H[:, 1], H[:, 2]
    M[:, 1, 0], M[:, 1, 1], M[:, 1, 2] = H[:, 1], H[:, 3], H[:, 4]
    M[:, 2, 0], M[:, 2, 1], M[:, 2, 2] = H[:, 2], H[:, 4], H[:, 5]
    return float(np.max(1.0 / np.linalg.eigvalsh(M)[:, 0]))


class SlabDomain:
    """The nodes one rank owns, their state and derivatives on the host
    between steps, and one RK2 step of them with a received halo.

    The methods are the phases of a step; SlabDecomposition runs them for
    ranks emulated in one process, DistributedSlabs for one rank per process
    with torch.distributed collectives."""

    def __init__(self, cfg, rank, world, gid, state, derivs=None, volume=None):
        self.cfg = cfg.copy()
        self.rank, self.world = rank, world
        self.gid = np.asarray(gid, dtype=np.int64)
        self.state = {k: np.array(v, dtype=np.float64).reshape(self.gid.size, c)
                      for (k, c), v in zip(STATE_KEYS, state)}
        n = self.gid.size
        self.derivs = derivs or {k: np.zeros((n, c)) for k, c in DERIV_KEYS}
        self.volume = np.zeros(n) if volume is None else np.asarray(volume, dtype=np.float64)
        self.time = 0.0
        self.last_dt = cfg.lastDt
        self.cycle = 0
        self.have_volume = volume is not None
        self.local = None          # the rank's problem of the current step (owned + halo)
        self.halo_gid = np.zeros(0, dtype=np.int64)
        lo, hi = cfg.xmin[0], cfg.xmax[0]
        w = (hi - lo) / world
        self.slab = (lo + rank * w, lo + (rank + 1) * w)

    @property
    def n(self):
        return self.gid.size

    # ---- phase 1: what the others need to know to pick the halo
    def extent(self):
        """[slab lo, slab hi (widened by the farthest owned node outside it),
        largest h]."""
        lo, hi = self.slab
        L = self.cfg.xmax[0] - self.cfg.xmin[0]
        gap = periodic_gap(self.state["position"][:, 0], lo, hi, L)
        widen = float(gap.max()) if self.n else 0.0
        return np.array([lo - widen, hi + widen, max_h(self.state["H"])])

    # ---- phase 2: rows for every other rank
    def rows(self, idx):
        out = np.empty((idx.size, ROW))
        out[:, 0] = self.gid[idx]
        c = 1
        for k, w in STATE_KEYS:
            out[:, c:c + w] = self.state[k][idx]
            c += w
        for k, w in DERIV_KEYS:
            out[:, c:c + w] = self.derivs[k][idx]
            c += w
        out[:, c] = self.volume[idx]
        return out

    def sends(self, extents):
        """extents: (world, 3) from phase 1.  Rows this rank sends to each rank
        (its nodes within the halo depth of that rank's slab)."""
        reach = KERNEL_EXTENT * float(np.max(extents[:, 2]))
        width = halo_depth(self.cfg) * reach
        L = self.cfg.xmax[0] - self.cfg.xmin[0]
        x = self.state["position"][:, 0]
        out = []
        for s in range(self.world):
            if s == self.rank:
                out.append(np.zeros((0, ROW)))
                continue
            sel = np.nonzero(periodic_gap(x, extents[s, 0], extents[s, 1], L) <= width)[0]
            out.append(self.rows(sel))
        return out

    # ---- phase 3: the rank's problem, owned nodes first, then the halo
    def build_local(self, received):
        halo = np.concatenate([r for r in received if r.size] or [np.zeros((0, ROW))])
        halo = halo[np.argsort(halo[:, 0], kind="stable")]
        self.halo_gid = halo[:, 0].astype(np.int64)
        rows = np.concatenate([self.rows(np.arange(self.n)), halo])
        n = rows.shape[0]
        cols = {}
        c = 1
        for k, w in STATE_KEYS + DERIV_KEYS:
            cols[k] = rows[:, c:c + w]
            c += w
        vol = rows[:, c]
        cfg = self.cfg.copy()
        cfg.lastDt = self.last_dt

        class Nodes:
            pass
        nodes = Nodes()
        nodes.n = n
        nodes.pos, nodes.vel = cols["position"], cols["velocity"]
        nodes.mass, nodes.rho = cols["mass"].ravel(), cols["mass density"].ravel()
        nodes.eps, nodes.H = cols["specific thermal energy"].ravel(), cols["H"]
        if self.local is not None:
            self.local.close()
        self.local = SPHHydro(cfg, nodes)
        self.local.time = self.time
        for k, _ in DERIV_KEYS:
            self.local.set_field(k, cols[k])
        if cfg.hydro == abi.HYDRO_CRKSPH and self.have_volume:
            self.local.set_field("node volume", vol)
        self.local.build_neighbors()

    # ---- phase 4: the domain's time-step vote (GenericHydro::dt)
    def vote(self):
        return self.local.dt()

    # ---- phase 5: one RK2 step with the agreed dt; keep the owned results
    def advance(self, dt):
        self.local.set_dt_bounds(dt, dt)
        t, last = self.local.step(1)
        self._keep()
        self.time, self.last_dt = t, last
        self.cycle += 1
        return t, last

    def evaluate(self):
        """Physics::initialize + evaluateDerivatives of the owned nodes at the
        current state (the controller's start-up evaluation)."""
        self.local.initialize(self.time)
        self.local.evaluateDerivatives(self.time)
        self._keep()

    def _keep(self):
        n = self.n
        for k, _ in STATE_KEYS:
            self.state[k] = self.local.field(k).reshape(self.local.n, -1)[:n].copy()
        for k, _ in DERIV_KEYS:
            self.derivs[k] = self.local.field(k).reshape(self.local.n, -1)[:n].copy()
        if self.cfg.hydro == abi.HYDRO_CRKSPH:
            self.volume = self.local.field("node volume")[:n].copy()
            self.have_volume = True

    def rows_global(self):
        """The owned rows of the current connectivity as sorted lists of
        (global node, periodic image code): image code = the rounded shift
        of the ghost's position from its root in box lengths."""
        off, nb, root = self.local.connectivity()
        gpos = self.local.ghost_positions()
        pos = self.local.field("position")
        all_gid = np.concatenate([self.gid, self.halo_gid])
        L = np.array(self.cfg.xmax) - np.array(self.cfg.xmin)
        nl = self.local.n
        out = []
        for i in range(self.n):
            row = []
            for j in nb[off[i]:off[i + 1]]:
                if j < nl:
                    row.append((int(all_gid[j]), 0, 0, 0))
                else:
                    r = int(root[j - nl])
                    s = np.rint((gpos[j - nl] - pos[r]) / L).astype(int)
                    row.append((int(all_gid[r]), int(s[0]), int(s[1]), int(s[2])))
            out.append(sorted(row))
        return out

    def close(self):
        if self.local is not None:
            self.local.close()
            self.local = None


def split(cfg, nodes, world):
    """The nodes of each slab: (global ids, state arrays) per rank."""
    owner = slab_of(nodes.pos[:, 0], world, cfg.xmin[0], cfg.xmax[0])
    parts = []
    for r in range(world):
        gid = np.nonzero(owner == r)[0]
        parts.append((gid, [nodes.pos[gid], nodes.vel[gid], nodes.mass[gid], nodes.rho[gid],
                            nodes.eps[gid], nodes.H[gid]]))
    return parts


class SlabDecomposition:
    """`world` slab domains of one problem in one process (one device): the
    exchange is a transpose of the per-rank send lists.  The phases and the
    data are those of DistributedSlabs, one rank per process."""

    def __init__(self, cfg, nodes, world):
        self.domains = [SlabDomain(cfg, r, world, gid, st) for r, (gid, st) in enumerate(split(cfg, nodes, world))]
        self.world = world

    def _exchange(self):
        ext = np.stack([d.extent() for d in self.domains])
        sends = [d.sends(ext) for d in self.domains]
        for r, d in enumerate(self.domains):
            d.build_local([sends[s][r] for s in range(self.world)])

    def initialize(self):
        """The start-up connectivity and one evaluation at the start time."""
        self._exchange()
        for d in self.domains:
            d.evaluate()

    def step(self, nsteps=1):
        for _ in range(nsteps):
            self._exchange()
            vote = min(d.vote() for d in self.domains)
            dt = select_dt(self.domains[0].cfg, vote, self.domains[0].last_dt)
            for d in self.domains:
                d.advance(dt)

    def field(self, key, n):
        """A field of all nodes in global order."""
        out = None
        for d in self.domains:
            v = d.state[key] if key in d.state else d.derivs[key]
            if out is None:
                out = np.zeros((n, v.shape[1]))
            out[d.gid] = v
        return out

    def close(self):
        for d in self.domains:
            d.close()


def select_dt(cfg, vote, last_dt):
    """Integrator::selectDt from the smallest domain vote (the device
    select_dt_kernel's arithmetic)."""
    dt = cfg.dtMax
    if 0.0 < vote < dt:
        dt = vote
    dt = min(dt, cfg.dtGrowth * last_dt)
    return min(cfg.dtMax, max(cfg.dtMin, dt))


class DistributedSlabs:
    """One slab domain per process over torch.distributed: the extents by
    all_gather, the halo rows by point-to-point send/recv (tensors on the
    device with NCCL, on the host with gloo), the time step by
    all_reduce(MIN).  Every rank takes the same collective steps in the same
    order."""

    def __init__(self, cfg, nodes, group=None, device=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = device or "cpu"
        gid, st = split(cfg, nodes, self.world)[self.rank]
        self.domain = SlabDomain(cfg, self.rank, self.world, gid, st)

    def _tensor(self, a):
        import torch
        return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=self.device)

    def _exchange(self):
        self.domain.build_local(self.exchange_rows())

    def exchange_rows(self):
        """The halo rows this rank receives, one array per source rank."""
        import torch
        dist = self.dist
        mine = self._tensor(self.domain.extent())
        ext = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(ext, mine, group=self.group)
        ext = np.stack([e.cpu().numpy() for e in ext])
        sends = self.domain.sends(ext)
        counts = self._tensor([s.shape[0] for s in sends])
        allc = [torch.empty_like(counts) for _ in range(self.world)]
        dist.all_gather(allc, counts, group=self.group)
        incoming = [int(allc[s][self.rank].item()) for s in range(self.world)]
        reqs, bufs = [], []
        for s in range(self.world):
            if s == self.rank:
                bufs.append(None)
                continue
            buf = torch.empty((incoming[s], ROW), dtype=torch.float64, device=self.device)
            bufs.append(buf)
            if incoming[s]:
                reqs.append(dist.irecv(buf, src=s, group=self.group))
        outs = [self._tensor(sends[s]) for s in range(self.world)]
        for s in range(self.world):
            if s != self.rank and sends[s].shape[0]:
                reqs.append(dist.isend(outs[s], dst=s, group=self.group))
        for r in reqs:
            r.wait()
        return [np.zeros((0, ROW)) if b is None else b.cpu().numpy() for b in bufs]

    def initialize(self):
        self._exchange()
        self.domain.evaluate()

    def step(self, nsteps=1):
        import torch
        for _ in range(nsteps):
            self._exchange()
            v = self._tensor([self.domain.vote()])
            self.dist.all_reduce(v, op=self.dist.ReduceOp.MIN, group=self.group)
            dt = select_dt(self.domain.cfg, float(v.item()), self.domain.last_dt)
            self.domain.advance(dt)

    def close(self):
        self.domain.close()
