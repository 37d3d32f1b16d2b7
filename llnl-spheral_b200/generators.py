"""Seeded synthetic node sets with the shapes of the benchmark configurations.

Lattices follow GenerateNodeDistribution3d.latticeDistribution
(src/NodeGenerators/GenerateNodeDistribution3d.py:573-621): node centres at
xmin + (i + 1/2) dx with x varying fastest, H = diag(1/(nPerh dx), ...),
mass = rho(x) dx dy dz.  Positions are then jittered by a uniform +-f*dx per
component from a seeded PCG64 stream.  Every array is AoS in the reference's
Field order (Vector: x,y,z; SymTensor: xx,xy,xz,yy,yz,zz).
"""
import numpy as np


class NodeSet:
    """AoS arrays of one FluidNodeList's internal nodes."""

    def __init__(self, pos, vel, mass, rho, eps, H, dx):
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.vel = np.ascontiguousarray(vel, dtype=np.float64)
        self.mass = np.ascontiguousarray(mass, dtype=np.float64)
        self.rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.eps = np.ascontiguousarray(eps, dtype=np.float64)
        self.H = np.ascontiguousarray(H, dtype=np.float64)
        self.dx = dx

    @property
    def n(self):
        return self.mass.shape[0]


def lattice(nx, ny, nz, xmin, xmax, nPerh, jitter=0.01, seed=20261203):
    xmin = np.asarray(xmin, dtype=np.float64)
    xmax = np.asarray(xmax, dtype=np.float64)
    d = (xmax - xmin) / np.array([nx, ny, nz], dtype=np.float64)
    n = nx * ny * nz
    ig = np.arange(n, dtype=np.int64)
    i = ig % nx
    j = (ig // nx) % ny
    k = ig // (nx * ny)
    lat = np.empty((n, 3))
    lat[:, 0] = xmin[0] + (i + 0.5) * d[0]
    lat[:, 1] = xmin[1] + (j + 0.5) * d[1]
    lat[:, 2] = xmin[2] + (k + 0.5) * d[2]
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = lat + rng.uniform(-jitter, jitter, size=(n, 3)) * d[None, :]
    H = np.zeros((n, 6))
    H[:, 0] = 1.0 / (nPerh * d[0])
    H[:, 3] = 1.0 / (nPerh * d[1])
    H[:, 5] = 1.0 / (nPerh * d[2])
    return lat, pos, H, d


def sod(nx=256, ny=32, nz=32, nPerh=1.51, gamma=5.0 / 3.0, rho1=1.0, P1=1.0, rho2=0.25, P2=0.1795,
        box=((0.0, 0.0, 0.0), (1.0, 0.125, 0.125)), jitter=0.01, seed=20261203, xsplit=None):
    """Planar Sod-type shock tube along x (benchmark configuration 1 at defaults)."""
    xmin, xmax = box
    lat, pos, H, d = lattice(nx, ny, nz, xmin, xmax, nPerh, jitter, seed)
    if xsplit is None:
        xsplit = 0.5 * (xmin[0] + xmax[0])
    left = lat[:, 0] < xsplit
    rho = np.where(left, rho1, rho2)
    P = np.where(left, P1, P2)
    mass = rho * d[0] * d[1] * d[2]
    eps = P / ((gamma - 1.0) * rho)
    vel = np.zeros_like(pos)
    return NodeSet(pos, vel, mass, rho, eps, H, d)


def kelvin_helmholtz(nx=128, ny=128, nz=128, nPerh=1.35, gamma=5.0 / 3.0, rho_in=2.0, rho_out=1.0,
                     vx_in=0.5, vx_out=-0.5, P=2.5, amp=0.01, width=0.05, jitter=0.01, seed=20261203,
                     box=((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))):
    """3-D Kelvin-Helmholtz in a periodic box (benchmark configurations 2/3 at defaults)."""
    xmin, xmax = box
    lat, pos, H, d = lattice(nx, ny, nz, xmin, xmax, nPerh, jitter, seed)
    ly = xmax[1] - xmin[1]
    y = (lat[:, 1] - xmin[1]) / ly
    inside = np.abs(y - 0.5) < 0.25
    rho = np.where(inside, rho_in, rho_out)
    vel = np.zeros_like(pos)
    vel[:, 0] = np.where(inside, vx_in, vx_out)
    xs = (lat[:, 0] - xmin[0]) / (xmax[0] - xmin[0])
    env = np.exp(-((y - 0.25) ** 2) / (2.0 * width ** 2)) + np.exp(-((y - 0.75) ** 2) / (2.0 * width ** 2))
    vel[:, 1] = amp * np.sin(4.0 * np.pi * xs) * env
    mass = rho * d[0] * d[1] * d[2]
    eps = P / ((gamma - 1.0) * rho)
    return NodeSet(pos, vel, mass, rho, eps, H, d)


def sod_config(abi, ns_box=((0.0, 0.0, 0.0), (1.0, 0.125, 0.125)), **kw):
    """Switches of benchmark configuration 1 (Sod, cubic B-spline, fixed dt 1e-4)."""
    base = dict(kernel=abi.KERNEL_BSPLINE, nPerh=1.51, Cl=1.0, Cq=1.0, gamma=5.0 / 3.0,
                xmin=ns_box[0], xmax=ns_box[1], dtMin=1.0e-4, dtMax=1.0e-4)
    base.update(kw)
    return abi.make_config(**base)


def kh_config(abi, **kw):
    """Switches of benchmark configuration 2 (KH, Wendland C4, Courant dt)."""
    base = dict(kernel=abi.KERNEL_WENDLANDC4, nPerh=1.35, Cl=1.0, Cq=1.0, gamma=5.0 / 3.0,
                xmin=(0.0, 0.0, 0.0), xmax=(1.0, 1.0, 1.0), dtMin=0.0, dtMax=0.1)
    base.update(kw)
    return abi.make_config(**base)
