"""Velocity sharding of one kinetic case over several backends, one per GPU (no reference counterpart).

Within one CIS sweep the discrete velocities are independent given the Shakhov target, the inflow states and the
wall densities (the reference's spec, docs/spec.md:98-99), so a case splits into contiguous ranges of the storage
order, each held by its own backend. The ranges are aligned to the mirror orbits of symmetry planes, so a symmetry
face finds its mirrored velocity in its own shard. What couples the shards is reduced across them:
* the 13 moment sums of every cell (added, then finalised once, kin_moment_sums / kin_set_moments);
* the 20 boundary sums of every boundary face, the per-cell residual sums and internal-face mass fluxes (added);
* the discrete equilibrium is solved by every shard on the full grid (KinSetupDesc.deq_*), which needs no f.

`ShardedBackend` presents the shards as one backend with the methods `KineticSolver` calls, so the host loop runs
unchanged. Its shards are either all in this process (a list of backends) or one per rank of a process group
(`allreduce(a, op)` reduces a NumPy array over the ranks with op "sum" or "min", e.g. `torch_allreduce()`).
The GSIS correction's negativity rules reduce over all velocities of a cell: it runs in two phases, the per-cell
extrema of every shard reduced with a minimum in between (kin_gsis_correction_extrema / _apply). Maxwell walls with
a non-mirror reflection are not sharded (their reflection may leave the shard).
"""
from __future__ import annotations

import numpy as np

from . import abi

MOMENT_SUMS = 13


def finalize_moments(sums: np.ndarray, weight: float, shift: np.ndarray) -> np.ndarray:
    """15 moments per cell from the 13 shifted sums (finalize_moments, kinetic_kernels.hpp:382-442)."""
    s = np.asarray(sums, float).reshape(-1, MOMENT_SUMS)
    out = np.zeros((len(s), 15))
    s0 = s[:, 0]
    pos = s0 > 0.0
    out[~pos, 0] = weight * s0[~pos]
    t = s[pos]
    u0 = shift[pos]
    s0 = t[:, 0]
    dx, dy, dz = t[:, 1] / s0, t[:, 2] / s0, t[:, 3] / s0
    rho = weight * s0
    pxx = weight * (t[:, 4] - s0 * dx * dx)
    pyy = weight * (t[:, 5] - s0 * dy * dy)
    pzz = weight * (t[:, 6] - s0 * dz * dz)
    pxy = weight * (t[:, 7] - s0 * dx * dy)
    pyz = weight * (t[:, 8] - s0 * dy * dz)
    pxz = weight * (t[:, 9] - s0 * dx * dz)
    p = (pxx + pyy + pzz) / 3.0
    tr2 = t[:, 4] + t[:, 5] + t[:, 6]
    du2 = dx * dx + dy * dy + dz * dz
    s2dx = t[:, 4] * dx + t[:, 7] * dy + t[:, 9] * dz
    s2dy = t[:, 7] * dx + t[:, 5] * dy + t[:, 8] * dz
    s2dz = t[:, 9] * dx + t[:, 8] * dy + t[:, 6] * dz
    out[pos] = np.stack([rho, u0[:, 0] + dx, u0[:, 1] + dy, u0[:, 2] + dz, p / rho, p, pxx - p, pyy - p, pzz - p,
                         pxy, pyz, pxz,
                         0.5 * weight * (t[:, 10] - dx * tr2 - 2.0 * s2dx + 2.0 * s0 * du2 * dx),
                         0.5 * weight * (t[:, 11] - dy * tr2 - 2.0 * s2dy + 2.0 * s0 * du2 * dy),
                         0.5 * weight * (t[:, 12] - dz * tr2 - 2.0 * s2dz + 2.0 * s0 * du2 * dz)], 1)
    return out


def orbit_size(setup: abi.SetupArrays) -> int:
    x = setup["bface_mirror_xor"]
    return 1 + (int(np.bitwise_or.reduce(x)) if x is not None and len(x) else 0)


def shard_ranges(setup: abi.SetupArrays, n: int) -> list:
    """n contiguous velocity ranges of the storage order, as equal as whole mirror orbits allow."""
    nv, orb = setup.nv, orbit_size(setup)
    units = nv // orb
    if n < 1 or n > units:
        raise ValueError(f"cannot split {nv} velocities ({units} mirror orbits) into {n} shards")
    cuts = [orb * (units * k // n) for k in range(n + 1)]
    return [(cuts[k], cuts[k + 1]) for k in range(n)]


def shard_setup(setup: abi.SetupArrays, lo: int, hi: int) -> abi.SetupArrays:
    """The set-up of the velocity range [lo, hi): the range's velocities, the full grid for the equilibrium."""
    if int(setup.scalars.get("n_maxwell_faces", 0) or 0) > 0:
        raise ValueError("velocity sharding does not handle Maxwell walls (their reflection may leave the shard)")
    s = setup.copy()
    for k in ("xi_x", "xi_y", "xi_z", "weights", "sweep_dir_of"):
        a = setup.arrays.get(k)
        s[k] = None if a is None else np.ascontiguousarray(a[lo:hi])
    s.scalars["nv"] = hi - lo
    s.scalars["deq_nv"] = setup.nv
    s["deq_xi_x"], s["deq_xi_y"], s["deq_xi_z"] = setup["xi_x"], setup["xi_y"], setup["xi_z"]
    s["deq_weights"] = setup.arrays.get("weights")
    return s


def torch_allreduce(group=None, device="cpu"):
    """An all-reduce (op "sum" or "min") of NumPy arrays over a torch.distributed process group (gloo on CPU, or NCCL
    with device="cuda"); every rank must call it in the same order."""
    import torch
    import torch.distributed as dist

    ops = {"sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN}

    def reduce(a: np.ndarray, op: str = "sum") -> np.ndarray:
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(device)
        dist.all_reduce(t, op=ops[op], group=group)
        return t.cpu().numpy().reshape(a.shape)

    return reduce


def torch_device_allreduce(group=None):
    """An in-place sum all-reduce of a CUDA tensor over a torch.distributed process group (NCCL over NVLink): the
    device data plane of ShardedBackend(device_allreduce=...)."""
    import torch.distributed as dist

    def reduce(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    return reduce


class ShardedBackend:
    """Velocity shards presented as one kinetic backend (the methods KineticSolver uses).

    device=True (B200 shards): the moment sums, boundary sums and per-cell residual sums are reduced in device
    memory: the local shards' device buffers are added on the device, `device_allreduce` (e.g.
    torch_device_allreduce(), NCCL) reduces them across ranks in place, and the moments are finalised on the device
    (kin_moment_sums / kin_boundary_sums / kin_sweep with NULL outputs, kin_device_sums, kin_finalize_moments)."""

    def __init__(self, setup: abi.SetupArrays, backends: list, ranges: list, allreduce=None, device=False,
                 device_allreduce=None):
        self.setup = setup
        self.backends = list(backends)
        self.ranges = list(ranges)
        self.allreduce = allreduce
        self.device = device
        self.device_allreduce = device_allreduce
        self.n_cells, self.nv, self.n_bfaces = setup.n_cells, setup.nv, setup.n_bfaces
        self.weight = float(setup.scalars["weight"]) if setup.arrays.get("weights") is None else 1.0
        self.shift = np.zeros((self.n_cells, 3))

    def _sum(self, arrays):
        total = arrays[0].copy()
        for a in arrays[1:]:
            total += a
        return self.allreduce(total) if self.allreduce is not None else total

    def _device_reduce(self, which):
        """Sum the local shards' device buffers of one kind into every one of them, then across ranks (in place)."""
        import torch

        ts = [be.device_sums(which) for be in self.backends]
        total = ts[0]
        for t in ts[1:]:
            total.add_(t.to(total.device))
        if self.device_allreduce is not None:
            self.device_allreduce(total)
        for t in ts[1:]:
            t.copy_(total.to(t.device))
        for t in ts:
            torch.cuda.synchronize(t.device)
        return ts

    def _min(self, arrays):
        low = arrays[0].copy()
        for a in arrays[1:]:
            np.minimum(low, a, out=low)
        return self.allreduce(low, "min") if self.allreduce is not None else low

    # --- KineticBackend methods ------------------------------------------------------------------------------
    def set_equilibrium(self, states):
        st = np.asarray(states, float).reshape(self.n_cells, 5)
        for be in self.backends:
            be.set_equilibrium(st)
        self.shift = st[:, 1:4].copy()

    def compute_moments(self):
        if self.device:
            for be in self.backends:
                be.moment_sums_to_device()
            self._device_reduce(abi.KIN_SUMS_MOMENTS)
            m = self.backends[0].finalize_moments()
            for be in self.backends[1:]:
                be.finalize_moments()
            pos = m[:, 0] > 0.0
            self.shift[pos] = m[pos, 1:4]
            return m
        sums = self._sum([be.moment_sums() for be in self.backends])
        m = finalize_moments(sums, self.weight, self.shift)
        for be in self.backends:
            be.set_moments(m)
        pos = m[:, 0] > 0.0
        self.shift[pos] = m[pos, 1:4]
        return m

    def scale_distribution(self, s):
        for be in self.backends:
            be.scale_distribution(s)

    def update_cell_params(self):
        for be in self.backends:
            be.update_cell_params()

    def deq_counts(self):
        return self.backends[0].deq_counts()

    def set_inflow(self, inflow):
        for be in self.backends:
            be.set_inflow(inflow)

    def boundary_sums(self):
        if self.device:
            for be in self.backends:
                be.boundary_sums_to_device()
            self._device_reduce(abi.KIN_SUMS_BOUNDARY)
            out = self.backends[0].read_sums(abi.KIN_SUMS_BOUNDARY, 20 * self.n_bfaces)
            return out.reshape(self.n_bfaces, abi.BOUNDARY_SUMS_PER_FACE)
        return self._sum([be.boundary_sums() for be in self.backends])

    def sweep(self):
        if self.device:
            for be in self.backends:
                be.sweep_to_device()
            self._device_reduce(abi.KIN_SUMS_RESIDUAL)
            return self.backends[0].read_sums(abi.KIN_SUMS_RESIDUAL, self.n_cells)
        return self._sum([be.sweep() for be in self.backends])

    def internal_face_mass_flux(self, cells, entries):
        return self._sum([be.internal_face_mass_flux(cells, entries) for be in self.backends])

    def discrete_maxwell(self, states, tolerance):
        return self.backends[0].discrete_maxwell(states, tolerance)

    def get_distribution(self):
        if self.allreduce is not None:
            raise NotImplementedError("the distribution of a sharded case across ranks is not gathered")
        return np.concatenate([be.get_distribution() for be in self.backends], axis=1)

    def set_distribution(self, f):
        if self.allreduce is not None:
            raise NotImplementedError("the distribution of a sharded case across ranks is not scattered")
        f = np.asarray(f, float).reshape(self.n_cells, self.nv)
        for be, (lo, hi) in zip(self.backends, self.ranges):
            be.set_distribution(np.ascontiguousarray(f[:, lo:hi]))

    def gsis_correction(self, w_half, w_new):
        """GSIS correction of every shard: the per-cell extrema of the negativity rule reduced over all shards
        (minimum), then applied by each shard; every shard reaches the same per-cell decision."""
        ext = self._min([be.gsis_correction_extrema(w_half, w_new) for be in self.backends])
        out = [be.gsis_correction_apply(w_half, w_new, ext) for be in self.backends]
        self.shift = np.asarray(w_new, float).reshape(self.n_cells, 5)[:, 1:4].copy()
        flags = out[0][1]
        skipped = flags == 2
        if skipped.any():
            self.shift[skipped] = np.asarray(w_half, float).reshape(self.n_cells, 5)[skipped, 1:4]
        return out[0][0], flags

    def launch_count(self):
        return sum(be.launch_count() for be in self.backends)

    def close(self):
        for be in self.backends:
            be.close()

    def take_timings(self):
        out = {}
        for be in self.backends:
            for k, v in be.take_timings().items():
                out[k] = out.get(k, 0.0) + v
        return out
