"""Octree node tables (HyperTreeBaseImpl, src/structure/HyperTree.h:98-243).

Construction follows HyperTree.cpp:11-132: breadth-first node ids, root 0 is
[-1,1]^3, child i of a node takes the upper half on axis k when bit k of i is
set; every coordinate is produced by float32 midpoints, so all boxes lie on
the dyadic plane grid of the tree depth.  SetActive/UpdateActive follow
HyperTree.cpp:163-206: active ids ascending, node_active_prefix_sum[n] is the
node's grid row or -1.

The tables are built on the host (the reference builds them on the CPU too);
device copies feed the CUDA kernels.
"""
import heapq

import numpy as np
import torch

from . import _lib


class HyperTreeBase:
    def __init__(self, d=3, max_depth=4):
        if d != 3:
            raise ValueError("only the 3-D tree is implemented (the reference dispatches D=3 only)")
        if not 1 <= max_depth <= 7:
            raise ValueError("max_depth must be in [1, 7]")
        self.D = d
        self.max_depth = max_depth
        ns = 1 << d
        n = sum(ns ** i for i in range(max_depth + 1))
        pmin = np.empty((n, 3), np.float32)
        pmax = np.empty((n, 3), np.float32)
        depth = np.zeros(n, np.int32)
        parent = np.full(n, -1, np.int32)
        children = np.full((n, ns), -1, np.int32)
        pmin[0] = -1.0
        pmax[0] = 1.0
        # one breadth-first layer at a time: child i of node n is 8 n + 1 + i and
        # takes, on axis k, the upper half [centre, max] when bit k of i is set
        bits = np.array([[(i >> k) & 1 for k in range(3)] for i in range(ns)], bool)  # [8, 3]
        layer_start, layer_count = 0, 1
        for dep in range(1, max_depth + 1):
            ids = np.arange(layer_start, layer_start + layer_count)
            center = (pmin[ids] + pmax[ids]) * np.float32(0.5)
            kids = (8 * ids[:, None] + 1 + np.arange(ns)[None, :])  # [L, 8]
            pmin[kids] = np.where(bits[None], center[:, None, :], pmin[ids][:, None, :])
            pmax[kids] = np.where(bits[None], pmax[ids][:, None, :], center[:, None, :])
            children[ids] = kids
            depth[kids] = dep
            parent[kids] = ids[:, None]
            layer_start, layer_count = layer_start + layer_count, layer_count * ns
        self.node_position_min = pmin
        self.node_position_max = pmax
        self.node_depth = depth
        self.node_parent = parent
        self.node_children = children
        self.node_active = np.zeros(n, np.int32)
        self.node_culled = np.zeros(n, np.int32)
        self.node_max_density = np.zeros(n, np.float32)
        self._dev = {}
        self.SetActive(0)

    # --- active set (HyperTree.cpp:163-206) ---
    def NumNodes(self):
        return self.node_position_min.shape[0]

    def NumActiveNodes(self):
        return int(self.active_node_ids.shape[0])

    def SetActive(self, depth):
        self.node_active = (self.node_depth == depth).astype(np.int32)
        self.UpdateActive()

    def SetActiveNodes(self, node_ids):
        act = np.zeros(self.NumNodes(), np.int32)
        act[np.asarray(node_ids, np.int64)] = 1
        self.node_active = act
        self.UpdateActive()

    def UpdateActive(self):
        ids = np.nonzero(self.node_active == 1)[0].astype(np.int64)
        pre = np.full(self.NumNodes(), -1, np.int64)
        pre[ids] = np.arange(ids.shape[0], dtype=np.int64)
        self.active_node_ids = ids
        self.node_active_prefix_sum = pre
        self._dev = {}

    def NodeCulling(self, threshold):
        """NodeCulling (samples/reconstruct.cpp:288-319): active nodes whose
        node_max_density (from ComputeMaxDensity) is below threshold become
        culled and inactive.  Returns the number of newly culled nodes."""
        new = ((self.node_max_density < threshold) & (self.node_active == 1)).astype(np.int32)
        k = int(new.sum())
        if k:
            self.node_culled = np.clip(self.node_culled + new, 0, 1)
            self.node_active = np.clip(self.node_active - new, 0, 1)
            self.UpdateActive()
        return k

    def copy(self):
        t = HyperTreeBase.__new__(HyperTreeBase)
        t.__dict__.update({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        t._dev = {}
        return t

    def GlobalNodeIdToLocalActiveId(self, node_id):
        if isinstance(node_id, torch.Tensor):
            return self.device_tables(node_id.device)["prefix"].index_select(0, node_id.reshape(-1)).reshape(
                node_id.shape)
        return self.node_active_prefix_sum[np.asarray(node_id)]

    # --- device tables ---
    def device_tables(self, device="cuda"):
        device = torch.device(device)
        key = str(device)
        if key not in self._dev:
            t = {
                "min": torch.from_numpy(self.node_position_min).to(device),
                "max": torch.from_numpy(self.node_position_max).to(device),
                "active": torch.from_numpy(self.active_node_ids).to(device),
                "prefix": torch.from_numpy(self.node_active_prefix_sum).to(device),
            }
            if device.type == "cuda":
                lib = _lib.load()
                A = self.NumActiveNodes()
                table = torch.empty(lib.neat_tree_table_bytes(self.max_depth), dtype=torch.uint8, device=device)
                status = torch.zeros(1, dtype=torch.int32, device=device)
                stream = torch.cuda.current_stream(device).cuda_stream
                _lib.check(lib.neat_tree_prepare(t["min"].data_ptr(), t["max"].data_ptr(), t["active"].data_ptr(), A,
                                                 self.max_depth, table.data_ptr(), status.data_ptr(), stream),
                           "neat_tree_prepare")
                st = int(status.item())
                if st:
                    raise _lib.NeatError(st, "neat_tree_prepare")
                t["table"] = table
                cells = self.cell_node_map()
                t["cell_node"] = torch.from_numpy(cells).to(device) if cells is not None else None
            self._dev[key] = t
        return self._dev[key]

    def cell_node_map(self):
        """For a tree of max_depth <= 5 whose active nodes are disjoint: the
        global id of the active node holding each finest cell, or -1, int32
        [2^D][2^D][2^D] (z, y, x) -- the cell map of the step's DDA hit search.
        None for deeper trees, or when an active node lies inside another."""
        D = self.max_depth
        if D > 5:
            return None
        N = 1 << D
        cells = np.full((N, N, N), -1, np.int32)
        for nid in self.active_node_ids:
            lo = np.rint((self.node_position_min[nid].astype(np.float64) + 1.0) * (N / 2)).astype(np.int64)
            hi = np.rint((self.node_position_max[nid].astype(np.float64) + 1.0) * (N / 2)).astype(np.int64)
            box = cells[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
            if (box != -1).any():
                return None
            box[...] = nid
        return cells

    # --- adaptive structure (stands in for the reference's MIP optimizer) ---
    def RefineByVariance(self, density_fn, target_active, samples_per_axis=6, start_depth=1):
        """Greedy refinement: start from all nodes of start_depth active, then
        repeatedly split the active node whose sampled density variance is the
        largest (ties: lower id) until target_active is reached or no active
        node can split.  density_fn(points [N,3] f64) -> [N] f64."""
        s = samples_per_axis
        g = (np.arange(s, dtype=np.float64) + 0.5) / s
        lattice = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        N = self.NumNodes()
        lo = self.node_position_min.astype(np.float64)
        hi = self.node_position_max.astype(np.float64)
        pts = lo[:, None, :] + lattice[None, :, :] * (hi - lo)[:, None, :]
        dens = np.asarray(density_fn(pts.reshape(-1, 3)), np.float64).reshape(N, -1)
        var = dens.var(axis=1)
        active = set(np.nonzero(self.node_depth == start_depth)[0].tolist())
        heap = [(-var[i], i) for i in active if self.node_depth[i] < self.max_depth]
        heapq.heapify(heap)
        while len(active) + 7 <= target_active and heap:
            _, nid = heapq.heappop(heap)
            active.discard(nid)
            for c in self.node_children[nid]:
                active.add(int(c))
                if self.node_depth[c] < self.max_depth:
                    heapq.heappush(heap, (-var[c], int(c)))
        self.SetActiveNodes(sorted(active))
        return self
