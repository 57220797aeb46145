"""Batched steady solves: many independent design points marched together.

A sweep's points have uneven meshes (element kind, order and refinement vary),
so the instances are grouped into buckets of one (kind, order); each bucket's
elements are concatenated, with connectivity offset, into one device mesh, and
each SSP-RK3 stage is one kernel launch per bucket over every instance in it.
An ``elem_inst`` array maps elements to instances, which carry their own back
pressure, tolerance and march state.  After every chunk (one step first, then
``check_interval`` steps, as the reference's march does) a device kernel
evaluates each running instance's residual and applies the reference's
convergence, non-finite, divergence, stall and iteration-cap tests
(src/timestepping/march.py:125-230); retired instances are no longer advanced,
so every instance ends on exactly the iteration the one-at-a-time march would.
Each chunk is one CUDA graph; the host reads one integer (the number of
instances still running) per chunk.

This replaces the reference's serial, warm-started ``sweep`` loop
(src/sweep.py:300-446) for the solve itself; refusal of shocked operating
points happens on the host before batching, as there.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .config import FLUX_IDS, SCHEMES, recommended_scheme, residual_scale, step_coefficient
from .autotune import choose_variant, set_struct_variant, tail_elements
from .layout import DeviceMesh, concat_arrays, host_arrays, physics_struct

STATUS = {0: "running", 1: "converged", 2: "non-finite", 3: "diverged", 4: "stalled", 5: "max_iterations"}


@dataclass
class Instance:
    ops: object
    flow: object
    opts: object
    U0: np.ndarray | None  # (E, NP, 4); None: the quasi-1D initial state, projected on the device
    length: float = 1.0
    geometry: object = None  # the nozzle geometry: adds the throat-normalised observables


@dataclass
class InstanceResult:
    status: str
    converged: bool
    iterations: int
    residual: float
    residual_initial: float
    U: np.ndarray | None


def blocks_of(ranges, width: int) -> np.ndarray:
    """The sorted block indices (``width`` elements per block) that hold an element of any of the
    half-open element ranges."""
    idx = [np.arange(lo // width, (hi - 1) // width + 1) for lo, hi in ranges if hi > lo]
    if not idx:
        return np.zeros(0, np.int32)
    return np.unique(np.concatenate(idx)).astype(np.int32)


class BatchSolver:
    def __init__(self, instances: list[Instance], device=None, variants: str = "batch", compact: bool = True):
        """``variants``: the launch variants' context in the variant table -- ``batch`` (measured on
        buckets marching side by side) or ``single`` (the one-solve choice, so a batch gives a plain
        solve's bits).  ``compact``: late in the march, launch only the blocks that hold elements of
        running instances (the same kernels on the same elements: the same bits)."""
        import torch

        if not instances:
            raise ValueError("empty batch")
        self.torch = torch
        self.lib = capi.load()
        self.instances = instances
        opts0 = instances[0].opts
        for inst in instances:
            o = inst.opts
            if (o.cfl, o.limiter, o.check_interval, o.max_iterations, o.stall_window, o.stall_ratio,
                    o.divergence_factor, o.scheme, getattr(o, "positivity_cfl", 0.0)) != (
                    opts0.cfl, opts0.limiter, opts0.check_interval, opts0.max_iterations, opts0.stall_window,
                    opts0.stall_ratio, opts0.divergence_factor, opts0.scheme, getattr(opts0, "positivity_cfl", 0.0)):
                raise ValueError("every instance of a batch must share the march options")
            if inst.flow.flux not in FLUX_IDS:
                raise NotImplementedError(f"flux {inst.flow.flux!r}")
        self.opts = opts0
        dev = torch.device(device if device is not None else "cuda")
        self.device = dev
        n = len(instances)

        # buckets of one (kind, order)
        keys = [(inst.ops.ref.kind, inst.ops.ref.order) for inst in instances]
        self.bucket_keys = sorted(set(keys), key=lambda k: (k[0], k[1]))
        self.members = [[i for i in range(n) if keys[i] == k] for k in self.bucket_keys]
        begin = np.zeros(n, np.int64)
        end = np.zeros(n, np.int64)
        local = np.zeros(n, np.int64)
        count = np.zeros(n)
        tol = np.zeros(n)
        p_back = np.zeros(n)
        self.meshes, self.buffers, self.phys, self.offsets, self.factors = [], [], [], [], []
        self._keep = []
        self.U0_soa = []  # each bucket's initial state, kept for reset()
        self.h2d_bytes = 0  # host -> device bytes of the set-up (states, geometry, connectivity)
        g_off = 0
        # lean instances (operators built without per-element arrays) get their metric terms built on the
        # device from the node coordinates; instances without an initial state get the quasi-1D one
        # projected on the device
        lean = [getattr(inst.ops, "inv_mass", None) is None for inst in instances]
        device_init = [inst.U0 is None for inst in instances]
        if len(set(lean)) > 1 or len(set(device_init)) > 1:
            raise ValueError("the instances of a batch are all lean or all not, and all carry an initial state or none")
        self.device_built = lean[0]
        if device_init[0]:
            from .nozzle import quasi1d_table, wall_parameters

            if any(inst.geometry is None for inst in instances):
                raise ValueError("an instance without an initial state needs its nozzle geometry")
            walls = np.stack([wall_parameters(inst.geometry) for inst in instances])
            q1d = [quasi1d_table(inst.geometry, inst.flow) for inst in instances]
        for key, mem in zip(self.bucket_keys, self.members):
            parts = [host_arrays(instances[i].ops, device_metrics=lean[0]) for i in mem]
            arrays = concat_arrays(parts)
            ref = instances[mem[0]].ops.ref
            dm = DeviceMesh(device=dev, arrays=arrays, ref=ref)
            if lean[0] or device_init[0]:
                nv = dm.nf
                X, en, n_off = [], [], 0
                for i in mem:
                    Xi = np.asarray(instances[i].ops.node_coords, float)
                    X.append(Xi)
                    en.append(np.asarray(instances[i].ops.topology.elem_nodes)[:, :nv] + n_off)
                    n_off += Xi.shape[0]
                X, en = np.concatenate(X), np.ascontiguousarray(np.concatenate(en))
            if lean[0]:
                dm.set_geometry(X, en)
                self.h2d_bytes += X.nbytes + en.size * 4
            flow0 = instances[mem[0]].flow
            for i in mem:
                f = instances[i].flow
                if (f.gamma, f.flux, f.entropy_fix, f.hllc_low_mach, f.backflow, f.total_pressure,
                        f.total_temperature, f.Rgas, f.inflow_angle) != (flow0.gamma, flow0.flux, flow0.entropy_fix,
                                                                          flow0.hllc_low_mach, flow0.backflow,
                                                                          flow0.total_pressure, flow0.total_temperature,
                                                                          flow0.Rgas, flow0.inflow_angle):
                    raise ValueError("instances of a bucket may differ only in back pressure")
            ph = physics_struct(flow0, opts0, ref)
            elem_inst = np.empty(arrays["n_elem"], np.int32)
            l_off = 0
            for i, part in zip(mem, parts):
                E_i = part["n_elem"]
                elem_inst[l_off:l_off + E_i] = i
                begin[i], end[i], local[i] = g_off + l_off, g_off + l_off + E_i, l_off
                count[i] = 4.0 * E_i * ref.n_basis
                f = instances[i].flow
                tol[i] = instances[i].opts.tolerance * residual_scale(f, instances[i].length)
                p_back[i] = f.back_pressure
                l_off += E_i
            self._keep.append(torch.as_tensor(elem_inst, device=dev))
            dm.elem_inst_t = self._keep[-1]
            if opts0.limiter == "superbee":
                # each instance is limited against its own domain: area shares and the maximum of
                # its cell averages per instance (4 numbers each)
                area = np.asarray(arrays["area"], float)
                share = np.empty_like(area)
                l_off = 0
                for part in parts:
                    E_i = part["n_elem"]
                    share[l_off:l_off + E_i] = area[l_off:l_off + E_i] / area[l_off:l_off + E_i].sum()
                    l_off += E_i
                dm.elem_share = torch.as_tensor(share, device=dev)
                dm.lim_scale = torch.zeros(4 * n, dtype=torch.float64, device=dev)
                dm.c.elem_share = dm.elem_share.data_ptr()
                dm.c.lim_scale = dm.lim_scale.data_ptr()
                dm.c.n_inst = n
            S = [dm.state() for _ in range(3)]
            dt = torch.zeros(dm.E, dtype=torch.float64, device=dev)
            if device_init[0]:
                dm.initial_state(ph, walls, q1d, X, en, elem_inst=dm.elem_inst_t, out=S[0])
                self.h2d_bytes += dm.initial_h2d_bytes
            else:
                U0 = np.concatenate([np.asarray(instances[i].U0, float) for i in mem])
                dm.pack(U0, S[0])
                self.h2d_bytes += U0.nbytes
            self.U0_soa.append(S[0].clone())
            choose_variant(dm, variants)
            self.h2d_bytes += sum(a.nbytes for a in arrays.values() if isinstance(a, np.ndarray))
            bf = capi.Buffers()
            bf.S0, bf.S1, bf.S2 = (x.data_ptr() for x in S)
            bf.dt = dt.data_ptr()
            self._keep += S + [dt]
            scheme = opts0.scheme or recommended_scheme(ref.order)
            if scheme not in SCHEMES:
                raise ValueError(f"unknown scheme {scheme!r}")
            pc = getattr(opts0, "positivity_cfl", 0.0)
            pscale = float(pc) if (pc > 0.0 and opts0.limiter != "none" and ref.order > 0) else 1.0
            if (scheme == "ssprk3") != (ref.order > 0):
                raise NotImplementedError("batches march SSP-RK3 above p = 0 and forward Euler at p = 0")
            self.meshes.append(dm)
            self.buffers.append((bf, S))
            self.phys.append(ph)
            self.offsets.append(g_off)
            self.factors.append(pscale * step_coefficient(ref.order, opts0.cfl, scheme))
            g_off += dm.E
        self.n_elem = g_off
        self.begin, self.end, self.local = begin, end, local

        T = lambda a, dt: torch.as_tensor(a, dtype=dt, device=dev)  # noqa: E731
        W = opts0.stall_window
        self.t = {
            "begin": T(begin, torch.int64), "end": T(end, torch.int64), "count": T(count, torch.float64),
            "tol": T(tol, torch.float64), "p_back": T(p_back, torch.float64),
            "elem_norm": torch.zeros(g_off, dtype=torch.float64, device=dev),
            "status": torch.zeros(n, dtype=torch.int32, device=dev), "iterations": torch.zeros(n, dtype=torch.int32, device=dev),
            "res0": torch.zeros(n, dtype=torch.float64, device=dev), "res": torch.zeros(n, dtype=torch.float64, device=dev),
            "window": torch.zeros(n * W, dtype=torch.float64, device=dev),
            "window_count": torch.zeros(n, dtype=torch.int32, device=dev),
            "n_running": torch.zeros(1, dtype=torch.int32, device=dev),
        }
        for dm in self.meshes:
            dm.set_batch(dm.elem_inst_t, self.t["status"], self.t["p_back"])
        bm = capi.BatchMarch()
        bm.n_inst = n
        for f, k in (("inst_begin", "begin"), ("inst_end", "end"), ("inst_count", "count"), ("inst_tol", "tol"),
                     ("elem_norm", "elem_norm"), ("status", "status"), ("iterations", "iterations"), ("res0", "res0"),
                     ("res", "res"), ("window", "window"), ("window_count", "window_count"), ("n_running", "n_running")):
            setattr(bm, f, self.t[k].data_ptr())
        bm.divergence_factor = float(opts0.divergence_factor)
        bm.stall_ratio = float(opts0.stall_ratio)
        bm.stall_window = int(W)
        bm.max_iterations = int(opts0.max_iterations)
        self.bm = bm
        nb = len(self.meshes)
        self._physs = (capi.Physics * nb)(*self.phys)
        self._bufs = (capi.Buffers * nb)(*[b for b, _ in self.buffers])
        self._offs = np.asarray(self.offsets, np.int64)
        self._facs = np.asarray(self.factors, float)
        self._elem_count = np.asarray(end - begin, np.int64)
        self._handles = {}  # march object -> the block lists it launches (kept alive with it)
        self._main = self._create(None, None)
        self.handle = self._main
        # Late in a march most instances have retired.  Two things follow, both taken between chunks when
        # the set of running instances has changed: (1) once the instances still marching hold few
        # elements, the batch's throughput variants leave the GPU idle and an element's latency decides,
        # so the march switches to the single-solve variants (the tail); (2) once the blocks holding
        # running elements are at most half of those a launch spans, a march object whose launches list
        # only those blocks replaces the current one, so a launch no longer walks every retired block.
        self.variants = variants
        self._tail_at = tail_elements() if variants == "batch" else 0
        self.compact = bool(compact)
        self._in_tail = False
        self._launched = self._blocks_launched(None, None)
        self.tail_switched_at = None  # iteration of the switch, if any
        self.compactions = 0
        self._last_running = n
        self.done = 0
        self.chunks = 0
        self.launches = 0
        self._obs = None

    def _meshes_for(self, context, running):
        """Mesh descriptors for a march object -- the buckets' own variants, or those of ``context`` --
        and, with ``running`` (a per-instance mask), each bucket's list of the blocks that hold elements
        of running instances (None without)."""
        meshes, lists = [], []
        for dm, mem in zip(self.meshes, self.members):
            mc = capi.Mesh()
            C.memmove(C.byref(mc), C.byref(dm.c), C.sizeof(capi.Mesh))
            if context is not None:
                set_struct_variant(mc, dm.kind, dm.order, context)
            blocks = None
            if running is not None:
                W = int(self.lib.nzb_block_width(C.byref(mc), 0))
                blocks = blocks_of([(int(self.local[i]), int(self.local[i] + self._elem_count[i])) for i in mem
                                    if running[i]], W)
            meshes.append(mc)
            lists.append(blocks)
        return meshes, lists

    def _blocks_launched(self, context, running) -> int:
        meshes, lists = self._meshes_for(context, running)
        return sum(int(self.lib.nzb_element_blocks(C.byref(m))) if b is None else int(b.size)
                   for m, b in zip(meshes, lists))

    def _create(self, context, running) -> int:
        meshes, lists = self._meshes_for(context, running)
        keep = []
        for mc, blocks in zip(meshes, lists):
            if blocks is not None:
                t = self.torch.as_tensor(blocks if blocks.size else np.zeros(1, np.int32), device=self.device)
                mc.fwd_blocks, mc.n_fwd_blocks = t.data_ptr(), int(blocks.size)
                keep.append(t)
        nb = len(meshes)
        h = capi.P()
        capi.check(self.lib.nzb_batch_create(nb, (capi.Mesh * nb)(*meshes), self._physs, self._bufs,
                                             self._offs.ctypes.data, self._facs.ctypes.data, C.byref(self.bm),
                                             C.byref(h)), "nzb_batch_create")
        self._handles[h.value] = keep
        # buckets with nothing to launch (every block of theirs retired) make no launches
        self._bucket_live = [b is None or b.size > 0 for b in lists]
        return h.value

    def _drop(self, h) -> None:
        if h and h in self._handles and h != getattr(self, "_main", None):
            self.lib.nzb_batch_destroy(h)
            del self._handles[h]

    def __del__(self):
        for h in list(getattr(self, "_handles", {})):
            self.lib.nzb_batch_destroy(h)
        self._handles = {}

    @property
    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def launches_per_chunk(self, n: int) -> int:
        """Kernel launches of one n-step chunk: 3 stages (SSP-RK3) or a stage and a copy (Euler) per
        bucket and step, plus the check."""
        live = getattr(self, "_bucket_live", [True] * len(self.meshes))
        return sum((3 if dm.order > 0 else 2) * n for dm, on in zip(self.meshes, live) if on) + 1

    def launch_chunk(self, n: int, first: bool) -> None:
        """Queue one n-step chunk (and its retirement check) on the current stream; no synchronisation."""
        capi.check(self.lib.nzb_batch_run(self.handle, int(n), 1 if first else 0, self._stream), "nzb_batch_run")
        self.done += n
        self.chunks += 1
        self.launches += self.launches_per_chunk(n)

    def n_running(self) -> int:
        """Instances still marching after the last queued chunk (waits for it)."""
        return int(self.t["n_running"].item())

    def active_elements(self) -> int:
        """Elements of the instances still marching (reads the statuses)."""
        st = self.t["status"].cpu().numpy()
        return int(self._elem_count[st == 0].sum())

    def _retarget(self, running: int) -> None:
        """Between chunks (nothing queued): the tail switch and the block-list compaction."""
        if running == self._last_running or not running:
            return
        self._last_running = running
        mask = self.t["status"].cpu().numpy() == 0
        tail = self._in_tail or (self._tail_at > 0 and int(self._elem_count[mask].sum()) <= self._tail_at)
        context = "single" if tail else None
        if not self.compact:
            mask = None
        need = self._blocks_launched(context, mask)
        if tail != self._in_tail or (mask is not None and 2 * need <= self._launched):
            old = self.handle
            self.handle = self._create(context, mask)
            self._drop(old)
            self._launched = need
            self.compactions += 1
            if tail and not self._in_tail:
                self._in_tail = True
                self.tail_switched_at = self.done

    _maybe_tail = _retarget

    def step_chunk(self, n: int, first: bool) -> int:
        self.launch_chunk(n, first)
        running = self.n_running()
        self._retarget(running)
        return running

    def reset(self) -> None:
        """Put every instance back at its initial state with a fresh march record."""
        self._drop(self.handle)
        self.handle = self._main
        self._bucket_live = [True] * len(self.meshes)
        self._in_tail = False
        self._launched = self._blocks_launched(None, None)
        self.tail_switched_at = None
        self.compactions = 0
        self._last_running = len(self.instances)
        for (bf, S), U0 in zip(self.buffers, self.U0_soa):
            S[0].copy_(U0)
        for k in ("status", "iterations", "res0", "res", "window", "window_count", "elem_norm", "n_running"):
            self.t[k].zero_()
        self.done = 0
        self.chunks = 0
        self.launches = 0

    def run(self) -> int:
        """March every instance to retirement; returns the number of chunks."""
        o = self.opts
        running = self.step_chunk(1, True)
        chunk = min(max(1, o.check_interval), o.max_iterations)
        while running and self.done < o.max_iterations:
            running = self.step_chunk(min(chunk, o.max_iterations - self.done), False)
        return self.chunks

    def results(self, with_state: bool = True) -> list[InstanceResult]:
        st = self.t["status"].cpu().numpy()
        its = self.t["iterations"].cpu().numpy()
        res = self.t["res"].cpu().numpy()
        res0 = self.t["res0"].cpu().numpy()
        states = {}
        if with_state:
            for dm, (bf, S), mem in zip(self.meshes, self.buffers, self.members):
                full = dm.unpack(S[0]).cpu().numpy()
                for i in mem:
                    states[i] = full[self.local[i]:self.local[i] + self.instances[i].ops.n_elem]
        return [InstanceResult(STATUS[int(st[i])], int(st[i]) == 1, int(its[i]), float(res[i]), float(res0[i]),
                               states.get(i)) for i in range(len(self.instances))]

    def observables(self) -> list[dict]:
        """Every instance's performance() metrics (thrust in both forms, mass flows, exit averages,
        entropy error), integrated on the device: one launch per bucket, and only the per-instance
        sums leave the device."""
        from .observables import DeviceObservables, from_sums

        if self._obs is None:
            self._obs = []
            for dm, ph, mem in zip(self.meshes, self.phys, self.members):
                parts, e_off, k_off = [], 0, 0
                for i in mem:
                    ops = self.instances[i].ops
                    parts.append((ops, e_off, k_off))
                    e_off += int(ops.n_elem)
                    k_off += int(ops.n_interior + ops.n_boundary)
                self._obs.append(DeviceObservables(dm, ph, parts, [self.instances[i].flow for i in mem]))
        for ob, (bf, S) in zip(self._obs, self.buffers):
            ob.launch(S[0])
        out = [None] * len(self.instances)
        for ob, mem in zip(self._obs, self.members):
            sums = ob.out.cpu().numpy()
            for j, i in enumerate(mem):
                inst = self.instances[i]
                out[i] = from_sums(sums[j], inst.flow, inst.geometry)
        return out
