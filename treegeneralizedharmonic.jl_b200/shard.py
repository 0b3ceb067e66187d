"""The batched RK4 step sharded over ranks, one GPU each.

TreeAMR's distribution of a forest's blocks over the ranks of a communicator, with the forest
itself on every rank (src/distributed.jl:1-22): the leaves are assigned per refinement level
in Morton order (tgh_partition), so every level's work, its prolongation included, is spread
over all ranks. A rank's problem computes its own leaves and holds halo copies of the other
ranks' leaves its ghost fill reads. Before each fill phase (0: the copies and the Dirichlet
ghosts; l >= 1: level l's prolongation, after the owners have filled level l - 1) the ranks
exchange the points the plan lists, 20 doubles each, in one all-to-all.

The plan is deterministic: every rank derives both its own requests and the other ranks'
requests to it from the forest and the owner map, so no host communication precedes a step.
"""
import ctypes

import numpy as np
import torch

from . import _abi
from .problem import _ptr

NV = 20


def partition(forest, nranks):
    """The owner rank of every leaf (tgh_partition): per level, Morton order, even runs."""
    lib = _abi.load_library()
    owner = np.zeros(forest.nblocks, dtype=np.int32)
    mesh = forest.mesh()
    st = lib.tgh_partition(ctypes.byref(mesh), int(nranks), ctypes.c_void_p(owner.ctypes.data))
    if st != _abi.TGH_OK:
        raise _abi.TGHError(st, "tgh_partition refused the mesh")
    return owner


def exchange_plan(case, forest, q, owner, rank, nranks, phase):
    """rank's exchange in one fill phase, computed on the host (tgh_shard_plan): per peer the
    point counts, and the (forest leaf, work index) pairs sent and received, peer-major."""
    lib = _abi.load_library()
    cfg, mesh = case.config(q), forest.mesh()
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    sc = np.zeros(nranks, dtype=np.int64)
    rc = np.zeros(nranks, dtype=np.int64)
    err = ctypes.create_string_buffer(512)
    args = (ctypes.byref(cfg), ctypes.byref(mesh), ctypes.c_void_p(owner.ctypes.data), int(rank), int(nranks),
            int(phase), ctypes.c_void_p(sc.ctypes.data), ctypes.c_void_p(rc.ctypes.data))
    st = lib.tgh_shard_plan(*args, None, None, err, 512)
    if st != _abi.TGH_OK:
        raise _abi.TGHError(st, err.value.decode())
    send = np.zeros((int(sc.sum()), 2), dtype=np.int32)
    recv = np.zeros((int(rc.sum()), 2), dtype=np.int32)
    st = lib.tgh_shard_plan(*args, ctypes.c_void_p(send.ctypes.data), ctypes.c_void_p(recv.ctypes.data), err, 512)
    if st != _abi.TGH_OK:
        raise _abi.TGHError(st, err.value.decode())
    return {"send_count": sc, "recv_count": rc, "send": send, "recv": recv}


class ShardedGHProblem:
    """One rank's part of a problem sharded over `nranks` ranks (one GPU per rank). Its state
    vectors hold the rank's own leaves, in forest order; `local(u)` cuts them out of a whole
    state vector."""

    def __init__(self, case, forest, q, rank, nranks, owner=None, group=None, margin_check=True, stream=None):
        if not torch.cuda.is_available():
            raise RuntimeError("ShardedGHProblem runs on a CUDA device; none is available")
        self.lib = _abi.load_library()
        self.case, self.forest, self.q = case, forest, int(q)
        self.rank, self.nranks, self.group = int(rank), int(nranks), group
        self.owner = partition(forest, nranks) if owner is None else np.ascontiguousarray(owner, dtype=np.int32)
        self.leaves = np.nonzero(self.owner == self.rank)[0]
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self._cfg = case.config(q)
        self._mesh = forest.mesh()
        h = ctypes.c_void_p()
        st = self.lib.tgh_problem_create_shard(ctypes.byref(self._cfg), ctypes.byref(self._mesh),
                                               ctypes.c_void_p(self.owner.ctypes.data), self.rank, self.nranks,
                                               ctypes.c_void_p(self.stream.cuda_stream), 1 if margin_check else 0,
                                               ctypes.byref(h))
        self._h = h
        if st != _abi.TGH_OK:
            msg = self.lib.tgh_last_error(h).decode() if h.value else "allocation failed"
            self.close()
            raise _abi.TGHError(st, msg)
        self.state_length = int(self.lib.tgh_state_length(h))
        self.phases = int(self.lib.tgh_shard_phases(h))
        self.send_count, self.recv_count, self.send_buf, self.recv_buf = [], [], [], []
        for ph in range(self.phases):
            sc = np.zeros(self.nranks, dtype=np.int64)
            rc = np.zeros(self.nranks, dtype=np.int64)
            self._check(self.lib.tgh_shard_counts(h, ph, ctypes.c_void_p(sc.ctypes.data),
                                                  ctypes.c_void_p(rc.ctypes.data)))
            self.send_count.append(sc)
            self.recv_count.append(rc)
            self.send_buf.append(torch.zeros(max(1, int(sc.sum())) * NV, dtype=torch.float64, device="cuda"))
            self.recv_buf.append(torch.zeros(max(1, int(rc.sum())) * NV, dtype=torch.float64, device="cuda"))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.tgh_problem_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _abi.TGH_OK:
            raise _abi.TGHError(st, self.lib.tgh_last_error(self._h).decode())

    def statevector(self):
        return torch.zeros(self.state_length, dtype=torch.float64, device="cuda")

    def local(self, u_all):
        """This rank's leaves' part of a whole state vector (forest order, block-major)."""
        per = u_all.numel() // self.forest.nblocks
        return u_all.view(self.forest.nblocks, per)[torch.as_tensor(self.leaves, device=u_all.device)].reshape(-1)

    # ---- pointwise verbs on this rank's leaves ----
    def initial_state(self, u, t):
        """The analytic state (through the core rule) at this rank's owned points."""
        self._check(self.lib.tgh_initial_state(self._h, _ptr(u), float(t)))
        return u

    def max_speed(self, u, t):
        """The largest characteristic speed over this rank's evolved points; the caller takes
        the maximum over ranks."""
        lam = ctypes.c_double()
        st = self.lib.tgh_max_speed(self._h, _ptr(u), float(t), ctypes.byref(lam))
        if st == _abi.TGH_ERR_SPEED and lam.value == 0.0:
            return 0.0  # no evolved point on this rank (all inside a frozen core)
        self._check(st)
        return lam.value

    def last_launch_count(self):
        """Kernels the last sharded step launched on this rank."""
        n = ctypes.c_long()
        self._check(self.lib.tgh_last_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def time_rhs(self, u, t, nlaunch=2):
        """ms per right-hand side (batched form, head + Pi) on this rank's leaves, timed on the
        working array as the last step left it."""
        ms = ctypes.c_double()
        self._check(self.lib.tgh_time_rhs(self._h, _ptr(u), float(t), 1, int(nlaunch), ctypes.byref(ms)))
        return ms.value

    # ---- the step's pieces (include/tgh.h) ----
    def begin(self, u):
        self._check(self.lib.tgh_shard_begin(self._h, _ptr(u)))

    def pack(self, stage, phase):
        self._check(self.lib.tgh_shard_pack(self._h, stage, phase, _ptr(self.send_buf[phase])))

    def unpack(self, stage, phase):
        self._check(self.lib.tgh_shard_unpack(self._h, stage, phase, _ptr(self.recv_buf[phase])))

    def fill(self, stage, phase, t, dt):
        self._check(self.lib.tgh_shard_fill(self._h, stage, phase, float(t), float(dt)))

    def rhs(self, stage, t, dt):
        self._check(self.lib.tgh_shard_rhs(self._h, stage, float(t), float(dt)))

    def end(self, u):
        self._check(self.lib.tgh_shard_end(self._h, _ptr(u)))

    def exchange(self, phase):
        """The phase's all-to-all over the process group: peer-major buffers of 20 doubles per
        point, counts from the plan. NCCL moves device buffers between GPUs; a gloo group (ranks
        that share a GPU, or tests) moves host copies of them, the waits all on the host."""
        import torch.distributed as dist
        if self.nranks == 1:
            return
        ns, nr = int(self.send_count[phase].sum()) * NV, int(self.recv_count[phase].sum()) * NV
        send, recv = self.send_buf[phase][:ns], self.recv_buf[phase][:nr]
        osz = [int(c) * NV for c in self.recv_count[phase]]
        isz = [int(c) * NV for c in self.send_count[phase]]
        if dist.get_backend(self.group) == "gloo":
            hs = send.cpu()  # ordered after pack on the current (the problem's) stream
            hr = torch.empty(nr, dtype=torch.float64)
            dist.all_to_all_single(hr, hs, output_split_sizes=osz, input_split_sizes=isz, group=self.group)
            recv.copy_(hr)
        else:
            dist.all_to_all_single(recv, send, output_split_sizes=osz, input_split_sizes=isz, group=self.group)

    def step(self, u, t, dt, nsteps=1):
        """nsteps RK4 steps of the batched form on this rank's leaves, exchanging with the other
        ranks before every fill phase; u holds this rank's leaves and is updated in place. The
        exchange is ordered on the problem's stream (the current stream while the step runs),
        whatever stream the caller has current."""
        with torch.cuda.stream(self.stream):
            self.begin(u)
            for n in range(int(nsteps)):
                tn = float(t) + n * float(dt)
                for st in range(4):
                    for ph in range(self.phases):
                        self.pack(st, ph)
                        self.exchange(ph)
                        self.unpack(st, ph)
                        self.fill(st, ph, tn, dt)
                    self.rhs(st, tn, dt)
            self.end(u)
