"""Row-block distributed vectors and matrices over several GPUs (one rank per GPU).

The B200 counterpart of HiFlow3's CoupledVector / CoupledMatrix / LaCouplings
(src/linear_algebra/coupled_vector.cc, coupled_matrix.cc, la_couplings.cc):
- every rank owns a contiguous block of rows (``offsets``);
- its matrix rows are split into the diagonal block (owned columns) and the
  off-diagonal block (ghost columns), b200la_rowblock_split;
- a vector holds its owned values (interior) and a ghost buffer; UpdateGhost
  packs the border values every peer needs with the gather kernel and moves
  them peer to peer (the reference's Isend/Irecv pair, coupled_vector.cc:975-1128);
- dot products and norms reduce the local value across ranks (the reference's
  MPI_Allreduce, coupled_vector.cc:331-436).

Transports: ``DistTransport`` over torch.distributed (NCCL for device tensors
between GPUs, gloo for host tensors) and ``LocalTransport``, several ranks in
one process (threads, one per rank, sharing a mailbox), which lets ranks share
a GPU.  No collective here waits inside a kernel, so ranks on one GPU cannot
deadlock one another.

The device exchange is stream-ordered and overlaps the diagonal-block SpMV,
as the reference overlaps its Isend/Irecv with the local product
(coupled_matrix.cc:433-467): the border is packed on the platform's stream,
an event hands it to a communication stream that moves it, the diagonal
block is multiplied meanwhile, and the platform's stream waits for the
transfer's event only before the off-diagonal block.  The host does not wait
for the transfer.

Only host logic (partition, couplings set-up, exchange protocol) runs without
a GPU; vectors and matrices live on the device and compute with the
platform's kernels, with no host fallback.
"""
import ctypes as C
import threading

import numpy as np

from . import CSR_lMatrix, F64, B200Error, Control, Result, lib, rowblock_split

__all__ = ["RowPartition", "LaCouplings", "DistTransport", "LocalTransport", "CoupledVector", "CoupledMatrix",
           "BlockPrecond", "CoupledCG", "CoupledGMRES", "CoupledMPIR", "CoupledAsyncJacobi", "exchange",
           "exchange_async", "Comm", "NativeCoupledMatrix"]


class RowPartition:
    """Owner ranges: rank r owns global rows [offsets[r], offsets[r+1])."""

    def __init__(self, offsets):
        self.offsets = np.asarray(offsets, np.int64)
        assert self.offsets[0] == 0 and np.all(np.diff(self.offsets) >= 0)

    @classmethod
    def even(cls, n, size):
        return cls([n * r // size for r in range(size + 1)])

    def owner(self, g):
        return np.searchsorted(self.offsets, np.asarray(g), side="right") - 1

    def range(self, rank):
        return int(self.offsets[rank]), int(self.offsets[rank + 1])


# ---------------------------------------------------------------- transports

class DistTransport:
    """torch.distributed (initialised process group) as the transport."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        self._comm = None

    def alltoall_lists(self, lists):
        """lists[q] -> peer q; returns what every peer sent to this rank."""
        allv = [None] * self.size
        self.dist.all_gather_object(allv, [list(map(int, x)) for x in lists], group=self.group)
        return [np.asarray(allv[q][self.rank], np.int64) for q in range(self.size)]

    def exchange(self, sends, recvs):
        """sends / recvs: {peer: tensor}; point-to-point, all posted together."""
        ops = [self.dist.P2POp(self.dist.irecv, t, q, self.group) for q, t in recvs.items() if t.numel()]
        ops += [self.dist.P2POp(self.dist.isend, t, q, self.group) for q, t in sends.items() if t.numel()]
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        # the platform's kernels run on their own stream: finish the transfers first
        if any(t.is_cuda for t in list(sends.values()) + list(recvs.values())):
            import torch
            torch.cuda.current_stream().synchronize()

    def exchange_async(self, sends, recvs, ready):
        """Device tensors: the point-to-point transfers run on a communication
        stream once ``ready`` (recorded on this rank's platform stream after
        the border was packed) has completed.  Returns the events the platform
        stream waits on before it reads the ghosts or packs the border again;
        the host does not wait."""
        import torch
        if self._comm is None:
            self._comm = torch.cuda.Stream()
        comm = self._comm
        comm.wait_event(ready)
        ops = [self.dist.P2POp(self.dist.irecv, t, q, self.group) for q, t in recvs.items() if t.numel()]
        ops += [self.dist.P2POp(self.dist.isend, t, q, self.group) for q, t in sends.items() if t.numel()]
        with torch.cuda.stream(comm):
            if ops:
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()   # the communication stream waits, not the host
        done = torch.cuda.Event()
        done.record(comm)
        return [done]

    def allreduce_sum(self, value, device):
        import torch
        t = torch.tensor([value], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())


class _Fabric:
    """Mailboxes and a barrier shared by the ranks of one LocalTransport."""

    def __init__(self, size):
        self.size = size
        self.barrier = threading.Barrier(size)
        self.box = {}


class LocalTransport:
    """Ranks of one process (one thread per rank).  Create all ranks' transports
    from one ``LocalTransport.group(size)`` call."""

    def __init__(self, fabric, rank):
        self.f, self.rank, self.size = fabric, rank, fabric.size
        self._comm = None

    @classmethod
    def group(cls, size):
        fab = _Fabric(size)
        return [cls(fab, r) for r in range(size)]

    def alltoall_lists(self, lists):
        for q in range(self.size):
            self.f.box[("a2a", self.rank, q)] = np.asarray(lists[q], np.int64)
        self.f.barrier.wait()
        out = [self.f.box[("a2a", q, self.rank)] for q in range(self.size)]
        self.f.barrier.wait()
        return out

    def exchange(self, sends, recvs):
        import torch
        for q, t in sends.items():
            self.f.box[("p2p", self.rank, q)] = t
        # the senders' streams must have produced their buffers before anyone copies
        torch.cuda.synchronize() if any(t.is_cuda for t in sends.values()) else None
        self.f.barrier.wait()
        for q, t in recvs.items():
            if t.numel():
                t.copy_(self.f.box[("p2p", q, self.rank)])
        if any(t.is_cuda for t in recvs.values()):
            torch.cuda.synchronize()
        self.f.barrier.wait()

    def exchange_async(self, sends, recvs, ready):
        """Stream-ordered exchange between thread ranks: each receiver copies
        from its senders' border buffers on its own communication stream, after
        the senders' pack events and its own (so the copy cannot overwrite
        ghosts its last off-diagonal product still reads).  Returns this rank's
        copy event and the copy events of the peers that read its border: the
        platform stream waits on all of them before it reads the ghosts or packs
        the border again."""
        import torch
        if self._comm is None:
            self._comm = torch.cuda.Stream()
        comm = self._comm
        for q, t in sends.items():
            self.f.box[("p2p", self.rank, q)] = (t, ready)
        self.f.barrier.wait()
        comm.wait_event(ready)
        with torch.cuda.stream(comm):
            for q, t in recvs.items():
                if t.numel():
                    src, ev = self.f.box[("p2p", q, self.rank)]
                    comm.wait_event(ev)
                    t.copy_(src, non_blocking=True)
        done = torch.cuda.Event()
        done.record(comm)
        self.f.box[("copied", self.rank)] = done
        self.f.barrier.wait()
        waits = [done] + [self.f.box[("copied", q)] for q, t in sends.items() if t.numel()]
        self.f.barrier.wait()
        return waits

    def allgather_objects(self, obj):
        """Every rank's obj, in rank order (pointers and events of the
        remote-gather product)."""
        self.f.box[("ag", self.rank)] = obj
        self.f.barrier.wait()
        out = [self.f.box[("ag", q)] for q in range(self.size)]
        self.f.barrier.wait()
        return out

    def allreduce_sum(self, value, device=None):
        self.f.box[("sum", self.rank)] = float(value)
        self.f.barrier.wait()
        tot = 0.0
        for q in range(self.size):   # every rank adds in the same order
            tot += self.f.box[("sum", q)]
        self.f.barrier.wait()
        return tot


def _pairs(transport, couplings, border_values, ghost_values):
    sends, recvs = {}, {}
    for q in range(transport.size):
        b0, b1 = couplings.border_offsets[q], couplings.border_offsets[q + 1]
        g0, g1 = couplings.ghost_offsets[q], couplings.ghost_offsets[q + 1]
        if b1 > b0:
            sends[q] = border_values[b0:b1]
        if g1 > g0:
            recvs[q] = ghost_values[g0:g1]
    return sends, recvs


def exchange(transport, couplings, border_values, ghost_values):
    """Move border values (ordered by peer, couplings.border_offsets) into the
    peers' ghost buffers (ordered by owner, couplings.ghost_offsets)."""
    transport.exchange(*_pairs(transport, couplings, border_values, ghost_values))


def exchange_async(transport, couplings, border_values, ghost_values, ready):
    """exchange() for device buffers, ordered on streams behind the event
    ``ready``; returns the events to wait on (transport.exchange_async)."""
    return transport.exchange_async(*_pairs(transport, couplings, border_values, ghost_values), ready)


class LaCouplings:
    """Ghost and border index sets of one rank (la_couplings.cc:62-230).

    ghost_global: ascending global numbers of the ghost columns; grouped by
    owner (owners hold contiguous ranges), ghost_offsets[q] marks owner q's
    part.  border_indices: local numbers of owned values that peers need,
    grouped by peer (border_offsets), in the order the peer lists its ghosts.
    """

    def __init__(self, partition, rank, ghost_global):
        self.part, self.rank = partition, rank
        self.ghost_global = np.asarray(ghost_global, np.int64)
        owners = partition.owner(self.ghost_global) if self.ghost_global.size else np.zeros(0, np.int64)
        if np.any(owners == rank):
            raise ValueError("a ghost column is owned by this rank")
        size = len(partition.offsets) - 1
        self.ghost_offsets = np.searchsorted(owners, np.arange(size + 1), side="left").astype(np.int64)
        # where each ghost lives: its owner and its number there
        self.ghost_owner = np.asarray(owners, np.int32)
        self.ghost_index = (self.ghost_global - partition.offsets[owners]).astype(np.int32) if owners.size \
            else np.zeros(0, np.int32)
        self.border_indices = None
        self.border_offsets = None

    def setup(self, transport):
        """Exchange the ghost lists: what this rank needs from every owner, and
        what every peer needs from this rank (its border)."""
        size = transport.size
        need = [self.ghost_global[self.ghost_offsets[q]:self.ghost_offsets[q + 1]] for q in range(size)]
        got = transport.alltoall_lists(need)
        r0, _ = self.part.range(self.rank)
        self.border_offsets = np.zeros(size + 1, np.int64)
        for q in range(size):
            self.border_offsets[q + 1] = self.border_offsets[q] + len(got[q])
        self.border_indices = (np.concatenate(got) - r0).astype(np.int32) if size else np.zeros(0, np.int32)
        return self


# ------------------------------------------------------------ device objects

class CoupledVector:
    """Owned values (an lVector on this rank's GPU) plus a ghost buffer."""

    def __init__(self, platform, couplings, transport, data_or_n, dtype=F64):
        import torch
        self.pf, self.cp, self.tr, self.dtype = platform, couplings, transport, dtype
        self.interior = platform.vector(data_or_n, dtype)
        td = torch.float64 if dtype == F64 else torch.float32
        dev = f"cuda:{platform.device}"
        with platform.on_stream():
            self.ghost = torch.zeros(len(couplings.ghost_global), dtype=td, device=dev)
            self.border = torch.zeros(len(couplings.border_indices), dtype=td, device=dev)
            self._bidx = torch.from_numpy(couplings.border_indices.astype(np.int32)).to(dev)

    def clone_without_content(self):
        return CoupledVector(self.pf, self.cp, self.tr, self.interior.get_size(), self.dtype)

    def begin_update(self):
        """Pack the border with the gather kernel on the platform's stream and
        start the exchange behind it; returns what end_update waits on."""
        import torch
        nb = self.border.numel()
        if nb:
            self.pf.check(lib().b200la_gather(self.pf.h, self.dtype, nb, C.c_void_p(self._bidx.data_ptr()),
                                              self.interior.ptr, C.c_void_p(self.border.data_ptr())), "gather")
        ready = torch.cuda.Event()
        ready.record(self.pf.stream())
        return exchange_async(self.tr, self.cp, self.border, self.ghost, ready)

    def end_update(self, waits):
        """The platform's stream waits for the exchange (ghosts in place, border
        free to be packed again); the host does not."""
        ls = self.pf.stream()
        for ev in waits:
            ls.wait_event(ev)

    def UpdateGhost(self):
        """Pack the border, exchange it with the peers, the ghosts ready for
        the platform's next kernel (CoupledVector::UpdateGhost)."""
        self.end_update(self.begin_update())

    def CastInteriorFrom(self, other):
        """The owned values of other in this vector's precision
        (CoupledVector::CastInteriorFrom, coupled_vector.cc:755-806)."""
        self.interior.CastFrom(other.interior)

    # global reductions (local kernel, then the sum across ranks)
    def Dot(self, other):
        return self.tr.allreduce_sum(self.interior.Dot(other.interior), f"cuda:{self.pf.device}")

    def Norm2(self):
        return float(np.sqrt(self.Dot(self)))

    # local BLAS1 (coupled_vector.cc:331-436 forward to the interior)
    def Axpy(self, v, a):
        self.interior.Axpy(v.interior, a)

    def ScaleAdd(self, a, v):
        self.interior.ScaleAdd(a, v.interior)

    def Scale(self, a):
        self.interior.Scale(a)

    def CopyFrom(self, v):
        self.interior.CopyFrom(v.interior)

    def Zeros(self):
        self.interior.Zeros()

    def numpy(self):
        return self.interior.numpy()


class CoupledMatrix:
    """Diagonal and off-diagonal blocks of this rank's rows on its GPU."""

    def __init__(self, platform, partition, rank, transport, row, col, val, dtype=F64, remote=False):
        """row/col/val: this rank's rows (CSR) with global column numbers.
        remote=True: VectorMult reads the ghost values straight from the
        owners' vectors (b200la_spmv_add_remote) instead of exchanging them;
        the owners' memory must be addressable from this GPU (ranks of one
        process, on one GPU or on GPUs with peer access), so the transport
        must be a LocalTransport."""
        n_global = int(partition.offsets[-1])
        r0, r1 = partition.range(rank)
        (rd, cd, vd), (ro, co, vo), ghosts = rowblock_split(row, col, val, n_global, r0, r1)
        self.pf, self.part, self.rank, self.tr = platform, partition, rank, transport
        self.couplings = LaCouplings(partition, rank, ghosts).setup(transport)
        self.n_local = r1 - r0
        self.diag_host = (rd, cd, vd)            # the local block, for preconditioner set-ups
        self.diag = CSR_lMatrix.from_csr(platform, rd, cd, vd, n_cols=self.n_local, dtype=dtype)
        self.offdiag = (CSR_lMatrix.from_csr(platform, ro, co, vo, n_cols=len(ghosts), dtype=dtype)
                        if len(co) else None)
        self.dtype = dtype
        self.remote = bool(remote)
        if self.remote:
            if not hasattr(transport, "allgather_objects"):
                raise NotImplementedError("remote ghost reads need the owners' memory in this process "
                                          "(LocalTransport ranks); across processes they would need CUDA IPC")
            import torch
            dev = f"cuda:{platform.device}"
            cp = self.couplings
            with platform.on_stream():
                self._gowner = torch.from_numpy(cp.ghost_owner.copy()).to(dev)
                self._gindex = torch.from_numpy(cp.ghost_index.copy()).to(dev)
            size = transport.size
            self._reads_from = [q for q in range(size) if cp.ghost_offsets[q + 1] > cp.ghost_offsets[q]]
            self._read_by = [q for q in range(size) if cp.border_offsets[q + 1] > cp.border_offsets[q]]
            self._owner_tables = {}
            # ranks on other GPUs of this process: their memory over NVLink
            devices = transport.allgather_objects(platform.device)
            for q in self._reads_from:
                if devices[q] != platform.device:
                    rc = lib().b200la_enable_peer_access(platform.device, devices[q])
                    if rc:
                        raise B200Error(rc, f"no peer access from GPU {platform.device} to GPU {devices[q]}")

    def vector(self, data_or_n=None):
        return CoupledVector(self.pf, self.couplings, self.tr,
                             self.n_local if data_or_n is None else data_or_n, self.dtype)

    def cast(self, dtype):
        """A copy of this matrix in another precision on the same couplings
        (CoupledMatrix::CastFrom over lMatrix::CastFrom of both blocks)."""
        M = object.__new__(CoupledMatrix)
        M.__dict__.update(self.__dict__)
        M.dtype = dtype
        M.diag = self.diag.CastFrom(dtype)
        M.offdiag = self.offdiag.CastFrom(dtype) if self.offdiag is not None else None
        if self.remote:
            M._owner_tables = {}
        return M

    def _owners_table(self, ptrs):
        """Device array of the owners' vector pointers (cached per pointer set)."""
        t = self._owner_tables.get(ptrs)
        if t is None:
            import torch
            if len(self._owner_tables) >= 64:
                self.pf.sync()
                self._owner_tables.clear()
            host = torch.tensor(list(ptrs), dtype=torch.int64).pin_memory()
            with self.pf.on_stream():
                t = torch.empty(len(ptrs), dtype=torch.int64, device=f"cuda:{self.pf.device}")
                t.copy_(host, non_blocking=True)
            self.pf.stream().synchronize()
            self._owner_tables[ptrs] = t
        return t

    def _vector_mult_remote(self, x, y):
        import torch
        ls = self.pf.stream()
        ready = torch.cuda.Event()
        ready.record(ls)
        peers = self.tr.allgather_objects((x.interior.t.data_ptr(), ready))
        for q in self._reads_from:               # the owners' values are final
            ls.wait_event(peers[q][1])
        self.diag.VectorMult(x.interior, y.interior)
        if self.offdiag is not None:
            owners = self._owners_table(tuple(p for p, _ in peers))
            self.pf.check(lib().b200la_spmv_add_remote(self.pf.h, self.offdiag.h, C.c_void_p(owners.data_ptr()),
                                                       C.c_void_p(self._gowner.data_ptr()),
                                                       C.c_void_p(self._gindex.data_ptr()), y.interior.ptr),
                          "spmv_add_remote")
        done = torch.cuda.Event()
        done.record(ls)
        readers = self.tr.allgather_objects(done)
        for q in self._read_by:                  # x is not rewritten before its readers finish
            ls.wait_event(readers[q])

    def VectorMult(self, x, y):
        """y = A x (coupled_matrix.cc:433-467): the ghost exchange starts, the
        diagonal block is multiplied while it runs, then the off-diagonal block
        once the ghosts have arrived.  In remote mode the off-diagonal block
        reads the ghosts from their owners instead (no exchange)."""
        if self.remote:
            return self._vector_mult_remote(x, y)
        waits = x.begin_update()
        self.diag.VectorMult(x.interior, y.interior)
        x.end_update(waits)
        if self.offdiag is not None:
            lib().b200la_spmv_add(self.pf.h, self.offdiag.h, C.c_void_p(x.ghost.data_ptr()), y.interior.ptr)


def check(ctl, it, v, res0):
    """IterateControl::Check (src/common/iterate_control.cc:84-110): 0 iterate,
    1 absolute, 2 relative, 3 divergence, 4 iteration limit."""
    if v < ctl.abstol:
        return 1
    if v < ctl.reltol * res0:
        return 2
    if v > ctl.divtol * res0:
        return 3
    if it >= ctl.maxits:
        return 4
    return 0


class BlockPrecond:
    """A preconditioner of the local block only (op.diagonal(), as
    PreconditionerBlockJacobiStand and PreconditionerMultiColoring bind the lmp
    preconditioners, preconditioner_bjacobi_standard.cc:45-156,
    preconditioner_mc.cc:49-273): "none", "jacobi", or "mcsgs" -- the rank's
    block coloured and permuted, r gathered into that order, the MC-SGS
    sweeps, z scattered back.  Across ranks this is block-Jacobi."""

    def __init__(self, A, kind="jacobi"):
        if kind not in ("jacobi", "none", "mcsgs"):
            raise ValueError("precond: jacobi, none or mcsgs")
        self.A, self.kind = A, kind
        if kind == "jacobi":
            self.invd = A.vector()
            A.pf.check(lib().b200la_csr_invdiag(A.pf.h, A.diag.h, self.invd.interior.ptr), "invdiag")
        if kind == "mcsgs":
            import torch
            from . import Preconditioner
            rd, cd, vd = A.diag_host
            self.P = Preconditioner.MultiColoringSGS(A.pf, rd, cd, vd, dtype=A.dtype)
            with A.pf.on_stream():
                self._perm = torch.from_numpy(np.asarray(self.P.perm, np.int32).copy()).to(f"cuda:{A.pf.device}")
            self._rp, self._zp = A.pf.vector(A.n_local, A.dtype), A.pf.vector(A.n_local, A.dtype)

    def apply(self, src, dst):
        """dst = M^-1 src (local block; no communication)."""
        A = self.A
        if self.kind == "mcsgs":
            pf, n = A.pf, A.n_local
            if n == 0:
                return
            perm = C.c_void_p(self._perm.data_ptr())
            pf.check(lib().b200la_gather(pf.h, A.dtype, n, perm, src.interior.ptr, self._rp.ptr), "gather")
            self.P.ApplyPreconditioner(self._rp, self._zp)
            pf.check(lib().b200la_scatter(pf.h, A.dtype, n, perm, self._zp.ptr, dst.interior.ptr), "scatter")
            return
        dst.CopyFrom(src)
        if self.kind == "jacobi":
            dst.interior.ElementWiseMult(self.invd.interior)


class CoupledCG:
    """CG<LAD>::Solve (src/linear_solver/cg.cc:84-248) on coupled objects, with
    a BlockPrecond of the local block: precond "jacobi" (default), "none" or
    "mcsgs"."""

    def __init__(self, A, jacobi=True, precond=None):
        self.A = A
        self.kind = precond or ("jacobi" if jacobi else "none")
        self.M = BlockPrecond(A, self.kind)
        self.iter, self.res, self.res0 = 0, 0.0, 0.0

    def Solve(self, b, x, maxits=10000, abstol=0.0, reltol=1e-10, divtol=1e6):
        A = self.A
        r, p, z, Ap = (A.vector() for _ in range(4))
        A.VectorMult(x, r)                       # r = b - A x
        r.ScaleAdd(-1.0, b)
        res = r.Norm2()
        self.res0 = res
        ctl = Control(maxits, abstol, reltol, divtol)

        precond = self.M.apply

        status, it = check(ctl, 0, res, self.res0), 0
        precond(r, z)
        p.CopyFrom(z)
        rho = r.Dot(z)
        while status == 0:
            it += 1
            A.VectorMult(p, Ap)
            alpha = rho / Ap.Dot(p)
            x.Axpy(p, alpha)
            r.Axpy(Ap, -alpha)
            res = r.Norm2()
            status = check(ctl, it, res, self.res0)
            if status:
                break
            precond(r, z)
            rho_new = r.Dot(z)
            p.ScaleAdd(rho_new / rho, z)         # p = beta p + z
            rho = rho_new
        self.iter, self.res = it, res
        return status


class CoupledGMRES:
    """GMRES<LAD>::SolveRight (src/linear_solver/gmres.cc:285-510) on coupled
    objects: restarted GMRES(m), modified Gram-Schmidt with global dots, Givens
    rotations on the host (gmres.h:77-97), right preconditioning with a
    BlockPrecond of the local block.  As in the reference, a restart
    normalises the new residual by the last Givens estimate |g[j+1]|, not by
    its recomputed norm."""

    def __init__(self, A, m=30, precond="none"):
        if m < 1:
            raise ValueError("m >= 1 required")
        self.A, self.m = A, int(m)
        self.M = BlockPrecond(A, precond) if precond != "none" else None
        self.iter, self.res, self.res0 = 0, 0.0, 0.0

    def _prec(self, src, dst):
        if self.M is None:
            dst.CopyFrom(src)
        else:
            self.M.apply(src, dst)

    def Solve(self, b, x, maxits=10000, abstol=0.0, reltol=1e-9, divtol=1e6):
        A = self.A
        ctl = Control(maxits, abstol, reltol, divtol)
        mb = min(self.m, maxits)                                    # gmres.cc:301
        V = [A.vector() for _ in range(mb + 1)]
        w, z = A.vector(), A.vector()
        A.VectorMult(x, V[0])                                       # V0 = b - A x
        V[0].ScaleAdd(-1.0, b)
        res = V[0].Norm2()
        self.res0, it = res, 0
        conv = check(ctl, it, res, self.res0)
        while conv == 0:
            H = np.zeros((mb, mb + 1))                              # H[j, i]: column j
            g, cs, sn = np.zeros(mb + 1), np.zeros(mb + 1), np.zeros(mb + 1)
            V[0].Scale(1.0 / res)
            g[0] = res
            j_end = mb - 1
            for j in range(mb):
                it += 1
                self._prec(V[j], z)
                A.VectorMult(z, w)
                for i in range(j + 1):                              # modified Gram-Schmidt
                    H[j, i] = w.Dot(V[i])
                    w.Axpy(V[i], -1.0 * H[j, i])
                H[j, j + 1] = w.Norm2()
                w.Scale(1.0 / H[j, j + 1])
                V[j + 1].CopyFrom(w)
                for k in range(j):                                  # earlier rotations
                    t = cs[k] * H[j, k] + sn[k] * H[j, k + 1]
                    H[j, k + 1] = -sn[k] * H[j, k] + cs[k] * H[j, k + 1]
                    H[j, k] = t
                beta = np.sqrt(H[j, j] * H[j, j] + H[j, j + 1] * H[j, j + 1])
                cs[j], sn[j] = H[j, j] / beta, H[j, j + 1] / beta
                t = cs[j] * H[j, j] + sn[j] * H[j, j + 1]
                H[j, j + 1] = -sn[j] * H[j, j] + cs[j] * H[j, j + 1]
                H[j, j] = t
                t = cs[j] * g[j] + sn[j] * g[j + 1]
                g[j + 1] = -sn[j] * g[j] + cs[j] * g[j + 1]
                g[j] = t
                res = abs(g[j + 1])
                conv = check(ctl, it, res, self.res0)
                if conv:
                    j_end = j
                    break
            # UpdateSolution (gmres.cc:487-510): back substitution, x += M^-1 (V y)
            y = g.copy()
            for i in range(j_end, -1, -1):
                y[i] /= H[i, i]
                for k in range(i):
                    y[k] -= H[i, k] * y[i]
            z.Zeros()
            for k in range(j_end + 1):
                z.Axpy(V[k], y[k])
            self._prec(z, w)
            x.Axpy(w, 1.0)
            if conv == 0:
                A.VectorMult(x, V[0])
                V[0].ScaleAdd(-1.0, b)
        self.iter, self.res = it, res
        return conv


class CoupledMPIR:
    """MPIR<LAD_high, LAD_low>::Solve (src/linear_solver/mpir.cc:69-326) on
    coupled objects: the FP64 residual r = b - A x across ranks, its FP32 copy
    (CastInteriorFrom), an FP32 coupled Jacobi-CG correction A32 c = r32 to the
    inner tolerance, x += (double) c; stop on the outer residual relative to
    the first one (the benchmark's criterion, as b200la_mpir)."""

    def __init__(self, A, A32=None, inner_precond="jacobi", max_outer=50):
        from . import F32
        self.A = A
        self.A32 = A32 if A32 is not None else A.cast(F32)
        self.inner_precond, self.max_outer = inner_precond, int(max_outer)
        self.outer, self.inner_iters, self.res, self.res0 = 0, 0, 0.0, 0.0

    def Solve(self, b, x, maxits=50, abstol=0.0, reltol=1e-10, divtol=1e6, inner=(10000, 0.0, 1e-4, 1e6)):
        A, A32 = self.A, self.A32
        r = A.vector()
        A.VectorMult(x, r)                                  # mpir.cc:125-128
        r.ScaleAdd(-1.0, b)
        res = r.Norm2()
        self.res0 = res
        r32, c32, c64 = A32.vector(), A32.vector(), A.vector()
        solver = CoupledCG(A32, precond=self.inner_precond)
        outer = total = 0
        limit = min(self.max_outer, maxits)
        while res > abstol and res > reltol * self.res0 and res < divtol and outer < limit:
            outer += 1
            r32.CastInteriorFrom(r)                         # mpir.cc:169-170
            c32.Zeros()
            solver.Solve(r32, c32, *inner)                  # mpir.cc:193
            total += solver.iter
            c64.CastInteriorFrom(c32)                       # mpir.cc:223, 253
            x.Axpy(c64, 1.0)
            A.VectorMult(x, r)                              # mpir.cc:271-273
            r.ScaleAdd(-1.0, b)
            res = r.Norm2()
        self.outer, self.inner_iters, self.res = outer, total, res
        return 1 if res < abstol else 2 if res < reltol * self.res0 else 3 if res >= divtol else 4


class CoupledAsyncJacobi:
    """AsynchronousIterationGPU<LAD>::SolveNormal / SolveDamped
    (src/linear_solver/gpu-based/async_iter_gpu.cc:538-630, 780-900) on coupled
    objects.  One check interval is n_global global iterations; each is n_block
    launches of n_inner asynchronous sweeps over this rank's rows
    (b200la_async_jacobi, the ghost values fixed), with the ghost update
    (GlobalUpdate) between global iterations.  Then the global residual
    ||b - A x|| (which updates the ghosts again) and IterateControl::Check on
    the sweep count."""

    def __init__(self, A, n_global=1, n_block=10, n_inner=10, w=1.0):
        if min(n_global, n_block, n_inner) < 1 or not w > 0.0:
            raise ValueError("n_global, n_block, n_inner >= 1 and w > 0 required")
        self.A, self.n_global, self.n_block, self.n_inner, self.w = A, n_global, n_block, n_inner, float(w)
        self.iter, self.res, self.res0 = 0, 0.0, 0.0

    def _residual(self, b, x, r):
        self.A.VectorMult(x, r)
        r.ScaleAdd(-1.0, b)                      # r = b - A x
        return r.Norm2()

    def Solve(self, b, x, maxits=100000, abstol=0.0, reltol=1e-8, divtol=1e6):
        A = self.A
        ctl = Control(maxits, abstol, reltol, divtol)
        # one batch per call: no tolerance, the limit at the batch's sweeps
        one = Control(self.n_block * self.n_inner, 0.0, 0.0, 1e300)
        r = A.vector()
        res = self._residual(b, x, r)
        self.res0, it = res, 0
        status = check(ctl, it, res, self.res0)
        oh = A.offdiag.h if A.offdiag is not None else None
        while status == 0:
            for g in range(self.n_global):
                out = Result()
                ghost = C.c_void_p(x.ghost.data_ptr()) if oh is not None else None
                A.pf.check(lib().b200la_async_jacobi(A.pf.h, A.diag.h, oh, b.interior.ptr, x.interior.ptr, ghost,
                                                     self.n_inner, self.n_block, self.w, C.byref(one),
                                                     C.byref(out)), "async_jacobi")
                it += self.n_block * self.n_inner
                if g < self.n_global - 1:
                    x.UpdateGhost()
            res = self._residual(b, x, r)
            status = check(ctl, it, res, self.res0)
        self.iter, self.res = it, res
        return status


# ------------------------------------------------------------ native coupled layer (C ABI)

COMM_ID_BYTES = 128


class Comm:
    """A b200la_comm: the communicator of the native coupled layer.

    ``Comm.local_group(size)`` -- communicators for ranks that are threads of
    this process (device copies ordered by events, a host barrier);
    ``Comm.nccl(platform, uid, rank, size)`` -- an NCCL communicator of this
    rank on the platform's GPU, ``uid`` from ``Comm.unique_id()`` on rank 0,
    handed to every rank by the caller (a torch.distributed broadcast, MPI)."""

    def __init__(self, handle):
        self.h = handle
        r, n = C.c_int(), C.c_int()
        lib().b200la_comm_info(self.h, C.byref(r), C.byref(n))
        self.rank, self.size = r.value, n.value

    @staticmethod
    def unique_id():
        buf = (C.c_char * COMM_ID_BYTES)()
        rc = lib().b200la_comm_unique_id(buf)
        if rc:
            raise B200Error(rc, "comm_unique_id: NCCL could not be loaded")
        return bytes(buf)

    @classmethod
    def nccl(cls, platform, uid, rank, size):
        buf = (C.c_char * COMM_ID_BYTES).from_buffer_copy(uid)
        h = C.c_void_p()
        platform.check(lib().b200la_comm_create_nccl(platform.h, buf, rank, size, C.byref(h)), "comm_create_nccl")
        return cls(h)

    @classmethod
    def local_group(cls, size):
        arr = (C.c_void_p * size)()
        rc = lib().b200la_comm_create_local(size, arr)
        if rc:
            raise B200Error(rc, "comm_create_local")
        return [cls(C.c_void_p(arr[q])) for q in range(size)]

    def close(self):
        if self.h:
            lib().b200la_comm_destroy(self.h)
            self.h = None


class NativeCoupledMatrix:
    """CoupledMatrix on the C ABI (b200la_coupled_*): the couplings are set up
    on the host once through ``transport`` (the index lists every peer needs,
    as LaCouplings::InitializeCouplings does with MPI), and the data path --
    border gather, ghost exchange overlapping the diagonal-block product,
    off-diagonal product, cross-rank sums, the coupled CG -- runs in the
    library over ``comm``."""

    def __init__(self, platform, comm, transport, partition, rank, row, col, val, dtype=F64):
        n_global = int(partition.offsets[-1])
        r0, r1 = partition.range(rank)
        (rd, cd, vd), (ro, co, vo), ghosts = rowblock_split(row, col, val, n_global, r0, r1)
        self.pf, self.comm, self.rank, self.dtype = platform, comm, rank, dtype
        self.couplings = LaCouplings(partition, rank, ghosts).setup(transport)
        self.n_local = r1 - r0
        self.diag_host = (rd, cd, vd)            # the local block, for block preconditioner set-ups
        self.diag = CSR_lMatrix.from_csr(platform, rd, cd, vd, n_cols=self.n_local, dtype=dtype)
        self.offdiag = (CSR_lMatrix.from_csr(platform, ro, co, vo, n_cols=len(ghosts), dtype=dtype)
                        if len(co) else None)
        self._precs = {}
        cp = self.couplings
        self._go = np.ascontiguousarray(cp.ghost_offsets, np.int32)
        self._bo = np.ascontiguousarray(cp.border_offsets, np.int32)
        self._bi = np.ascontiguousarray(cp.border_indices, np.int32)
        h = C.c_void_p()
        platform.check(lib().b200la_coupled_create(platform.h, comm.h, self.diag.h,
                                                   self.offdiag.h if self.offdiag is not None else None,
                                                   self._go.ctypes.data, self._bo.ctypes.data,
                                                   self._bi.ctypes.data if self._bi.size else None, C.byref(h)),
                       "coupled_create")
        self.h = h
        self.iter, self.res, self.res0, self.status = 0, 0.0, 0.0, 0

    def vector(self, data_or_n=None):
        return self.pf.vector(self.n_local if data_or_n is None else data_or_n, self.dtype)

    def UpdateGhost(self, x):
        """The ghost values of x (CoupledVector::UpdateGhost), as a host array."""
        import torch
        with self.pf.on_stream():
            g = torch.zeros(len(self.couplings.ghost_global),
                            dtype=torch.float64 if self.dtype == F64 else torch.float32, device=f"cuda:{self.pf.device}")
        self.pf.check(lib().b200la_coupled_update_ghost(self.pf.h, self.h, x.ptr,
                                                        C.c_void_p(g.data_ptr()) if g.numel() else None),
                      "coupled_update_ghost")
        return g.cpu().numpy()

    def VectorMult(self, x, y):
        self.pf.check(lib().b200la_coupled_spmv(self.pf.h, self.h, x.ptr, y.ptr), "coupled_spmv")

    def Dot(self, x, y):
        out = C.c_double()
        self.pf.check(lib().b200la_coupled_dot(self.pf.h, self.h, x.ptr, y.ptr, C.byref(out)), "coupled_dot")
        return out.value

    def CG(self, b, x, precond=None, maxits=100000, abstol=0.0, reltol=1e-10, divtol=1e6):
        """CG<LAD>::Solve over the coupled rows, block-Jacobi across ranks:
        precond None, "jacobi" (the Jacobi preconditioner of this rank's
        diagonal block) or "mcsgs" (the multicoloured symmetric Gauss-Seidel
        of the block, PreconditionerMultiColoring on op.diagonal())."""
        from . import Preconditioner
        P = None
        if precond is not None:
            if precond not in self._precs:
                if precond == "jacobi":
                    self._precs[precond] = Preconditioner.Jacobi(self.pf, self.diag)
                elif precond == "mcsgs":
                    self._precs[precond] = Preconditioner.MultiColoringSGS(self.pf, *self.diag_host,
                                                                           dtype=self.dtype)
                else:
                    raise ValueError(f"unknown block preconditioner {precond!r}")
            P = self._precs[precond]
        ctl, res = Control(maxits, abstol, reltol, divtol), Result()
        self.pf.check(lib().b200la_coupled_cg(self.pf.h, self.h, P.h if P is not None else None, b.ptr, x.ptr,
                                              C.byref(ctl), C.byref(res)), "coupled_cg")
        self.iter, self.res, self.res0, self.status = res.iters, res.res, res.res0, res.status
        return res.status

    def close(self):
        if getattr(self, "h", None):
            self.pf.sync()
            lib().b200la_coupled_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
