"""
An in-process stand-in for the torch.distributed calls DistributedSolver
makes, with one host thread per rank: lets the multi-rank solver run its
real patch kernels on a single GPU, the ranks' kernels never waiting on one
another on the device (every exchange is a host-side copy between
synchronised streams). Test infrastructure only.
"""

import threading
from enum import Enum

import torch


class ReduceOp(Enum):
    MAX = "max"
    SUM = "sum"


class P2POp:
    def __init__(self, op, tensor, peer, group=None):
        self.op, self.tensor, self.peer = op, tensor, peer


def _sync():
    if torch.cuda.is_available():
        torch.cuda.synchronize()


class _Done:
    def wait(self):
        return True


class ThreadComm:
    """World of `size` ranks; each rank's thread calls set_rank(r) first."""

    ReduceOp = ReduceOp
    P2POp = P2POp

    def __init__(self, size, timeout=60.0):
        self.size = size
        self.timeout = timeout
        self._local = threading.local()
        self._barrier = threading.Barrier(size, timeout=timeout)
        self._slots = [None] * size
        self._mail = {}
        self._cv = threading.Condition()

    def set_rank(self, r):
        self._local.rank = r

    def get_rank(self, group=None):
        return self._local.rank

    def get_world_size(self, group=None):
        return self.size

    def get_global_rank(self, group, r):
        return r

    # point to point: the op tags name functions, as in torch.distributed
    def isend(self, *a, **k):
        raise RuntimeError("use batch_isend_irecv")

    def irecv(self, *a, **k):
        raise RuntimeError("use batch_isend_irecv")

    def batch_isend_irecv(self, ops):
        me = self.get_rank()
        _sync()
        with self._cv:
            for op in ops:
                if op.op == self.isend:
                    self._mail.setdefault((me, op.peer), []).append(op.tensor.clone())
            self._cv.notify_all()
        for op in ops:
            if op.op == self.irecv:
                with self._cv:
                    ok = self._cv.wait_for(lambda: self._mail.get((op.peer, me)), timeout=self.timeout)
                    if not ok:
                        raise TimeoutError(f"rank {me}: nothing from {op.peer}")
                    data = self._mail[(op.peer, me)].pop(0)
                op.tensor.copy_(data)
        _sync()
        return [_Done() for _ in ops]

    def _gather(self, value):
        me = self.get_rank()
        self._barrier.wait()
        self._slots[me] = value
        self._barrier.wait()
        out = list(self._slots)
        self._barrier.wait()
        return out

    def all_reduce(self, tensor, op=ReduceOp.SUM, group=None):
        _sync()
        vals = self._gather(tensor.detach().clone())
        res = vals[0].clone()
        for v in vals[1:]:
            res = torch.maximum(res, v) if op == ReduceOp.MAX else res + v
        tensor.copy_(res)
        _sync()

    def all_gather_object(self, out, obj, group=None):
        vals = self._gather(obj)
        out[:] = vals

    def run(self, fn):
        """fn(rank) on `size` threads; returns the results in rank order."""
        results = [None] * self.size
        errors = []

        def body(r):
            try:
                self.set_rank(r)
                results[r] = fn(r)
            except BaseException as exc:
                errors.append(exc)
                self._barrier.abort()

        threads = [threading.Thread(target=body, args=(r,)) for r in range(self.size)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return results
