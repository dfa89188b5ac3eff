"""Fake MPI module (single process).  See the package docstring."""
import os
import numpy as np

PROC_NULL = -2
SUM = "sum"
MAX = "max"
MIN = "min"
_initialized = [False]


def Is_initialized():
    return _initialized[0]


def Init():
    _initialized[0] = True


def Finalize():
    pass


class _Comm:
    def __init__(self, periods=(1, 1, 1)):
        self.periods = list(periods)

    def Get_rank(self):
        return int(os.environ.get("PF_FAKE_RANK", "0"))

    def Get_size(self):
        return 1

    def Create_cart(self, dims, periods=None, reorder=True):
        return _Comm(periods if periods is not None else (0, 0, 0))

    def Get_coords(self, rank):
        return (0, 0, 0)

    def Sub(self, remain):
        return _Comm(self.periods)

    def Shift(self, direction, disp):
        if self.periods[direction]:
            return (0, 0)
        return (PROC_NULL, PROC_NULL)

    def Sendrecv(self, sendbuf, dest, sendtag, recvbuf, source, recvtag):
        if source != PROC_NULL and dest != PROC_NULL:
            np.copyto(recvbuf, np.asarray(sendbuf).reshape(recvbuf.shape))

    def Allreduce(self, sendbuf, recvbuf, op=None):
        np.copyto(recvbuf, sendbuf)

    def Barrier(self):
        pass

    def Free(self):
        pass


COMM_WORLD = _Comm()
