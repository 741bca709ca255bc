"""Python side of the batched SPD entry points (include/plasma_b200.h).

A Batch owns a plan: the orders of its matrices, their packed layout in one
device array (matrix i column-major n_i x n_i at off_a[i], vector i at
off_b[i]) and the processing order.  Arrays are CUDA torch tensors; every
operation is one kernel launch (or one CUDA-graph replay) enqueued on torch's
current stream.  No reference counterpart: PLASMA solves one matrix at a time.
"""
import ctypes

import numpy as np
import torch

from . import PlasmaRealDouble, PlasmaRealFloat, lib

_CUDA_STREAM_LEGACY = 1          # cudaStreamLegacy


class Batch:
    def __init__(self, sizes, dtype=torch.float64, graph=False):
        self.L = lib()
        self.sizes = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32))
        self.dtype = dtype
        self.prec = PlasmaRealDouble if dtype == torch.float64 else PlasmaRealFloat
        self._p = "d" if dtype == torch.float64 else "s"
        plan = ctypes.c_void_p()
        rc = self.L.plasma_batch_create(self.prec, len(self.sizes),
                                        self.sizes.ctypes.data, ctypes.byref(plan))
        if rc != 0:
            raise RuntimeError(f"plasma_batch_create failed: {rc}")
        self.plan = plan
        self.off_a = np.zeros(len(self.sizes), dtype=np.int64)
        self.off_b = np.zeros(len(self.sizes), dtype=np.int64)
        self.L.plasma_batch_offsets(plan, self.off_a.ctypes.data, self.off_b.ctypes.data)
        self.matrix_elems = self.L.plasma_batch_matrix_elems(plan)
        self.vector_elems = self.L.plasma_batch_vector_elems(plan)
        if graph:
            self.L.plasma_batch_set_graph(plan, 1)

    def close(self):
        if self.plan:
            self.L.plasma_batch_destroy(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ packing
    def pack_matrices(self, mats):
        """One device array holding every matrix (numpy, any order: each is
        symmetric or its lower triangle is what counts)."""
        host = np.zeros(max(self.matrix_elems, 1), dtype=np.float64)
        for i, m in enumerate(mats):
            n = self.sizes[i]
            host[self.off_a[i]:self.off_a[i] + n * n] = np.asarray(m, np.float64).reshape(n, n).T.ravel()
        return torch.tensor(host, dtype=self.dtype, device="cuda")

    def pack_vectors(self, vecs):
        host = np.zeros(max(self.vector_elems, 1), dtype=np.float64)
        for i, v in enumerate(vecs):
            n = self.sizes[i]
            host[self.off_b[i]:self.off_b[i] + n] = np.asarray(v, np.float64).ravel()
        return torch.tensor(host, dtype=self.dtype, device="cuda")

    def matrix(self, A, i):
        """Matrix i of a packed array as a numpy (row-major) array."""
        n = int(self.sizes[i])
        h = A[self.off_a[i]:self.off_a[i] + n * n].double().cpu().numpy()
        return h.reshape(n, n).T.copy()

    def vector(self, B, i):
        n = int(self.sizes[i])
        return B[self.off_b[i]:self.off_b[i] + n].double().cpu().numpy().copy()

    # --------------------------------------------------------- operations
    def _call(self, name, *args):
        # enqueue on torch's current stream, so that the operation is ordered
        # with the torch work that produced its inputs and consumes its outputs
        # (torch reports the legacy default stream as handle 0, which the
        # library reads as "its own stream": pass cudaStreamLegacy instead)
        prev = self.L.plasma_get_stream()
        cur = torch.cuda.current_stream().cuda_stream or _CUDA_STREAM_LEGACY
        self.L.plasma_set_stream(ctypes.c_void_p(cur))
        try:
            rc = getattr(self.L, f"plasma_{self._p}{name}")(self.plan, *args)
        finally:
            self.L.plasma_set_stream(ctypes.c_void_p(prev))
        if rc != 0:
            raise RuntimeError(f"plasma_{self._p}{name} failed: {rc}")

    def posv(self, A, B, info):
        self._call("posv_batched", A.data_ptr(), B.data_ptr(), info.data_ptr())

    def potrf(self, A, info):
        self._call("potrf_batched", A.data_ptr(), info.data_ptr())

    def potrs(self, Lf, B):
        self._call("potrs_batched", Lf.data_ptr(), B.data_ptr())

    def potrf_adjoint(self, Lf, Lbar):
        self._call("potrf_adjoint_batched", Lf.data_ptr(), Lbar.data_ptr())

    def potrs_adjoint(self, Lf, X, Xbar, Lbar):
        self._call("potrs_adjoint_batched", Lf.data_ptr(), X.data_ptr(), Xbar.data_ptr(),
                   Lbar.data_ptr())

    def info_buffer(self):
        return torch.zeros(max(len(self.sizes), 1), dtype=torch.int32, device="cuda")
