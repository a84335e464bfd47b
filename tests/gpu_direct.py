"""A Float64 sparse direct solve on the GPU, as a test oracle: cuSOLVER's sparse Cholesky
(cusolverSpDcsrlsvchol, device path) on the assembled system in CSR.

TEST INFRASTRUCTURE ONLY: it stands in for the reference's CholeskyDirectSolver (CHOLMOD on the CPU,
src/linear_solver.jl:127-221) as an exact reference on the GPU; nothing in the product calls it.
The matrix is reordered with symrcm (reorder = 1) before the factorisation.  Measured host wall time
on one B200, copies included: 2.5 s at 301^2, 3.6 s at 512 x 360, 36 s at 1024^2, about 10x per 4x
in cells and slower than SciPy's SuperLU on the host.  Use it at 1024^2 and below; at 4096^2 the
tight Float64 CG is the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import site

import numpy as np


def _load(sub: str, name: str) -> C.CDLL:
    for d in site.getsitepackages():
        p = os.path.join(d, "nvidia", sub, "lib", name)
        if os.path.exists(p):
            return C.CDLL(p)
    return C.CDLL(name)


def cholesky_solve(M, b: np.ndarray, tol: float = 1e-14) -> np.ndarray:
    """Solves M x = b (M a SciPy sparse SPD matrix, b a vector) on the current CUDA device."""
    import torch

    sparse = _load("cusparse", "libcusparse.so.12")
    solver = _load("cusolver", "libcusolver.so.11")
    M = M.tocsr()
    m, nnz = M.shape[0], M.nnz
    dev = torch.device("cuda")
    val = torch.from_numpy(np.ascontiguousarray(M.data, dtype=np.float64)).to(dev)
    rowp = torch.from_numpy(np.ascontiguousarray(M.indptr, dtype=np.int32)).to(dev)
    col = torch.from_numpy(np.ascontiguousarray(M.indices, dtype=np.int32)).to(dev)
    rhs = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).to(dev)
    x = torch.zeros(m, dtype=torch.float64, device=dev)
    descr, handle = C.c_void_p(), C.c_void_p()
    assert sparse.cusparseCreateMatDescr(C.byref(descr)) == 0
    try:
        assert sparse.cusparseSetMatType(descr, 0) == 0        # general
        assert sparse.cusparseSetMatIndexBase(descr, 0) == 0   # zero-based
        assert solver.cusolverSpCreate(C.byref(handle)) == 0
        try:
            assert solver.cusolverSpSetStream(handle, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
            sing = C.c_int(-2)
            st = solver.cusolverSpDcsrlsvchol(handle, C.c_int(m), C.c_int(nnz), descr,
                                              C.c_void_p(val.data_ptr()), C.c_void_p(rowp.data_ptr()),
                                              C.c_void_p(col.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                              C.c_double(tol), C.c_int(1), C.c_void_p(x.data_ptr()),
                                              C.byref(sing))
            torch.cuda.synchronize()
            if st != 0:
                raise RuntimeError(f"cusolverSpDcsrlsvchol returned status {st}")
            if sing.value != -1:
                raise RuntimeError(f"matrix not positive definite at row {sing.value}")
        finally:
            solver.cusolverSpDestroy(handle)
    finally:
        sparse.cusparseDestroyMatDescr(descr)
    return x.cpu().numpy()
