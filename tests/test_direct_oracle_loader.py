"""The GPU direct-solve oracle's libraries load on a machine without a GPU and export the entry
points tests/gpu_direct.py binds (no device call is made)."""
from gpu_direct import _load


def test_cusolver_and_cusparse_export_the_bound_symbols():
    solver = _load("cusolver", "libcusolver.so.11")
    sparse = _load("cusparse", "libcusparse.so.12")
    for name in ("cusolverSpCreate", "cusolverSpSetStream", "cusolverSpDcsrlsvchol", "cusolverSpDestroy"):
        assert hasattr(solver, name), name
    for name in ("cusparseCreateMatDescr", "cusparseSetMatType", "cusparseSetMatIndexBase",
                 "cusparseDestroyMatDescr"):
        assert hasattr(sparse, name), name
