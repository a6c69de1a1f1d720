"""The allocation-free PCG entry point (nb2_pcg_solve_noalloc).

It serves callers that must not allocate device memory while they solve -- codes that place
every device byte through their own pool or arena, or that must not trigger allocator growth
in the middle of a time step.  They hand in device buffers they own; the solver's work space is
a fixed array inside the library.  This test owns its device buffers (through torch), calls the
entry point twice in a row through the C-ABI and checks both results (solution, iteration count
and final relative residual) against the allocating entry point nb2_pcg_solve on the same
systems; then it checks the refusals (a system beyond the fixed work space, a column index out
of range), the iteration limit status, and a call on a stream the caller created.

The file name sorts last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import random_displacement, rel_err
from neon_b200 import problem as P

pytestmark = pytest.mark.gpu


def _system(api, n_cells, seed):
    """A Dirichlet-constrained linear-elastic stiffness (host CSR) and a right-hand side."""
    pr = P.config_c1(n_cells)
    g = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    g.update_internal_variables(random_displacement(pr.mesh, 1e-4, seed))
    K, _ = g.assemble()
    rp, col = g.sparsity_pattern()
    rng = np.random.Generator(np.random.PCG64(seed))
    b = rng.standard_normal(g.ndofs)
    dofs = np.concatenate([t.dofs for t in pr.dirichlet])
    g.apply_dirichlet(dofs, K, b)
    g.close()
    return rp, col, K, b


def test_noalloc_pcg_matches_allocating_entry_point():
    import torch
    from neon_b200 import api, build
    build.build()
    L = api.lib()
    tol, maxit = 1e-12, 20000
    rp, col, K, _ = _system(api, 8, 3)
    n = len(rp) - 1
    assert n <= 131072
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(K).to(dev)
    for call, seed in enumerate((5, 6)):  # two calls in a row share the fixed work space
        b = np.random.Generator(np.random.PCG64(seed)).standard_normal(n)
        x_ref = np.zeros(n)
        cg = api.ConjugateGradient(tol, maxit)
        cg.solve((rp, col, K), x_ref, b)
        d_b = torch.from_numpy(b).to(dev)
        d_x = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        it = C.c_int32()
        err = C.c_double()
        st = L.nb2_pcg_solve_noalloc(n, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                     d_b.data_ptr(), d_x.data_ptr(), tol, maxit, None,
                                     C.byref(it), C.byref(err))
        assert st == api.OK, (call, st)
        x = d_x.cpu().numpy()
        assert rel_err(x, x_ref) < 1e-9, call
        assert abs(it.value - cg.iterations) <= max(2, 0.02 * cg.iterations)
        assert err.value <= tol and cg.error <= tol
        if it.value == cg.iterations:  # same iterates: the same final residual
            assert abs(err.value - cg.error) <= 1e-6 * cg.error
    # a system beyond the fixed work space is refused, not run
    st = L.nb2_pcg_solve_noalloc(131072 + 1, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                 d_b.data_ptr(), d_x.data_ptr(), tol, maxit, None, None, None)
    assert st == api.E_INPUT
    # a column index outside [0, n) (inside the caller's buffer) is refused before any solve
    bad_col = col.copy()
    bad_col[len(bad_col) // 2] = n
    d_bad = torch.from_numpy(bad_col).to(dev)
    torch.cuda.synchronize()
    st = L.nb2_pcg_solve_noalloc(n, d_rp.data_ptr(), d_bad.data_ptr(), d_val.data_ptr(),
                                 d_b.data_ptr(), d_x.data_ptr(), tol, maxit, None, None, None)
    assert st == api.E_INPUT
    # the iteration limit gives the same status as the allocating entry point
    it = C.c_int32()
    st = L.nb2_pcg_solve_noalloc(n, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                 d_b.data_ptr(), d_x.data_ptr(), tol, 3, None, C.byref(it), None)
    assert st == api.E_CG_MAXIT and it.value == 3
    with pytest.raises(api.ComputationalError):
        api.ConjugateGradient(tol, 3).solve((rp, col, K), np.zeros(n), b)
    # on a stream the caller created, after work queued on it
    s = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        d_b2 = d_b * 2.0
        d_x2 = torch.zeros(n, dtype=torch.float64, device=dev)
    err = C.c_double()
    st = L.nb2_pcg_solve_noalloc(n, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                 d_b2.data_ptr(), d_x2.data_ptr(), tol, maxit,
                                 C.c_void_p(s.cuda_stream), None, C.byref(err))
    assert st == api.OK
    s.synchronize()
    assert rel_err(d_x2.cpu().numpy(), 2.0 * x_ref) < 1e-9
