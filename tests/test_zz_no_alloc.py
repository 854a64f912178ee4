"""mzb_conj_grad_noalloc: the CG solve for callers that cannot allocate device memory
(their host owns every allocation, or they must not take the synchronisation an
allocation can imply). It must give the same answer as the allocating entry point
mzb_conj_grad on the same inputs, call after call, although its work arrays are one
static device array shared by all calls, and the implicit-Jacobi solves must match the
CPU oracle's conj_grad. This file is collected last so that a failure here stops a run
only after every other test ran."""
import numpy as np
import pytest

from maze_poisson_b200.c_api import CAPI

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_noalloc_cg_matches_allocating_entry_point(product_path, oracle_lib):
    import torch

    lib = CAPI(product_path)
    lib.solver_initialize()  # the allocating entry point uses the library's system state
    stream = torch.cuda.current_stream().cuda_stream
    # calls in a row with different sizes and preconditioners, then the first again: the
    # shared work area keeps the previous call's contents in between. n = 64 and 32 take
    # the TMA-staged CG kernel, n = 40 and 20 (not multiples of 16) the general engine.
    for n, precond, seed in [(64, 0, 1), (32, 1, 2), (40, 1, 4), (20, 0, 5), (64, 0, 3)]:
        rng = np.random.default_rng(seed)
        xt = rng.standard_normal((n, n, n))
        b = np.empty_like(xt)
        lib.mzb_laplace(xt, b, n)
        x0 = 0.05 * rng.standard_normal((n, n, n))
        x_ref = np.empty_like(b)
        it_ref = lib.mzb_conj_grad(b, x0, x_ref, 1e-9, n, precond)

        db = torch.from_numpy(b).cuda()
        dx0 = torch.from_numpy(x0).cuda()
        dx = torch.full_like(db, float("nan"))
        torch.cuda.synchronize()
        it = lib.mzb_conj_grad_noalloc(db.data_ptr(), dx0.data_ptr(), dx.data_ptr(), 1e-9, n, precond,
                                       stream)
        assert it == it_ref and it > 0, (n, it, it_ref)
        x = dx.cpu().numpy()
        assert rel(x, x_ref) < 1e-12, n
        if precond == 0:  # the oracle restates the reference's conj_grad (implicit Jacobi)
            x_orc = np.empty_like(b)
            it_orc = oracle_lib.orc_conj_grad(b.reshape(-1), x0.reshape(-1), x_orc.reshape(-1), 1e-9, n)
            assert abs(it - it_orc) <= 1, (n, it, it_orc)
            assert rel(x, x_orc) < 1e-10, n


def test_noalloc_rejects_what_it_cannot_serve(product_path):
    import torch

    lib = CAPI(product_path)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    assert lib.mzb_conj_grad_noalloc(p, p, p, 1e-9, 80, 0, None) == -2
    assert lib.mzb_conj_grad_noalloc(p, p, p, 1e-9, 1, 0, None) == -2
    assert lib.mzb_conj_grad_noalloc(p, p, p, 1e-9, 16, 2, None) == -2
    host = np.zeros(16 ** 3)
    assert lib.mzb_conj_grad_noalloc(host.ctypes.data, p, p, 1e-9, 16, 0, None) == -2
