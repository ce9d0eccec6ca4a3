"""hrn_misfit_noalloc, the misfit entry whose scratch is a static device array,
against hrn_misfit on the same forward history and data.  Collected last so it
also runs after every other test has used the library in this process.

Callers that cannot let a library allocate device memory (a driver whose memory
pool already holds the device's free memory, or a loop that must not take the
device-wide synchronization of cudaMalloc / cudaFree) use this entry; the tests
check its value against hrn_misfit on two calls in a row, on uneven shots with
masked receivers and receivers sharing an equation, with the device's free memory
held by torch's caching allocator, and that a host pointer is refused before any
kernel is launched."""
import ctypes as C

import numpy as np
import pytest

from problems import RHO, tiny

pytestmark = pytest.mark.gpu


def _solver(p, precision, lam, mu):
    from hirensi_b200.solver import Solver
    s = Solver(precision)
    s.set_mesh(p["mesh"], RHO)
    s.assemble(lam, mu)
    s.set_history(p["mesh"].store_eq)
    s.set_shots(p["nstep"], p["dt"], p["src_eq"], p["src_b"], p["ftab"])
    s.set_receivers(p["eqdis"], p["eqdis_map"])
    return s


def _noalloc(lib, s, d):
    out = C.c_double(np.nan)
    rc = lib.hrn_misfit_noalloc(s.h, C.c_void_p(d.data_ptr()), C.byref(out))
    assert rc == 0, lib.hrn_last_error(s.h)
    return out.value


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_misfit_matches_misfit_on_consecutive_calls(gpu_lib, precision):
    import torch
    p = tiny(nshot=2, nstep=150)
    s = _solver(p, precision, p["lam_t"], p["mu_t"])
    s.forward()
    dis = s.traces()                       # data of the true model, [nshot][nrec3][nstep+1]
    d = torch.from_numpy(dis).to("cuda:0")
    torch.cuda.synchronize()
    s.assemble(p["lam"], p["mu"])
    s.forward()
    ref = s.misfit(dis)
    assert ref > 0.0
    first = _noalloc(gpu_lib, s, d)
    second = _noalloc(gpu_lib, s, d)
    assert abs(first - ref) <= 1e-14 * ref
    assert second == first
    # a one-shot problem after the two-shot one: no stale terms from the shared scratch
    p1 = tiny(nshot=1, nstep=90, seed=3)
    s1 = _solver(p1, precision, p1["lam_t"], p1["mu_t"])
    s1.forward()
    dis1 = s1.traces()
    d1 = torch.from_numpy(dis1).to("cuda:0")
    torch.cuda.synchronize()
    s1.assemble(p1["lam"], p1["mu"])
    s1.forward()
    ref1 = s1.misfit(dis1)
    assert abs(_noalloc(gpu_lib, s1, d1) - ref1) <= 1e-14 * ref1
    assert abs(_noalloc(gpu_lib, s, d) - ref) <= 1e-14 * ref
    s1.close()
    s.close()


def test_noalloc_rejects_problems_above_the_scratch_limit(gpu_lib):
    p = tiny(nshot=8, nstep=16384)
    s = _solver(p, "fp64", p["lam"], p["mu"])
    out = C.c_double()
    rc = gpu_lib.hrn_misfit_noalloc(s.h, None, C.byref(out))
    assert rc == 1                          # HRN_EARG
    assert b"131072" in gpu_lib.hrn_last_error(s.h)
    s.close()


def test_noalloc_uneven_shots_masks_and_shared_equations(gpu_lib):
    """Shots of uneven record length, receiver masks and receivers listed twice (their
    residuals add before squaring): the branches of the misfit kernel that an even
    batch does not take."""
    import torch
    p = tiny(nshot=3, nstep=120)
    lens = np.array([120, 70, 95], np.int32)
    eqdis = np.concatenate([p["eqdis"], p["eqdis"][:6]])
    emap = np.concatenate([p["eqdis_map"], p["eqdis_map"][:6]])
    nrec3 = eqdis.size
    mask = np.ones((3, nrec3), np.uint8)
    mask[1, nrec3 // 2:] = 0
    mask[2, ::2] = 0
    s = _solver(p, "fp64", p["lam_t"], p["mu_t"])
    s.set_receivers(eqdis, emap)
    s.set_shot_records(lens, mask)
    s.forward()
    dis = s.traces()
    rng = np.random.default_rng(7)
    dis = np.ascontiguousarray(dis * (1.0 + 0.05 * rng.standard_normal(dis.shape)))
    d = torch.from_numpy(dis).to("cuda:0")
    torch.cuda.synchronize()
    s.assemble(p["lam"], p["mu"])
    s.forward()
    ref = s.misfit(dis)
    assert ref > 0.0
    first = _noalloc(gpu_lib, s, d)
    second = _noalloc(gpu_lib, s, d)
    assert abs(first - ref) <= 1e-14 * ref
    assert second == first
    s.close()


def test_noalloc_with_the_free_memory_held_by_torch(gpu_lib):
    """The entry runs while torch's caching allocator holds all but 64 MiB of the
    device's free memory, and the device's free memory does not change across it."""
    import torch
    p = tiny(nshot=2, nstep=150)
    s = _solver(p, "fp64", p["lam_t"], p["mu_t"])
    s.forward()
    dis = s.traces()
    d = torch.from_numpy(dis).to("cuda:0")
    s.assemble(p["lam"], p["mu"])
    s.forward()
    ref = s.misfit(dis)
    _noalloc(gpu_lib, s, d)                 # kernels loaded, scratch address known
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    hold = torch.empty(max(free - (64 << 20), 0), dtype=torch.uint8, device="cuda:0")
    try:
        torch.cuda.synchronize()
        before, _ = torch.cuda.mem_get_info()
        first = _noalloc(gpu_lib, s, d)
        second = _noalloc(gpu_lib, s, d)
        after, _ = torch.cuda.mem_get_info()
    finally:
        del hold
        torch.cuda.empty_cache()
    assert after == before
    assert abs(first - ref) <= 1e-14 * ref and second == first
    s.close()


def test_noalloc_refuses_a_host_pointer(gpu_lib):
    """hrn_misfit takes a host pointer of the same C type; handing one to the
    no-alloc entry returns HRN_EARG and launches nothing."""
    p = tiny(nshot=1, nstep=60)
    s = _solver(p, "fp64", p["lam"], p["mu"])
    s.forward()
    dis = np.ascontiguousarray(s.traces())
    n0 = s.launch_count()
    out = C.c_double()
    rc = gpu_lib.hrn_misfit_noalloc(s.h, C.c_void_p(dis.ctypes.data), C.byref(out))
    assert rc == 1                          # HRN_EARG
    assert b"device" in gpu_lib.hrn_last_error(s.h)
    assert s.launch_count() == n0
    s.close()
