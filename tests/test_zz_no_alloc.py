"""The allocation-free Bouzidi entry point, for callers that cannot allocate
device memory (their memory is held by another allocator's pool, or their
loop must not allocate): called through the C ABI, it must give the same
result as ol_bouzidi_sparse with caller-owned scratch, on two calls in a row
(the shared library-owned scratch keeps the previous call's contents)."""
import ctypes as C

import numpy as np
import pytest

from helpers import perturbed_state, small_sphere_case

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from openludwig_b200 import _native as N  # noqa: E402

DEV = torch.device("cuda:0")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def test_noalloc_matches_caller_scratch_twice():
    c, mesh, p, hosts = small_sphere_case(resolution=8)
    h = hosts[0]
    n = h.n_blocks
    assert 0 < h.n_boundary <= 65536
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    arrs = {k: _t(getattr(h, k)) for k in ("cell_block", "cell_x", "cell_y", "cell_z",
                                           "neighbor_table")}
    q = _t(h.q_map.view(np.int16))
    scratch = torch.empty(27 * h.n_boundary, dtype=torch.float32, device=DEV)
    for seed in (21, 22):   # two calls in a row on different states
        f_post, _ = perturbed_state(n, seed=seed)
        a, b = _t(f_post), _t(f_post)
        N.call("ol_bouzidi_sparse", _ptr(a), _ptr(q), _ptr(arrs["cell_block"]),
               _ptr(arrs["cell_x"]), _ptr(arrs["cell_y"]), _ptr(arrs["cell_z"]),
               N.i32(h.n_boundary), _ptr(arrs["neighbor_table"]), N.i32(n), N.f32(0.001),
               _ptr(scratch), st)
        N.call("ol_bouzidi_sparse_noalloc", _ptr(b), _ptr(q), _ptr(arrs["cell_block"]),
               _ptr(arrs["cell_x"]), _ptr(arrs["cell_y"]), _ptr(arrs["cell_z"]),
               N.i32(h.n_boundary), _ptr(arrs["neighbor_table"]), N.i32(n), N.f32(0.001), st)
        torch.cuda.synchronize()
        ga, gb = a.cpu().numpy(), b.cpu().numpy()
        # same kernels, same arguments, only the scratch differs: same bits
        assert np.array_equal(gb, ga)
        assert not np.array_equal(gb, f_post)   # the correction was applied


def test_noalloc_rejects_oversize_lists():
    lib = N.lib()
    rc = lib.ol_bouzidi_sparse_noalloc(None, None, None, None, None, None, N.i32(65537), None,
                                       N.i32(1), N.f32(0.001), None)
    assert rc == 1
    assert b"exceed" in lib.ol_last_error()
