"""The allocation-free batched eigensolver against the allocating one.

dvr3d_b200_diag_batched_noalloc exists for callers that may not allocate device memory
(a host inside a framework whose memory pool owns the GPU, or a latency-critical loop where
cudaMalloc and its device-wide synchronisation must not happen): it runs the same kernels as
dvr3d_b200_diag_batched with all scratch taken from a fixed array inside the library. This
file is collected last so that a run stopping at the first failure has run everything else.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from dvr3d_b200 import _abi

pytestmark = pytest.mark.gpu

SIZES = [1, 7, 40, 64, 129, 231, 300]


def _blocks(seed: int):
    rng = np.random.default_rng(seed)
    offs, woffs, flat, sym = [], [], [], []
    o = wo = 0
    for n in SIZES:
        a = rng.standard_normal((n, n))
        a = 0.5 * (a + a.T)
        sym.append(a.copy())
        a[np.triu_indices(n, 1)] = 1.0e3  # only the lower triangle is read
        flat.append(a.ravel(order="F"))
        offs.append(o)
        woffs.append(wo)
        o += n * n
        wo += n
    return offs, woffs, np.concatenate(flat), wo, sym


def _call(lib, handle, offs, woffs, flat, nw, noalloc: bool):
    import torch

    a = torch.tensor(flat, dtype=torch.float64, device="cuda")
    w = torch.zeros(nw, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    nb = len(SIZES)
    n_arr = (C.c_int * nb)(*SIZES)
    o_arr = (C.c_longlong * nb)(*offs)
    w_arr = (C.c_longlong * nb)(*woffs)
    if noalloc:
        rc = lib.dvr3d_b200_diag_batched_noalloc(None, nb, n_arr, o_arr, w_arr, C.c_void_p(a.data_ptr()),
                                                 C.c_void_p(w.data_ptr()), 1)
    else:
        rc = lib.dvr3d_b200_diag_batched(handle, nb, n_arr, o_arr, w_arr, C.c_void_p(a.data_ptr()),
                                         C.c_void_p(w.data_ptr()), 1)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return a.cpu().numpy(), w.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(ctx):
    lib = _abi.load_library()
    offs, woffs, flat, nw, sym = _blocks(11)
    a_ref, w_ref = _call(lib, ctx._h, offs, woffs, flat, nw, noalloc=False)
    for call in range(2):  # two calls in a row share the fixed scratch
        a_got, w_got = _call(lib, None, offs, woffs, flat, nw, noalloc=True)
        np.testing.assert_allclose(w_got, w_ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(a_got, a_ref, rtol=0, atol=1e-12)
        for b, n in enumerate(SIZES):
            w = w_got[woffs[b]:woffs[b] + n]
            z = a_got[offs[b]:offs[b] + n * n].reshape(n, n, order="F")
            np.testing.assert_allclose(w, np.linalg.eigvalsh(sym[b]), rtol=0, atol=1e-12)
            res = np.abs(sym[b] @ z - z * w).max()
            assert res < 1e-11, (call, n, res)
            assert np.abs(z.T @ z - np.eye(n)).max() < 1e-11


def test_noalloc_rejects_requests_beyond_its_scratch(ctx):
    lib = _abi.load_library()
    nb = 60  # 60 blocks of 1024 need ~3.4 GB of scratch
    n_arr = (C.c_int * nb)(*([1024] * nb))
    o_arr = (C.c_longlong * nb)(*[i * 1024 * 1024 for i in range(nb)])
    w_arr = (C.c_longlong * nb)(*[i * 1024 for i in range(nb)])
    rc = lib.dvr3d_b200_diag_batched_noalloc(None, nb, n_arr, o_arr, w_arr, C.c_void_p(16), C.c_void_p(16), 1)
    assert rc == _abi.DVR3D_ERR_SCRATCH
    assert b"64 MiB" in lib.dvr3d_b200_strerror(rc)
    # nothing ran; a valid request still works afterwards
    offs, woffs, flat, nw, sym = _blocks(3)
    a, w = _call(lib, None, offs, woffs, flat, nw, noalloc=True)
    np.testing.assert_allclose(w[woffs[-1]:], np.linalg.eigvalsh(sym[-1]), rtol=0, atol=1e-12)


def test_noalloc_rejects_more_blocks_than_one_launch_indexes(ctx):
    """Block counts beyond 65535 are refused on the host, before any device work (the
    copy-in launch indexes blocks by blockIdx.y); the caller's pointers are not touched."""
    lib = _abi.load_library()
    nb = 65536
    n_arr = (C.c_int * nb)(*([1] * nb))
    o_arr = (C.c_longlong * nb)(*range(nb))
    w_arr = (C.c_longlong * nb)(*range(nb))
    rc = lib.dvr3d_b200_diag_batched_noalloc(None, nb, n_arr, o_arr, w_arr, C.c_void_p(16), C.c_void_p(16), 1)
    assert rc == _abi.DVR3D_ERR_ARG
