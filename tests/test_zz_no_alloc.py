"""The allocation-free volume entry point, through the C-ABI.

Callers that cannot allocate device memory when they call the library (a
host code whose memory pool owns the whole GPU, or a time loop that must
not pay cudaMalloc's device synchronisation) use r3d_volume_dense_noalloc:
its scratch is a fixed array inside the library.  Its result must agree with
the allocating entry point r3d_volume within the 1e-12 relative tolerance of
the FP64 volume, on two calls in a row (the second call reuses the shared
array the first one left behind).  This file is collected last so that a
run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

import reef3d_b200 as r3d

pytestmark = pytest.mark.gpu


def test_noalloc_volume_matches_r3d_volume_twice(port_lib):
    import torch

    lib = r3d.load_library()
    nx, ny, nz = 48, 40, 36
    rng = np.random.default_rng(11)
    xn, yn, zn = r3d.uniform_nodes(nx), r3d.uniform_nodes(ny), r3d.uniform_nodes(nz)
    c = lambda a: 0.5 * (a[5:-6] + a[6:-5])  # interior cell centres
    X, Y, Z = np.meshgrid(c(xn), c(yn), c(zn), indexing="ij")
    base = np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2 + (Z - 0.55) ** 2) - 0.3
    psi = port_lib(nx, ny, nz, xn, yn, zn, f45=2.1).psi
    torch.cuda.set_device(0)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):
        phi = base + 0.01 * rng.standard_normal(base.shape)
        dense = np.ascontiguousarray(phi.transpose(2, 1, 0))  # index i + nx*(j + ny*k)
        with r3d.LevelSet(nx, ny, nz, xn, yn, zn, f45=2.1, precision=r3d.FP64) as ls:
            ls.upload(r3d.PHI, dense, layout=r3d.LAYOUT_DENSE)
            ref1, ref2 = ls.volume()
        dphi = torch.from_numpy(dense).to("cuda")
        rc = lib.r3d_volume_dense_noalloc(ctypes.c_void_p(dphi.data_ptr()), nx, ny, nz, 1.0 / nx, 1.0 / ny,
                                          1.0 / nz, psi, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == r3d.R3D_OK, lib.r3d_last_error(None)
        torch.cuda.synchronize()
        v1, v2 = out.cpu().tolist()
        assert abs(v1 - ref1) <= 1e-12 * abs(ref1), (call, v1, ref1)
        assert abs(v2 - ref2) <= 1e-12 * abs(ref2), (call, v2, ref2)

    # sizes beyond the fixed array are refused with a clear error
    rc = lib.r3d_volume_dense_noalloc(ctypes.c_void_p(dphi.data_ptr()), 4, 300, 300, 0.1, 0.1, 0.1, psi,
                                      ctypes.c_void_p(out.data_ptr()), None)
    assert rc == r3d.R3D_EINVAL
    assert b"65536" in lib.r3d_last_error(None)
