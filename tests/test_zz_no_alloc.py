"""sph_boundary_psi_noalloc: boundary volumes for callers that may not allocate
device memory (their framework owns the memory pool and forbids allocations
behind its back, or real-time code must not allocate after start-up).  The caller
owns every input and output buffer; the library uses only its fixed static
scratch.  This test checks, through the C ABI, that two calls in a row give
the psi that the allocating path (sph_set_boundary + sph_get_boundary)
computes, and that oversize input is refused before any GPU work.

Kept in its own file, collected last, so a failure here never hides the rest
of the suite; it must also pass alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from tests.helpers import normrel

pytestmark = pytest.mark.gpu


def _context_psi(params, bx):
    from warpsph_b200 import _lib
    from warpsph_b200.tables import kernel_tables

    L = _lib.load()
    ctx = ctypes.c_void_p()
    cp = params.to_c()
    _lib.check(None, L.sph_create(ctypes.byref(cp), ctypes.byref(ctx)))
    w, g = kernel_tables(params)
    _lib.check(ctx, L.sph_set_tables(ctx, _lib.ptr(w), len(w), _lib.ptr(g), len(g)))
    _lib.check(ctx, L.sph_set_boundary(ctx, _lib.ptr(bx), None, len(bx)))
    psi = np.zeros(len(bx), np.float32)
    _lib.check(ctx, L.sph_get_boundary(ctx, None, _lib.ptr(psi)))
    L.sph_destroy(ctx)
    return psi


def _sparse_wide_boundary():
    """Eight 12 x 12 x 3 plates of boundary particles (spacing 0.02 m) at the
    corners of a 6 m cube: about 7.8 M cells of the fine grid (h = 0.04 m),
    more than SPH_NOALLOC_MAX_CELLS, so the no-allocation path coarsens its
    grid while the context path keeps the fine one."""
    d = 0.02
    g = np.stack(np.meshgrid(np.arange(12), np.arange(3), np.arange(12), indexing="ij"), -1).reshape(-1, 3) * d
    plates = [g + np.array(c) for c in np.array(np.meshgrid([0, 6], [0, 6], [0, 6], indexing="ij")).reshape(3, -1).T]
    return np.ascontiguousarray(np.concatenate(plates), dtype=np.float32)


def _case(name):
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    if name == "sparse_wide":
        return preset_params("dam_break_8k"), _sparse_wide_boundary()
    if name == "dam_break_8k_domain":
        # an explicit grid extent (params.domain_*): no bounding-box readback
        params = preset_params("dam_break_8k", domain_min=(-0.1, -0.1, -0.1), domain_max=(1.1, 0.7, 0.5))
        return params, np.ascontiguousarray(preset_scene("dam_break_8k").boundary_x, dtype=np.float32)
    return preset_params(name), np.ascontiguousarray(preset_scene(name).boundary_x, dtype=np.float32)


@pytest.mark.parametrize("case", ["dam_break_8k", "dam_break_1m", "dam_break_8k_domain", "sparse_wide"])
def test_noalloc_psi_matches_allocating_path(case):
    import torch

    from warpsph_b200 import _lib
    from warpsph_b200.tables import kernel_tables

    params, bx = _case(case)
    ref = _context_psi(params, bx)

    L = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    d_x = torch.from_numpy(bx).to(dev)
    d_w = torch.from_numpy(kernel_tables(params)[0]).to(dev)
    cp = params.to_c()
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        d_psi = torch.full((len(bx),), float("nan"), dtype=torch.float32, device=dev)
        rc = L.sph_boundary_psi_noalloc(ctypes.byref(cp), ctypes.c_void_p(d_x.data_ptr()), len(bx),
                                        ctypes.c_void_p(d_w.data_ptr()), ctypes.c_void_p(d_psi.data_ptr()),
                                        ctypes.c_void_p(stream.cuda_stream))
        assert rc == _lib.SPH_OK, f"call {call}: rc {rc}"
        stream.synchronize()
        psi = d_psi.cpu().numpy()
        assert np.all(np.isfinite(psi)), f"call {call}"
        assert normrel(psi, ref) < 1e-5, f"call {call}"


def test_noalloc_rejects_oversize_input():
    from warpsph_b200 import _lib
    from warpsph_b200.params import SolverParams

    L = _lib.load()
    cp = SolverParams().to_c()
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    rc = L.sph_boundary_psi_noalloc(ctypes.byref(cp), fake, _lib.SPH_NOALLOC_MAX_BOUNDARY + 1, fake, fake, None)
    assert rc == _lib.SPH_E_TOO_LARGE


def test_noalloc_rejects_nonfinite_domain():
    from warpsph_b200 import _lib
    from warpsph_b200.params import SolverParams

    L = _lib.load()
    fake = ctypes.c_void_p(256)  # never dereferenced: the domain check comes first
    for bad in (float("nan"), float("inf")):
        cp = SolverParams(domain_min=(0.0, 0.0, 0.0), domain_max=(1.0, bad, 1.0)).to_c()
        rc = L.sph_boundary_psi_noalloc(ctypes.byref(cp), fake, 10, fake, fake, None)
        assert rc == _lib.SPH_E_INVALID
