"""Batched Helmholtz single-layer sweep against one-at-a-time mixed-precision assembly:
three ellipsoidally stretched icospheres of uneven size, several wavenumbers in [1, 20];
complex64 output, relative Frobenius error <= 1e-6 per matrix and every entry within
1e-6 of the largest.  The sweep computes the tile pairs of one triangle and mirrors the
rest; the single assemblies here use two space objects, so they compute every pair."""

import numpy as np
import pytest

from bempp import shapes
from bempp.assembly.boundary import (BoundaryAssemblerOptions, OperatorType, Precision,
                                     create_helmholtz_assembler)
from bempp.function_space import function_space
from ndelement.ciarlet import Continuity, Family, create_family
from ndelement.reference_cell import ReferenceCellType
from ndgrid.grid import Grid

pytestmark = pytest.mark.gpu


def stretched(level, seed):
    pts, cells = shapes.icosphere(level)
    return Grid(shapes.ellipsoidal_stretch(pts, seed), cells)


def single(grid, k):
    import torch

    opts = BoundaryAssemblerOptions()
    opts.set_regular_quadrature_degree(ReferenceCellType.Triangle, 6)
    opts.set_precision(Precision.FP64)
    a = create_helmholtz_assembler(OperatorType.SingleLayer, k, opts)
    fam = create_family(Family.Lagrange, 0, Continuity.Discontinuous)
    sp, sp2 = function_space(grid, fam), function_space(grid, fam)  # every pair computed
    out = torch.empty((sp.global_size, sp.global_size), dtype=torch.complex128, device="cuda")
    a.assemble_into_device(sp2, sp, out, torch.cuda.current_stream().cuda_stream)
    return out


def test_sweep_matches_single_assemblies():
    import torch

    from bempp.sweep import helmholtz_single_layer_sweep, last_tuning

    grids = [stretched(1, 1280), stretched(3, 5120), stretched(2, 20480)]
    ks = np.linspace(1.0, 20.0, 5)
    outs = helmholtz_single_layer_sweep(grids, ks)
    outs2 = helmholtz_single_layer_sweep(grids, ks)  # graph replay
    torch.cuda.synchronize()
    for g, o, o2 in zip(grids, outs, outs2):
        assert torch.equal(o, o2)
        for j, k in enumerate(ks):
            ref = single(g, k)
            d = o[j].to(torch.complex128) - ref
            err = (torch.linalg.norm(d) / torch.linalg.norm(ref)).item()
            assert err <= 1e-6, (len(g.cells), k, err)
            # entrywise as well: the mirrored blocks' vertex-sharing entries (own Duffy rule)
            assert d.abs().max().item() <= 1e-6 * ref.abs().max().item(), (len(g.cells), k)
    kc, bps, ms, shape = last_tuning()
    assert kc >= 1 and bps >= 1 and ms > 0 and shape in (1, 2)


@pytest.mark.parametrize("kchunk,bps,shape", [(2, 6, 1), (4, 3, 2), (1, 2, 2)])
def test_every_tuner_candidate_shape_is_correct(kchunk, bps, shape):
    """The launch variants the autotuner chooses among (tile shape 1 x 1 or 2 x 2 tile
    pairs per work item, the 80- and 128-register builds): each fixed by hand must give
    the same matrices as the single assemblies."""
    import torch

    from bempp.sweep import helmholtz_single_layer_sweep, last_tuning, set_tuning

    grids = [stretched(2, 1280), stretched(3, 5120)]
    ks = np.array([2.0, 11.0, 19.5])
    set_tuning(kchunk, bps, shape)
    try:
        outs = helmholtz_single_layer_sweep(grids, ks)
        torch.cuda.synchronize()
        assert last_tuning()[0] == kchunk and last_tuning()[3] == shape
    finally:
        set_tuning(0)
    for g, o in zip(grids, outs):
        for j, k in enumerate(ks):
            ref = single(g, k)
            d = o[j].to(torch.complex128) - ref
            assert (torch.linalg.norm(d) / torch.linalg.norm(ref)).item() <= 1e-6
            assert d.abs().max().item() <= 1e-6 * ref.abs().max().item()
